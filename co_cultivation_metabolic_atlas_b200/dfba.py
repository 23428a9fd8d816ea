"""Device-resident dynamic FBA for the synthetic three-species community.

One ``DeviceCommunity.step`` is the reference simulator's step
(``src/dfba_simulator.py:1757-1797``) for every environment at once:

1. uptake bounds from the current medium (Michaelis-Menten with the
   physical-inventory cap, ``set_uptake_constraints`` ``:640-667``);
2. one batched LP solve of every (environment, species) FBA problem through
   the C ABI engine (all species in one persistent launch);
3. biomass Euler step (``update_biomass`` ``:1294-1324``, without the pH
   model, which the synthetic medium does not carry);
4. medium Euler step with the beginning-of-step biomass
   (``_update_environment`` ``:1326-1435``, ``integration_biomass`` ``:1680``).

With ``parsimonious=True`` every (environment, species) LP gets the
parsimonious second stage of ``parsimonious.py`` (weighted exchange fluxes
minimised at the stage-1 growth, a unique optimum) on a second engine, and
the Euler steps use its fluxes.

Everything stays on the GPU; the LP batch is laid out species-major
(all environments of species 0, then species 1, then species 2).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .engine import EngineOptions, LPEngine, SolveConfig, SolveResult

CARRYING_CAPACITY = 20.0


def uptake_lower(conc, total, dt, mm):
    """Michaelis-Menten uptake lower bounds of one species' medium exchanges
    (``set_uptake_constraints``, ``src/dfba_simulator.py:640-667``):
    ``conc`` (E, k) concentrations, ``total`` (E, 1) floored total biomass,
    ``mm`` the species' ``vmax``/``km``/original lower (``orig``)/upper
    (``ub``) rows; rounded to 6 decimals (``_safe_lb`` ``:553-563``)."""
    v_kin = mm["vmax"] * conc / (mm["km"] + conc)
    v_phys = torch.minimum(conc / (total * dt), mm["vmax"] * 10.0)
    limit = torch.minimum(v_kin, v_phys)
    lb = torch.clamp(torch.maximum(-limit, mm["orig"]), max=0.0)
    lb = torch.minimum(lb, mm["ub"])
    return torch.round(lb * 1e6) / 1e6


def euler_biomass(biomass, mu, capacity, dt):
    """Biomass Euler step (``update_biomass``, ``src/dfba_simulator.py:
    1294-1324``, without the pH model): growth clipped to [-0.5, 2],
    logistic capacity factor for positive growth."""
    mu = mu.clamp(-0.5, 2.0)
    total = biomass.sum(dim=1, keepdim=True)
    cap = torch.clamp(1.0 - total / capacity, min=0.0)
    dX = mu * biomass * torch.where(mu > 0, cap, torch.ones_like(cap)) * dt
    return torch.clamp(biomass + dX, 0.0, capacity)


@dataclass
class StepStats:
    lps: int
    certified: torch.Tensor      # scalar int64 (device)
    iterations: torch.Tensor     # int32 [lps] (device)
    status: torch.Tensor


class DeviceCommunity:
    """All environments of a synthetic community on one GPU."""

    def __init__(self, models, medium, biomass, *, dt=0.05, capacity=CARRYING_CAPACITY,
                 options: EngineOptions | None = None, config: SolveConfig | None = None,
                 warm_start: str = "previous", learned=None, horizon_steps: int = 960, device=None,
                 parsimonious: bool = False, stage2_config: SolveConfig | None = None):
        if warm_start not in ("cold", "previous", "extrapolate", "learned"):
            raise ValueError("warm_start must be 'cold', 'previous', 'extrapolate' or 'learned'")
        if warm_start == "learned" and learned is None:
            raise ValueError("warm_start='learned' needs a LearnedWarmStart")
        self.learned = learned
        self.horizon_steps = int(horizon_steps)
        self.step_index = 0
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        dev = self.device
        self.models = models
        self.dt = float(dt)
        self.capacity = float(capacity)
        self.config = config or SolveConfig()
        self.warm_start = warm_start
        E = medium.shape[0]
        self.E = E
        self.S = len(models)
        self.medium = torch.as_tensor(medium, dtype=torch.float64, device=dev).clone()
        self.biomass = torch.as_tensor(biomass, dtype=torch.float64, device=dev).clone()
        self.engine = LPEngine([(m.S, m.S.shape[0]) for m in models], options=options, device=dev)
        sid = np.repeat(np.arange(self.S, dtype=np.int32), E)
        co, ro, tc, tr = self.engine.layout(sid)
        self.species_id = sid
        self.col_offsets = torch.as_tensor(co, device=dev)
        self.total_cols, self.total_rows = tc, tr
        lower, upper, cost = [], [], []
        self.mm = []          # per species: flat column index tensor (E, k), medium ids, vmax, km, orig lb/ub
        self.bio_index = []   # flat index of every instance's biomass column
        base = 0
        for s, mdl in enumerate(models):
            n = mdl.S.shape[1]
            lower.append(np.tile(mdl.lower, E))
            upper.append(np.tile(mdl.upper, E))
            cost.append(np.tile(mdl.cost, E))
            starts = base + np.arange(E, dtype=np.int64) * n
            flat = starts[:, None] + mdl.medium_columns[None, :]
            self.mm.append(dict(
                flat=torch.as_tensor(flat, device=dev),
                ids=torch.as_tensor(mdl.medium_ids, device=dev),
                vmax=torch.as_tensor(mdl.vmax, device=dev)[None, :],
                km=torch.as_tensor(mdl.km, device=dev)[None, :],
                orig=torch.as_tensor(mdl.lower[mdl.medium_columns], device=dev)[None, :],
                ub=torch.as_tensor(mdl.upper[mdl.medium_columns], device=dev)[None, :]))
            self.bio_index.append(torch.as_tensor(starts + mdl.biomass, device=dev))
            base += E * n
        self.lower = torch.as_tensor(np.concatenate(lower), device=dev)
        self.upper = torch.as_tensor(np.concatenate(upper), device=dev)
        self.cost = torch.as_tensor(np.concatenate(cost), device=dev)
        self.engine.set_instances(sid, self.lower, self.upper, self.cost)
        self.result: SolveResult | None = None
        self.prev: SolveResult | None = None
        self.prev2: SolveResult | None = None
        self._bufs = [self.engine.allocate_result() for _ in range(3)]
        self._which = 0
        self._wx = self._wy = None
        self.parsimonious = bool(parsimonious)
        # the parsimonious LPs need 1e4 iterations where FBA needs 1e2-1e3
        self.stage2_config = stage2_config or SolveConfig(max_iterations=100_000, fp32_max_iterations=100_000)
        self.engine2 = None
        if self.parsimonious:
            self._init_stage2(options)

    # -- parsimonious second stage ----------------------------------------
    def _init_stage2(self, options):
        """Second engine with the stage-2 matrices ``[S 0; E -I; -E -I]``
        and the index maps between the two stages' flat layouts."""
        from .parsimonious import stage_cost, stage_matrix
        dev = self.device
        E, sid = self.E, self.species_id
        self.engine2 = LPEngine([(stage_matrix(m), m.S.shape[0]) for m in self.models], options=options, device=dev)
        co2, ro2, tc2, tr2 = self.engine2.layout(sid)
        co1 = self.col_offsets.cpu().numpy()
        _, ro1, _, _ = self.engine.layout(sid)
        vmap, tmap, ex1, ymap = [], [], [], []
        cost2, up_t = [], []
        bio1, bio2 = [], []
        for s, m in enumerate(self.models):
            r, n = m.S.shape
            k = m.n_exchange
            for e in range(E):
                i = s * E + e
                vmap.append(co2[i] + np.arange(n))
                tmap.append(co2[i] + n + np.arange(k))
                ex1.append(co1[i] + np.arange(k))
                ymap.append(ro2[i] + np.arange(r))
                bio1.append(co1[i] + m.biomass)
                bio2.append(co2[i] + m.biomass)
            cost2.append(np.tile(stage_cost(m, s), E))
        t = lambda a: torch.as_tensor(np.concatenate(a) if isinstance(a, list) else a, device=dev)  # noqa: E731
        self._vmap, self._tmap, self._ex1, self._ymap = (t(vmap).long(), t(tmap).long(), t(ex1).long(),
                                                         t(ymap).long())
        self._bio1, self._bio2 = t(np.asarray(bio1)).long(), t(np.asarray(bio2)).long()
        self.lower2 = torch.zeros(tc2, dtype=torch.float64, device=dev)
        self.upper2 = torch.zeros(tc2, dtype=torch.float64, device=dev)
        self.cost2 = t(cost2).double()
        self.total_cols2, self.total_rows2 = tc2, tr2
        self._stage2_bounds()
        self.upper2.index_put_((self._vmap,), self.upper)
        self.engine2.set_instances(sid, self.lower2, self.upper2, self.cost2)
        self._bufs2 = [self.engine2.allocate_result() for _ in range(3)]
        self.prev_p = self.prev2_p = None
        self._wx2 = torch.zeros(tc2, dtype=torch.float64, device=dev)
        self._wy2 = torch.zeros(max(1, tr2), dtype=torch.float64, device=dev)

    def _stage2_bounds(self, growth=None):
        """Stage-2 bounds from the current stage-1 bounds (and the stage-1
        growth fluxes, ``(E S,)`` in the batch order): ``parsimonious.
        stage_bounds`` on the device."""
        from .parsimonious import GROWTH_FLOOR_ABS, GROWTH_RELAXATION
        self.lower2.index_put_((self._vmap,), self.lower)
        lo_ex = self.lower[self._ex1]
        self.upper2.index_put_((self._tmap,), torch.maximum(lo_ex.abs(), self.upper[self._ex1].abs()))
        if growth is not None:
            floor = torch.maximum(self.lower[self._bio1], growth * (1.0 - GROWTH_RELAXATION) - GROWTH_FLOOR_ABS)
            self.lower2.index_put_((self._bio2,), torch.minimum(floor, self.upper[self._bio1]))

    def solve_stage2(self, res: SolveResult) -> SolveResult:
        """The parsimonious second stage of every LP of the step, warm
        started from the last two stage-2 solutions (extrapolated) or, at
        the first step, from stage 1's solution with ``t = |v_exchange|``."""
        self._stage2_bounds(res.x[self._bio1])
        # the buffer index of this step's stage-1 result (``solve`` has
        # advanced the rotation already)
        out = self._bufs2[(self._which + 2) % 3]
        nc, nr = self.total_cols2, self.total_rows2
        self.engine2.set_iteration_hints(None if self.prev_p is None else self.prev_p.iterations)
        if self.prev_p is not None:
            if self.prev2_p is not None:
                torch.sub(self.prev_p.x[:nc] * 2.0, self.prev2_p.x[:nc], out=self._wx2)
                torch.sub(self.prev_p.y[:nr] * 2.0, self.prev2_p.y[:nr], out=self._wy2[:nr])
            else:
                self._wx2.copy_(self.prev_p.x[:nc])
                self._wy2[:nr].copy_(self.prev_p.y[:nr])
            omega = self.prev_p.omega
        else:
            self._wx2.zero_()
            self._wx2.index_put_((self._vmap,), res.x[:self.total_cols])
            self._wx2.index_put_((self._tmap,), res.x[self._ex1].abs())
            self._wy2.zero_()
            self._wy2.index_put_((self._ymap,), res.y[:self.total_rows])
            omega = res.omega
        res2 = self.engine2.solve(warm_x=self._wx2, warm_y=self._wy2[:nr], warm_omega=omega,
                                  config=self.stage2_config, out=out)
        self.prev2_p, self.prev_p = self.prev_p, res2
        return res2

    def stage2_fluxes(self, res2: SolveResult):
        """Stage-2 fluxes in stage 1's flat layout."""
        return res2.x.index_select(0, self._vmap)

    # -- pieces of one step --------------------------------------------------
    def uptake_bounds(self):
        """Write Michaelis-Menten uptake bounds into the bound batch."""
        total = self.biomass.clamp_min(1e-6).sum(dim=1, keepdim=True)          # (E, 1)
        for mm in self.mm:
            lb = uptake_lower(self.medium[:, mm["ids"]], total, self.dt, mm)
            self.lower.index_put_((mm["flat"].reshape(-1),), lb.reshape(-1))

    def solve(self):
        out = self._bufs[self._which]
        # the previous step's iteration counts tell the kernel which
        # instances need no early termination tests
        self.engine.set_iteration_hints(None if self.prev is None else self.prev.iterations)
        if self.warm_start == "learned":
            wx, wy, wo = self.learned.propose(self, self.step_index / self.horizon_steps)
            res = self.engine.solve(warm_x=wx, warm_y=wy, warm_omega=wo, config=self.config, out=out)
        elif self.warm_start == "extrapolate" and self.prev is not None and self.prev2 is not None:
            # first-order prediction from the last two certified solutions
            # (the kernel projects x onto the new bounds and y_ub onto <= 0)
            if self._wx is None:
                self._wx = torch.empty(self.total_cols, dtype=torch.float64, device=self.device)
                self._wy = torch.empty(max(1, self.total_rows), dtype=torch.float64, device=self.device)
            torch.sub(self.prev.x[:self.total_cols] * 2.0, self.prev2.x[:self.total_cols], out=self._wx)
            torch.sub(self.prev.y[:self.total_rows] * 2.0, self.prev2.y[:self.total_rows],
                      out=self._wy[:self.total_rows])
            res = self.engine.solve(warm_x=self._wx, warm_y=self._wy[:self.total_rows], warm_omega=self.prev.omega,
                                    config=self.config, out=out)
        else:
            warm = self.prev if (self.warm_start in ("previous", "extrapolate") and self.prev is not None) else None
            res = self.engine.solve(warm_x=None if warm is None else warm.x[:self.total_cols],
                                    warm_y=None if warm is None else warm.y[:self.total_rows],
                                    warm_omega=None if warm is None else warm.omega,
                                    config=self.config, out=out)
        self._which = (self._which + 1) % 3
        self.prev2 = self.prev
        self.prev = res
        self.result = res
        return res

    def integrate(self, res: SolveResult, x=None):
        """Euler biomass and medium updates from the solved fluxes (``x``
        in stage 1's flat layout; default ``res.x``)."""
        x = res.x if x is None else x
        E = self.E
        mu = torch.stack([x[idx] for idx in self.bio_index], dim=1)            # (E, S)
        X0 = self.biomass.clone()
        # state tensors are updated in place: their addresses stay fixed, so
        # a captured step replays on the current state
        self.biomass.copy_(euler_biomass(self.biomass, mu, self.capacity, self.dt))
        delta = torch.zeros_like(self.medium)
        for s, mm in enumerate(self.mm):
            v = x[mm["flat"]]                                                   # (E, k)
            contrib = v * X0[:, s:s + 1] * self.dt
            delta.index_add_(1, mm["ids"], contrib)
        self.medium.copy_(torch.clamp(self.medium + delta, min=0.0))
        self.step_index += 1

    @staticmethod
    def certified_mask(res: SolveResult):
        mt = res.metrics
        return (res.status == 0) & (mt[:, 0] <= 1e-5) & (mt[:, 1] <= 1e-7) & (mt[:, 2] <= 1e-7)

    def certified(self, res: SolveResult):
        """Count of LPs that meet the engine's FP64 tolerances AND the
        reference's certificate gate (primal <= 1e-5, dual <= 1e-7, relative
        KKT gap <= 1e-7, ``src/gpu_block_lp.py:84``) -- on the device."""
        return self.certified_mask(res).sum()

    def step(self) -> StepStats:
        """One dFBA step: a captured graph's replay after ``capture``,
        otherwise eager launches."""
        if getattr(self, "_graphs", None):
            return self._graph_step()
        return self._eager_step()

    # -- CUDA-graph-captured steps ---------------------------------------
    def capture(self):
        """Capture the next three dFBA steps as CUDA graphs (uptake bounds,
        the engine's launches, Euler updates, certified count); ``step``
        then replays them in turn.  Three graphs because a step reads the
        result buffers of the two previous steps and writes the third, in a
        rotation of period three; each graph bakes its buffers' addresses.
        Needs two eager steps first (the warm-start history exists and the
        engine's workspace is allocated) and a warm start that does not call
        the network (it runs only at an environment's first step)."""
        if self.prev is None or self.prev2 is None:
            raise RuntimeError("run two steps before capturing")
        if self.warm_start == "learned" and self.prev is None:
            raise RuntimeError("the network's first-step seed is not captured")
        if self.warm_start == "extrapolate" and self._wx is None:
            raise RuntimeError("run a warm-started step before capturing")
        saved = (self.step_index, self.prev, self.prev2, self.result, self._which,
                 getattr(self, "prev_p", None), getattr(self, "prev2_p", None))
        old_stream = self.engine.stream
        self._graphs, self._graph_stats = [], []
        torch.cuda.synchronize(self.device)
        # graph k brackets its PDHG launches by the engine's timing slot k
        self.engine.timing_slots(3)
        try:
            for k in range(3):
                g = torch.cuda.CUDAGraph()
                self.engine.use_timing_slot(k)
                with torch.cuda.graph(g):
                    self.engine.set_stream(torch.cuda.current_stream(self.device))
                    if self.engine2 is not None:
                        self.engine2.set_stream(torch.cuda.current_stream(self.device))
                    st = self._eager_step()
                self._graphs.append(g)
                self._graph_stats.append(st)
        finally:
            self.engine.use_timing_slot(-1)
            self.engine.set_stream(old_stream)
            if self.engine2 is not None:
                self.engine2.set_stream(old_stream)
            # capture ran nothing: the state is where it was
            (self.step_index, self.prev, self.prev2, self.result, self._which, self.prev_p,
             self.prev2_p) = saved
        self._replay = 0

    def last_replay_slot(self, back: int = 0):
        """Timing slot (the graph index) of the step replayed ``back`` steps
        before the last one."""
        return (self._replay - 1 - back) % 3

    def release_graphs(self):
        self._graphs, self._graph_stats = [], []

    def _eager_step(self) -> StepStats:
        self.uptake_bounds()
        res = self.solve()
        if not self.parsimonious:
            self.integrate(res)
            return StepStats(lps=self.E * self.S, certified=self.certified(res),
                             iterations=res.iterations, status=res.status)
        res2 = self.solve_stage2(res)
        self.integrate(res, self.stage2_fluxes(res2))
        cert = self.certified_mask(res).sum() + self.certified_mask(res2).sum()
        return StepStats(lps=2 * self.E * self.S, certified=cert,
                         iterations=torch.cat([res.iterations, res2.iterations]),
                         status=torch.cat([res.status, res2.status]))

    def _graph_step(self) -> StepStats:
        k = self._replay
        self._graphs[k].replay()
        res = self._bufs[self._which]
        if self.parsimonious:
            self.prev2_p, self.prev_p = self.prev_p, self._bufs2[self._which]
        self._which = (self._which + 1) % 3
        self.prev2, self.prev, self.result = self.prev, res, res
        self.step_index += 1
        self._replay = (k + 1) % 3
        return self._graph_stats[k]

    def close(self):
        self.release_graphs()
        self.engine.close()
        if self.engine2 is not None:
            self.engine2.close()
