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
                 warm_start: str = "previous", learned=None, horizon_steps: int = 960, device=None):
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

    def integrate(self, res: SolveResult):
        """Euler biomass and medium updates from the solved fluxes."""
        x = res.x
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

    def certified(self, res: SolveResult):
        """Count of LPs that meet the engine's FP64 tolerances AND the
        reference's certificate gate (primal <= 1e-5, dual <= 1e-7, relative
        KKT gap <= 1e-7, ``src/gpu_block_lp.py:84``) -- on the device."""
        mt = res.metrics
        ok = (res.status == 0) & (mt[:, 0] <= 1e-5) & (mt[:, 1] <= 1e-7) & (mt[:, 2] <= 1e-7)
        return ok.sum()

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
        saved = (self.step_index, self.prev, self.prev2, self.result, self._which)
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
                    st = self._eager_step()
                self._graphs.append(g)
                self._graph_stats.append(st)
        finally:
            self.engine.use_timing_slot(-1)
            self.engine.set_stream(old_stream)
            # capture ran nothing: the state is where it was
            self.step_index, self.prev, self.prev2, self.result, self._which = saved
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
        self.integrate(res)
        return StepStats(lps=self.E * self.S, certified=self.certified(res),
                         iterations=res.iterations, status=res.status)

    def _graph_step(self) -> StepStats:
        k = self._replay
        self._graphs[k].replay()
        res = self._bufs[self._which]
        self._which = (self._which + 1) % 3
        self.prev2, self.prev, self.result = self.prev, res, res
        self.step_index += 1
        self._replay = (k + 1) % 3
        return self._graph_stats[k]

    def close(self):
        self.release_graphs()
        self.engine.close()
