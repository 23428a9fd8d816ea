"""Drop-in ``solve_batch`` backend for the dFBA rollout.

``B200LPBackend`` has the public contract of the reference's batched GPU LP
service ``TemporalGpuLPBackend`` (``src/temporal_gpu_lp.py:18-199``) and of
the CPU comparator ``RepeatedCpuLP.solve_batch``
(``src/cpu_repeated_lp.py:783-818``):

* ``solve_batch(requests, *, environment_ids=None) -> list[row]`` where each
  request is ``(c, linprog_kwargs)`` and each row is a ``SimpleNamespace``
  with ``success``, ``x``, ``fun``, ``message``, ``diagnostics`` (plus ``y``,
  the HiGHS-convention row duals, and ``status``).  ``x``/``fun``/``y`` are
  ``None`` when ``success`` is False (``src/temporal_gpu_lp.py:174-180``);
  a failed solve is never replaced by a CPU solve.
* ``reset(environment_ids=None)`` clears per-environment warm-start state
  (``src/temporal_gpu_lp.py:72-84``).
* ``name``, ``method``, ``history`` attributes.
* invalid input raises ``ValueError`` before any state changes; an exception
  during solving does not advance per-environment state
  (``src/temporal_gpu_lp.py:182-186``).

Success means: the engine's FP64 tolerances are met (status OPTIMAL) AND the
reference's original-LP certificate gate passes on the returned primal/dual
pair (``primal <= 1e-5, dual <= 1e-7, relative KKT gap <= 1e-7``,
``src/gpu_block_lp.py:84``).

With ``equality_reduction=True`` (the reference's ``equality_reduction``
option, ``src/temporal_gpu_lp.py:22-52``) each request is presolved by the
exact homogeneous-equality reduction (``reduction.py``; one plan per
equality block), the reduced LPs are solved on the GPU, and the primal is
expanded and the duals lifted back; the row is accepted only when the
original-LP certificate passes on the lifted pair.

Requests stopped by the iteration cap get one more GPU pass, alone, from
their own iterates, of up to ``retry_iterations`` (default 1,000,000; 0
disables) iterations; cold genome-scale LPs need 10^5 to 7 x 10^5
iterations, far above the first pass's budget.  A row is still accepted only on its certificate.

With ``split_rows=L`` (off by default) rows longer than ``L`` (the hub
metabolites of genome-scale models hold up to ~1,200 reactions) are split
exactly into segments with auxiliary variables (``rowsplit.py``) before the
solve, so that no slice of the kernel walks or pads to a thousand-entry row;
the solution is restricted back and accepted only on the original LP's
certificate.  Measured on the reference's five consortium models: the split
solves are ~12x faster, but the restricted duals (one per row where the
split LP has one per segment) miss the 1e-7 KKT-gap gate on most LPs
(relative gaps 1.6e-7 to 9.5e-6), so those rows fail closed.
"""

from __future__ import annotations

import time
from types import SimpleNamespace

import numpy as np
import torch

from . import _native as N
from .engine import EngineOptions, LPEngine, SolveConfig
from .lp_trace import certificate as original_certificate
from .problem import matrix_key, normalize_batch
from .reduction import EqualityReduction
from .rowsplit import RowSplit

PRIMAL_GATE = 1e-5
DUAL_GATE = 1e-7
GAP_GATE = 1e-7


class B200LPBackend:
    name = 'b200_batched_halpern_pdhg'
    method = 'species_shared_persistent_halpern_pdhg_fp32_fp64'

    def __init__(self, *, mode='previous', precision='mixed', iterations=20000,
                 fp32_iterations=20000, check_interval=64, stage=None,
                 options: EngineOptions | None = None, warm_start_model=None, device=None,
                 equality_reduction=False, split_rows=None, retry_iterations=1_000_000):
        if mode not in ('cold', 'previous', 'mlp'):
            raise ValueError('Unknown warm-start mode')
        if mode == 'mlp' and warm_start_model is None:
            raise ValueError('mode="mlp" needs a warm_start_model')
        for name, value in (('iterations', iterations), ('fp32_iterations', fp32_iterations),
                            ('check_interval', check_interval)):
            if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, np.integer)):
                raise ValueError(f'{name} must be an integer')
        if iterations < 0 or fp32_iterations < 0 or check_interval < 1:
            raise ValueError('Invalid correction budget')
        if not torch.cuda.is_available():
            raise RuntimeError('CUDA is required (no CPU fallback)')
        self.mode = mode
        self.stage = stage
        self.config = SolveConfig(precision=precision, max_iterations=int(iterations),
                                  fp32_max_iterations=int(fp32_iterations),
                                  check_every=int(check_interval))
        self.config.native()  # validates
        self.options = options or EngineOptions()
        self.device = torch.device(device) if device is not None else torch.device('cuda')
        self.model = warm_start_model
        if mode == 'mlp' and equality_reduction:
            raise ValueError('the learned warm start proposes original-space points; use equality_reduction=False')
        self.equality_reduction = bool(equality_reduction)
        if split_rows is not None and (isinstance(split_rows, (bool, np.bool_)) or
                                       not isinstance(split_rows, (int, np.integer)) or split_rows < 2):
            raise ValueError('split_rows must be None or an integer >= 2')
        self.split_rows = None if split_rows is None else int(split_rows)
        self._split_plans: dict = {}
        if isinstance(retry_iterations, (bool, np.bool_)) or not isinstance(retry_iterations, (int, np.integer)) \
                or retry_iterations < 0:
            raise ValueError('retry_iterations must be a non-negative integer')
        self.retry_iterations = int(retry_iterations)
        self._plans: dict = {}
        self._keys: list[str] = []
        self._matrices = []
        self._engine: LPEngine | None = None
        self._staging: dict = {}
        self.last_certified: dict = {}
        self.history: list[dict] = []

    def _pinned(self, name, size, dtype):
        """A pinned host buffer kept across calls (grown when a batch needs
        more): pinning a fresh copy of every batch array each call costs
        more than the copy itself."""
        buf = self._staging.get(name)
        if buf is None or buf.dtype != dtype or buf.numel() < size:
            buf = torch.empty(max(1, int(size * 1.25)), dtype=dtype, pin_memory=True)
            self._staging[name] = buf
        return buf[:size]

    def _to_device(self, name, a):
        """Host array -> device through the named pinned staging buffer.  The
        copy is asynchronous; the buffer is not rewritten before the solve's
        results are read back (a synchronisation) in the same call."""
        a = np.asarray(a, dtype=np.float64)
        buf = self._pinned(name, a.size, torch.float64)
        buf.numpy()[:] = a.ravel()
        return buf.to(self.device, non_blocking=True)

    def _to_host(self, name, t):
        """Device tensor -> NumPy through the named pinned staging buffer."""
        buf = self._pinned(name, t.numel(), t.dtype)
        buf.copy_(t.reshape(-1))
        return buf.numpy().reshape(tuple(t.shape))

    # ------------------------------------------------------------------
    def reset(self, environment_ids=None):
        ids = None if environment_ids is None else list(environment_ids)
        if ids is not None and len(set(ids)) != len(ids):
            raise ValueError('Reset requires unique environment IDs')
        if ids is None:
            self.last_certified.clear()
        else:
            for env in ids:
                self.last_certified.pop(env, None)
        if self.mode == 'mlp':
            self.model.reset(ids)

    @staticmethod
    def _matrix_keys(problems):
        """Content key of every request's matrix, hashed once per distinct
        canonical matrix object (``normalize_batch`` shares one object among
        requests that passed the same matrices)."""
        memo = {}
        out = []
        for p in problems:
            k = memo.get((id(p[0]), p[5]))
            if k is None:
                k = memo[(id(p[0]), p[5])] = matrix_key(p[0], p[5])
            out.append(k)
        return out

    def _engine_for(self, problems):
        keys = self._matrix_keys(problems)
        new = [(k, p) for k, p in zip(keys, problems) if k not in self._keys]
        rebuilt = False
        if new:
            seen = set()
            for k, p in new:
                if k in seen:
                    continue
                seen.add(k)
                self._keys.append(k)
                self._matrices.append((p[0], p[5]))
            if self._engine is not None:
                self._engine.close()
            self._engine = LPEngine(self._matrices, options=self.options, device=self.device)
            rebuilt = True
        index = {k: i for i, k in enumerate(self._keys)}
        return np.array([index[k] for k in keys], dtype=np.int32), rebuilt, keys

    def solve_batch(self, requests, *, environment_ids=None):
        started = time.perf_counter()
        ids = list(range(len(requests))) if environment_ids is None else list(environment_ids)
        if not requests or len(ids) != len(requests) or len(set(ids)) != len(ids):
            raise ValueError('Nonempty requests and unique environment IDs required')
        originals = normalize_batch(requests)
        if self.stage is not None and any(kw.get('_stage', self.stage) != self.stage for _, kw in requests):
            raise ValueError('Use a separate backend and history for each LP stage')
        reduced = self._reduce(originals) if self.equality_reduction else None
        problems = originals if reduced is None else [r.problem if r is not None else o
                                                        for r, o in zip(reduced, originals)]
        splits = self._splits(problems)
        problems = [sp.split_problem(p) if sp is not None else p for sp, p in zip(splits, problems)]
        prep = time.perf_counter()
        species, rebuilt, keys = self._engine_for(problems)
        eng = self._engine
        lower = np.concatenate([p[2] for p in problems])
        upper = np.concatenate([p[3] for p in problems])
        cost = np.concatenate([p[4] for p in problems])
        rhs = np.concatenate([p[1] for p in problems])
        co, ro, tc, tr = eng.layout(species)
        warm_x = warm_y = warm_o = None
        if self.mode == 'previous':
            wx = np.zeros(tc)
            wy = np.zeros(tr)
            wo = np.ones(len(ids))
            for i, env in enumerate(ids):
                prev = self.last_certified.get(env)
                if prev is not None and prev[0] == species[i]:
                    n = eng.shapes[species[i]][1]
                    m = eng.shapes[species[i]][0]
                    px, py = prev[1], prev[2]
                    if reduced is not None and reduced[i] is not None:
                        px = reduced[i].compress_primal(px)
                        py = py[reduced[i].plan.kept_rows]
                    if splits[i] is not None:
                        px, py = splits[i].extend_primal(px), splits[i].extend_dual(py)
                    wx[co[i]:co[i] + n] = px
                    wy[ro[i]:ro[i] + m] = py
                    wo[i] = prev[3]
            warm_x, warm_y, warm_o = wx, wy, wo
        elif self.mode == 'mlp':
            warm_x, warm_y, warm_o = self.model.propose(ids, problems, species, eng, keys=keys)
        d = self._to_device
        if warm_x is not None and isinstance(warm_x, torch.Tensor):
            wxd, wyd, wod = warm_x, warm_y, warm_o    # proposed on the device (learned warm start)
        else:
            wxd = None if warm_x is None else d('warm_x', warm_x)
            wyd = None if warm_y is None or not tr else d('warm_y', warm_y)
            wod = None if warm_o is None else d('warm_omega', warm_o)
        eng.set_instances(species, d('lower', lower), d('upper', upper), d('cost', cost),
                          d('rhs', rhs) if tr else None)
        res = eng.solve(warm_x=wxd, warm_y=wyd if tr else None, warm_omega=wod, config=self.config)
        status = self._to_host('status', res.status).copy()
        iters = self._to_host('iterations', res.iterations).copy()
        metrics = self._to_host('metrics', res.metrics).copy()
        # x and y stay in the staging buffers: every row copies its slice
        # before the next call can rewrite them
        x = self._to_host('x', res.x[:tc])
        y = self._to_host('y', res.y[:tr]) if tr else np.zeros(0)
        # (the retry pass is rare: plain transfers)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)  # noqa: E731
        retried = self._retry(eng, res, species, co, ro, lower, upper, cost, rhs, tr, status, iters, metrics, x, y, t)
        solved = time.perf_counter()
        rows = []
        certified = {}
        for i, env in enumerate(ids):
            n = eng.shapes[species[i]][1]
            m = eng.shapes[species[i]][0]
            mt = metrics[i]
            gate = bool(status[i] == N.STATUS_OPTIMAL and mt[0] <= PRIMAL_GATE and mt[1] <= DUAL_GATE
                        and mt[2] <= GAP_GATE)
            xi = x[co[i]:co[i] + n].copy()
            yi = y[ro[i]:ro[i] + m].copy()
            cert = dict(primal_residual=float(mt[0]), dual_violation=float(mt[1]),
                        relative_kkt_gap=float(mt[2]))
            note = None
            if splits[i] is not None:
                # back to the unsplit LP; the kernel's metrics were the split LP's
                xi, yi = splits[i].restrict(xi, yi)
                if reduced is None:
                    cert = original_certificate(originals[i], xi, yi)
                    gate = gate and cert.pop('certificate_passed')
            if reduced is not None:
                if reduced[i] is None:
                    gate, note = False, 'bounds infeasible under the eliminated equalities'
                else:
                    # expand and lift, then certify the ORIGINAL LP
                    xi, yi, cert, ok = self._postsolve(reduced[i], originals[i], xi, yi)
                    gate = gate and ok
            diag = dict(cert, objective=float(mt[3]),
                        dual_objective=float(mt[4]), relative_gap=float(mt[5]),
                        certificate_passed=gate, accepted_iteration=int(iters[i]) if gate else -1,
                        iterations=int(iters[i]), status=N.STATUS_NAMES.get(int(status[i]), 'unknown'),
                        environment_id=env, stage=self.stage, success=gate, cpu_lp_calls=0,
                        mode=self.mode, solver=self.name, equality_reduction=reduced is not None)
            if gate:
                certified[env] = (species[i], xi, yi, float(mt[7]))
            rows.append(SimpleNamespace(
                success=gate, x=xi if gate else None, y=yi if gate else None,
                fun=float(originals[i][4] @ xi) if gate else None, status=int(status[i]),
                message=('Original-LP certified GPU solution' if gate else
                         f'GPU solve not certified ({note or diag["status"]}); no CPU fallback'),
                diagnostics=diag))
        # commit per-environment state only after every row is built
        for env in ids:
            if env in certified:
                self.last_certified[env] = certified[env]
            else:
                self.last_certified.pop(env, None)
        if self.mode == 'mlp':
            self.model.commit(ids, {env: (v[1], v[2], v[3]) for env, v in certified.items()}, keys)
        self.history.append(dict(stage=self.stage, mode=self.mode, batch=len(ids), environment_ids=ids,
                                 accepted=sum(r.success for r in rows), cpu_lp_calls=0,
                                 engine_rebuilt=rebuilt, iterations=iters.tolist(), retried=retried,
                                 host_preparation_seconds=prep - started,
                                 solve_seconds=solved - prep,
                                 total_seconds=time.perf_counter() - started,
                                 rows=[r.diagnostics for r in rows]))
        return rows

    def _retry(self, eng, res, species, co, ro, lower, upper, cost, rhs, tr, status, iters, metrics, x, y, t):
        """Requests stopped by the iteration cap continue on the GPU, alone,
        from their own iterates for up to ``retry_iterations`` more; their
        results replace the first pass's (host arrays, in place).  Returns
        the retried request indices."""
        lag = np.flatnonzero(status == N.STATUS_ITERATION_LIMIT)
        if self.retry_iterations == 0 or lag.size == 0:
            return []
        cols = [np.arange(co[i], co[i] + eng.shapes[species[i]][1]) for i in lag]
        rows = [np.arange(ro[i], ro[i] + eng.shapes[species[i]][0]) for i in lag]
        ci, ri = np.concatenate(cols), np.concatenate(rows) if tr else np.empty(0, np.int64)
        eng.set_instances(species[lag], t(lower[ci]), t(upper[ci]), t(cost[ci]), t(rhs[ri]) if tr else None)
        # a continuation: the FP32-valued re-centred phase from the first
        # pass's iterates (no BF16 phase, no cold fallback)
        cfg = SolveConfig(**{**self.config.__dict__, 'max_iterations': self.retry_iterations,
                             'fp32_max_iterations': self.retry_iterations, 'fp32_values_phase': 2,
                             'fallback_iterations': 0})
        r2 = eng.solve(warm_x=res.x[torch.as_tensor(ci, device=res.x.device)],
                       warm_y=res.y[torch.as_tensor(ri, device=res.y.device)] if tr else None,
                       warm_omega=res.omega[torch.as_tensor(lag, device=res.omega.device)], config=cfg)
        status[lag] = r2.status.cpu().numpy()
        iters[lag] += r2.iterations.cpu().numpy()
        metrics[lag] = r2.metrics.cpu().numpy()
        x[ci] = r2.x.cpu().numpy()[:ci.size]
        if tr:
            y[ri] = r2.y.cpu().numpy()[:ri.size]
        return lag.tolist()

    def _splits(self, problems):
        """The long-row split plan of every request's matrix (built once per
        matrix), or None where no row exceeds ``split_rows``."""
        if self.split_rows is None or self.mode == 'mlp':
            # the learned warm start proposes points of the unsplit LPs
            return [None] * len(problems)
        out = []
        for p, key in zip(problems, self._matrix_keys(problems)):
            if key not in self._split_plans:
                plan = RowSplit(p[0], p[5], max_length=self.split_rows)
                self._split_plans[key] = plan if plan.active else None
            out.append(self._split_plans[key])
        return out

    def _reduce(self, originals):
        """Reduce every request with the plan of its equality block (built
        once per block); a request whose bounds are infeasible under the
        eliminated equalities maps to None (a failed row)."""
        out = []
        for p, key in zip(originals, self._matrix_keys(originals)):
            plan = self._plans.get(key)
            if plan is None:
                plan = self._plans[key] = EqualityReduction(p)
            try:
                out.append(plan.reduce(p))
            except ValueError as exc:
                if 'infeasible' not in str(exc):
                    raise
                out.append(None)
        return out

    @staticmethod
    def _postsolve(red, original, z, y_red):
        """Original-space primal and duals of a reduced solution and the
        original-LP certificate of the pair."""
        ra, _, _, _, rc, _ = red.problem
        x = red.expand_primal(z)
        try:
            y = red.lift_dual(y_red, rc - np.asarray(ra.T @ y_red).ravel())
        except (ValueError, ArithmeticError):
            return x, np.full(original[0].shape[0], np.nan), dict(primal_residual=np.inf, dual_violation=np.inf,
                                                                  relative_kkt_gap=np.inf), False
        cert = original_certificate(original, x, y)
        ok = cert.pop('certificate_passed')
        return x, y, cert, ok

    def close(self):
        if self._engine is not None:
            self._engine.close()
            self._engine = None
        self._staging.clear()  # the pinned host buffers
