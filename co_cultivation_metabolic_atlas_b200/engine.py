"""Batched LP engine over the C ABI (device tensors via PyTorch).

``LPEngine`` is the tensor-level interface: species matrices are registered
once; a batch binds flat per-instance bound/objective tensors; ``solve`` runs
the persistent CUDA kernels and returns device tensors.  The reference's
equivalent is ``GpuPdhgCorrector`` + ``GpuPdhgWorkspace``
(``src/gpu_pdhg_corrector.py:75-438``, ``src/gpu_pdhg_workspace.py:55-384``),
which rebuild a block-diagonal copy of every matrix per call; here each
species matrix is stored once and shared by all of its instances.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch
from scipy.sparse import csr_matrix

from . import _native as N


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


@dataclass
class SolveResult:
    status: torch.Tensor       # int32 [count]
    objective: torch.Tensor    # float64 [count]
    x: torch.Tensor            # float64 [total_cols]
    y: torch.Tensor            # float64 [total_rows]
    iterations: torch.Tensor   # int32 [count]
    metrics: torch.Tensor      # float64 [count, 8]
    omega: torch.Tensor        # float64 [count]


@dataclass
class SolveConfig:
    precision: str = "mixed"           # "fp64" | "mixed" | "fp32"
    max_iterations: int = 20000
    fp32_max_iterations: int = 20000
    check_every: int = 64
    tol_primal: float = 1e-9
    tol_dual: float = 1e-9
    tol_gap: float = 1e-7
    fp32_tol_primal: float = 1e-6
    fp32_tol_dual: float = 1e-6
    fp32_tol_gap: float = 1e-4
    reflection: float = 1.0
    restarts: bool = True
    fp32_stall_checks: int = 6
    fp64_stall_checks: int = 8
    floor_tol: float = 1e-7
    fp32_passthrough_tol: float = 1e-3
    fallback_iterations: int = 4096
    recentre: bool = True              # MIXED: re-centred FP32 phase (FP64 tolerances)
    # MIXED re-centred: True / 1 -- hand-offs continue with FP32 matrix
    # values; False / 0 -- in FP64; 2 -- continuation: every instance runs
    # with FP32 matrix values from the warm point (no BF16 phase, no cold
    # fallback), for iterates an earlier call stopped at its cap
    fp32_values_phase: int = 1
    # the certificate gate a stall-floor acceptance must also pass
    # (src/gpu_block_lp.py:84)
    gate_primal: float = 1e-5
    gate_dual: float = 1e-7
    gate_gap: float = 1e-7
    # primal-weight update at a restart: log w <- theta log(|dy|/|dx|) +
    # (1 - theta) log w (0.3 measured: 5 % fewer cold iterations, but 25 %
    # more on the warm-started community steps on the GPU)
    primal_weight_smoothing: float = 0.5

    def native(self) -> N.SolveParams:
        p = N.default_solve_params()
        prec = {"fp64": N.PRECISION_FP64, "mixed": N.PRECISION_MIXED, "fp32": N.PRECISION_FP32}
        if self.precision not in prec:
            raise ValueError("precision must be 'fp64', 'mixed' or 'fp32'")
        p.precision = prec[self.precision]
        for name in ("max_iterations", "fp32_max_iterations", "check_every", "fp32_stall_checks",
                     "fp64_stall_checks", "fallback_iterations"):
            value = getattr(self, name)
            if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, np.integer)):
                raise ValueError(f"{name} must be an integer")
            setattr(p, name, int(value))
        for name in ("tol_primal", "tol_dual", "tol_gap", "fp32_tol_primal", "fp32_tol_dual",
                     "fp32_tol_gap", "reflection", "floor_tol", "fp32_passthrough_tol", "gate_primal",
                     "gate_dual", "gate_gap", "primal_weight_smoothing"):
            setattr(p, name, float(getattr(self, name)))
        p.restarts = 1 if self.restarts else 0
        p.fp32_recentre = 1 if self.recentre else 0
        fv = self.fp32_values_phase
        if isinstance(fv, (bool, np.bool_)):
            fv = int(fv)
        if not isinstance(fv, (int, np.integer)) or fv not in (0, 1, 2):
            raise ValueError("fp32_values_phase must be a bool or 0, 1 or 2")
        p.fp32_values_phase = int(fv)
        return p


@dataclass
class EngineOptions:
    ruiz_iterations: int = 10
    power_iterations: int = 256
    step_safety: float = 0.99
    warps_per_block: int = 16
    blocks_per_sm: int = 0
    max_dynamic_smem: int = 0
    stage_matrix: bool = True
    fp64_max_dynamic_smem: int = 0
    pair_instances: bool = True        # two instances per CTA in the re-centred phase where possible
    spread_banks: bool = True          # order row entries for conflict-free shared-memory gathers

    def native(self) -> N.Options:
        o = N.default_options()
        o.ruiz_iterations = int(self.ruiz_iterations)
        o.power_iterations = int(self.power_iterations)
        o.step_safety = float(self.step_safety)
        o.warps_per_block = int(self.warps_per_block)
        o.blocks_per_sm = int(self.blocks_per_sm)
        o.max_dynamic_smem = int(self.max_dynamic_smem)
        o.stage_matrix = 1 if self.stage_matrix else 0
        o.fp64_max_dynamic_smem = int(self.fp64_max_dynamic_smem)
        o.pair_instances = 1 if self.pair_instances else 0
        o.spread_banks = 1 if self.spread_banks else 0
        return o


def _host_csr(a):
    a = csr_matrix(a, dtype=np.float64)
    indptr = np.ascontiguousarray(a.indptr, dtype=np.int64)
    indices = np.ascontiguousarray(a.indices, dtype=np.int32)
    data = np.ascontiguousarray(a.data, dtype=np.float64)
    return a.shape, indptr, indices, data


def prepare_matrix(a, options: EngineOptions | None = None):
    """Host-only preprocessing (scalings, spectral norm, step); no GPU."""
    lib = N.load()
    (m, n), indptr, indices, data = _host_csr(a)
    dr = np.empty(m)
    dc = np.empty(n)
    smax = ctypes.c_double()
    eta = ctypes.c_double()
    opt = (options or EngineOptions()).native()
    N.check(lib.fbalp_prepare_matrix(
        m, n, indptr.ctypes.data_as(N.c_int64_p), indices.ctypes.data_as(N.c_int32_p),
        data.ctypes.data_as(N.c_double_p), ctypes.byref(opt), dr.ctypes.data_as(N.c_double_p),
        dc.ctypes.data_as(N.c_double_p), ctypes.byref(smax), ctypes.byref(eta)))
    return dict(dr=dr, dc=dc, sigma_max=smax.value, eta=eta.value)


class LPEngine:
    """Species-shared batched LP engine on one CUDA device.

    ``matrices`` is a sequence of ``(A, neq)`` pairs (SciPy sparse or dense);
    rows ``[0, neq)`` are equalities and the rest ``<=`` inequalities.
    """

    def __init__(self, matrices, *, options: EngineOptions | None = None, device=None,
                 stream: torch.cuda.Stream | None = None):
        if not torch.cuda.is_available():
            raise RuntimeError("a CUDA device is required (no CPU fallback)")
        self.lib = N.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.options = options or EngineOptions()
        mats = [(_host_csr(a), int(neq)) for a, neq in matrices]
        if not mats:
            raise ValueError("at least one species matrix is required")
        k = len(mats)
        self.shapes = [(s[0][0], s[0][1]) for s, _ in mats]
        self.neq = [q for _, q in mats]
        rows = (ctypes.c_int32 * k)(*[s[0] for s in self.shapes])
        cols = (ctypes.c_int32 * k)(*[s[1] for s in self.shapes])
        neqs = (ctypes.c_int32 * k)(*self.neq)
        self._keep = [m for m, _ in mats]
        ip = (N.c_int64_p * k)(*[m[1].ctypes.data_as(N.c_int64_p) for m in self._keep])
        ix = (N.c_int32_p * k)(*[m[2].ctypes.data_as(N.c_int32_p) for m in self._keep])
        vv = (N.c_double_p * k)(*[m[3].ctypes.data_as(N.c_double_p) for m in self._keep])
        self.stream = stream or torch.cuda.current_stream(self.device)
        handle = ctypes.c_void_p()
        opt = self.options.native()
        with torch.cuda.device(self.device):
            N.check(self.lib.fbalp_engine_create(k, rows, cols, neqs, ip, ix, vv, ctypes.byref(opt),
                                                 ctypes.c_void_p(self.stream.cuda_stream),
                                                 ctypes.byref(handle)))
        self.handle = handle
        self.count = 0
        self._bound = None
        self.species_id = None
        self.col_offsets = None
        self.row_offsets = None
        self.total_cols = 0
        self.total_rows = 0

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.fbalp_engine_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: torch.cuda.Stream):
        self.stream = stream
        N.check(self.lib.fbalp_engine_set_stream(self.handle, ctypes.c_void_p(stream.cuda_stream)))

    # -- batch -------------------------------------------------------------
    def layout(self, species_id):
        """Column/row offsets of a batch (host numpy), same rule as the C ABI."""
        sid = np.asarray(species_id, dtype=np.int64)
        n = np.array([s[1] for s in self.shapes])[sid]
        m = np.array([s[0] for s in self.shapes])[sid]
        co = np.concatenate([[0], np.cumsum(n)[:-1]]) if len(sid) else np.empty(0, np.int64)
        ro = np.concatenate([[0], np.cumsum(m)[:-1]]) if len(sid) else np.empty(0, np.int64)
        return co.astype(np.int64), ro.astype(np.int64), int(n.sum()), int(m.sum())

    def _dev(self, t, size, name, dtype=torch.float64):
        if t is None:
            return None
        if not isinstance(t, torch.Tensor):
            t = torch.as_tensor(np.asarray(t, dtype=np.float64))
        if t.numel() != size:
            raise ValueError(f"{name} must have {size} elements")
        return t.to(device=self.device, dtype=dtype).contiguous().reshape(-1)

    def set_instances(self, species_id, lower, upper, cost, rhs=None):
        sid = np.ascontiguousarray(np.asarray(species_id, dtype=np.int32).reshape(-1))
        if sid.size < 1:
            raise ValueError("at least one instance is required")
        if sid.min() < 0 or sid.max() >= len(self.shapes):
            raise ValueError("species id out of range")
        co, ro, tc, tr = self.layout(sid)
        lower = self._dev(lower, tc, "lower")
        upper = self._dev(upper, tc, "upper")
        cost = self._dev(cost, tc, "cost")
        rhs = self._dev(rhs, tr, "rhs")
        N.check(self.lib.fbalp_engine_set_instances(self.handle, int(sid.size), sid.ctypes.data_as(N.c_int32_p),
                                                    _ptr(lower), _ptr(upper), _ptr(cost), _ptr(rhs)))
        self._bound = (lower, upper, cost, rhs)  # the engine keeps raw pointers
        self.species_id = sid
        self.count = int(sid.size)
        self.col_offsets, self.row_offsets = co, ro
        self.total_cols, self.total_rows = tc, tr

    def set_instance_data(self, lower, upper, cost, rhs=None):
        """Point the bound batch at new device tensors of the same layout
        (no layout recomputation, no synchronisation)."""
        if self._bound is None:
            raise RuntimeError("set_instances must be called first")
        lower = self._dev(lower, self.total_cols, "lower")
        upper = self._dev(upper, self.total_cols, "upper")
        cost = self._dev(cost, self.total_cols, "cost")
        rhs = self._dev(rhs, self.total_rows, "rhs")
        N.check(self.lib.fbalp_engine_set_instance_data(self.handle, _ptr(lower), _ptr(upper), _ptr(cost), _ptr(rhs)))
        self._bound = (lower, upper, cost, rhs)

    def set_iteration_hints(self, hints):
        """Per-instance iteration hints (device int32, e.g. the previous
        solve's iteration counts; None clears): instances expected to take at
        least one test period skip the early termination tests."""
        if self._bound is None:
            raise RuntimeError("set_instances must be called first")
        h = None if hints is None else self._dev(hints, self.count, "hints", dtype=torch.int32)
        N.check(self.lib.fbalp_engine_set_iteration_hints(self.handle, _ptr(h)))
        self._hints = h

    def set_patches(self, species, rows, cols):
        """Declare up to 8 per-instance matrix entries of one species
        (original row / column indices)."""
        rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).reshape(-1))
        cols = np.ascontiguousarray(np.asarray(cols, dtype=np.int32).reshape(-1))
        if rows.shape != cols.shape:
            raise ValueError("rows and cols must have the same length")
        N.check(self.lib.fbalp_engine_set_patches(self.handle, int(species), int(rows.size),
                                                  rows.ctypes.data_as(N.c_int32_p), cols.ctypes.data_as(N.c_int32_p)))

    def set_patch_values(self, values):
        """Per-instance deltas of the patched entries: device (count, stride)
        float64 (None clears)."""
        if values is None:
            N.check(self.lib.fbalp_engine_set_patch_values(self.handle, None, 0))
            self._patch_values = None
            return
        if not isinstance(values, torch.Tensor):
            values = torch.as_tensor(np.asarray(values, dtype=np.float64))
        values = values.to(device=self.device, dtype=torch.float64).contiguous()
        if values.ndim != 2 or values.shape[0] != self.count:
            raise ValueError("patch values must have shape (count, stride)")
        N.check(self.lib.fbalp_engine_set_patch_values(self.handle, _ptr(values), int(values.shape[1])))
        self._patch_values = values

    def allocate_result(self) -> SolveResult:
        dev = self.device
        c = self.count
        return SolveResult(
            status=torch.empty(c, dtype=torch.int32, device=dev),
            objective=torch.empty(c, dtype=torch.float64, device=dev),
            x=torch.empty(max(1, self.total_cols), dtype=torch.float64, device=dev),
            y=torch.empty(max(1, self.total_rows), dtype=torch.float64, device=dev),
            iterations=torch.empty(c, dtype=torch.int32, device=dev),
            metrics=torch.empty((c, N.METRICS), dtype=torch.float64, device=dev),
            omega=torch.empty(c, dtype=torch.float64, device=dev))

    def solve(self, *, warm_x=None, warm_y=None, warm_omega=None, config: SolveConfig | None = None,
              out: SolveResult | None = None) -> SolveResult:
        if self._bound is None:
            raise RuntimeError("set_instances must be called before solve")
        cfg = config or SolveConfig()
        params = cfg.native()
        wx = self._dev(warm_x, self.total_cols, "warm_x")
        wy = self._dev(warm_y, self.total_rows, "warm_y") if self.total_rows else None
        wo = self._dev(warm_omega, self.count, "warm_omega")
        res = out or self.allocate_result()
        N.check(self.lib.fbalp_engine_solve(
            self.handle, _ptr(wx), _ptr(wy), _ptr(wo), ctypes.byref(params), _ptr(res.status),
            _ptr(res.objective), _ptr(res.x), _ptr(res.y), _ptr(res.iterations), _ptr(res.metrics),
            _ptr(res.omega)))
        self._warm_keep = (wx, wy, wo)
        return res

    def phase_times(self):
        """Device milliseconds of the last solve's (FP32, FP64) phases."""
        a = ctypes.c_float()
        b = ctypes.c_float()
        N.check(self.lib.fbalp_engine_phase_times(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def phase_kernels(self):
        """Names of the kernels the last solve launched for its (first,
        FP64) phases (None for a phase that did not run)."""
        a = ctypes.c_int32()
        b = ctypes.c_int32()
        N.check(self.lib.fbalp_engine_phase_kernels(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return N.KERNEL_NAMES[a.value], N.KERNEL_NAMES[b.value]

    def timing_slots(self, slots: int):
        """Create ``slots`` timing slots (benchmark instrumentation)."""
        N.check(self.lib.fbalp_engine_timing_slots(self.handle, int(slots)))

    def use_timing_slot(self, slot: int):
        """Bracket the following solves' phase launches by the events of
        ``slot`` (-1: none); captured launches keep their slot in the graph."""
        N.check(self.lib.fbalp_engine_use_timing_slot(self.handle, int(slot)))

    def slot_times(self, slot: int):
        """Device milliseconds of the (FP32, FP64) phase launches last
        recorded in ``slot``; waits for them."""
        a = ctypes.c_float()
        b = ctypes.c_float()
        N.check(self.lib.fbalp_engine_slot_times(self.handle, int(slot), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def phase_iterations(self):
        """FP32-phase iteration counts of the last mixed solve (device int32)."""
        out = torch.empty(self.count, dtype=torch.int32, device=self.device)
        N.check(self.lib.fbalp_engine_phase_iterations(self.handle, _ptr(out)))
        return out
