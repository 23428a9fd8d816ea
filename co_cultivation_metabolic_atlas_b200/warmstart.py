"""Learned warm start: an MLP from the dFBA state to primal-dual LP solutions.

The reference trains a PyTorch MLP/GRU on CPU-HiGHS traces to propose
(x, y) seeds for its PDHG corrector (``src/temporal_lp_model.py:58-285``
TemporalLPModel / TemporalLPSession, ``src/temporal_lp_data.py:62-175``
codec, ``scripts/train_temporal_lp.py:23-88`` training).  Here:

* the network is input 44 (40 medium concentrations, 3 biomass values,
  normalised time) -> 4 hidden layers of width 512 with GELU -> the
  concatenated per-species primal fluxes and equality duals;
* weights and activations are BF16 with FP32 accumulation, and every GEMM,
  GELU, MSE gradient and Adam update runs on the project's own sm_100a
  kernels (``include/fbalp_mlp.h``; tcgen05 tensor-core GEMM with TMEM
  accumulators) -- torch only allocates device memory;
* training data are (state -> certified solution) pairs produced by the
  engine's own dFBA rollouts (``collect``);
* the network seeds an environment's first solve (no history); afterwards
  the proposal is the temporal base -- the previous certified solution,
  extrapolated linearly from the last two -- as the reference's
  ``TemporalLPModel`` proposes the previous solution when its residual head
  is zero (``src/temporal_lp_model.py:58-142``).  A trained residual network
  over the base was measured to cost PDHG iterations on these degenerate
  LPs (its corrections move the seed off the optimal face the base sits on),
  so it is not used; the network's first-step seed, besides cutting that
  step's iterations about threefold, also leads the trajectory to optimal
  points from which the later warm-started solves converge faster;
* ``LearnedWarmStart.propose`` turns a batch of states into warm starts; every
  seed is still driven by PDHG to the same tolerances (cold PDHG remains the
  fallback behaviour of any seed).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N

BF16 = torch.bfloat16
F32 = torch.float32


def _p(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(code):
    if code != 0:
        raise RuntimeError(f"tensor-core kernel call failed with code {code}")


class TensorCoreOps:
    """Thin wrappers of the C ABI kernels on torch device tensors."""

    def __init__(self):
        self.lib = N.load()

    def gemm(self, A, B, M, N_, K, *, transA=False, transB=False, bias=None, epilogue=0, alpha=1.0,
             out32=None, out16=None, Z=None, accumulate=False):
        lda = A.shape[-1]
        ldb = B.shape[-1]
        ldc = (out32 if out32 is not None else out16).shape[-1]
        ldz = Z.shape[-1] if Z is not None else 0
        _check(self.lib.fbalp_gemm_bf16(M, N_, K, _p(A), lda, int(transA), _p(B), ldb, int(transB), _p(bias),
                                        epilogue, float(alpha), _p(out32), _p(out16), ldc, _p(Z), ldz,
                                        int(accumulate), _stream()))

    def error_flag(self, clear=True):
        v = ctypes.c_int()
        _check(self.lib.fbalp_mlp_error_flag(ctypes.byref(v), int(clear)))
        return v.value

    def gelu_backward(self, dH, Z, dZ32=None, dZ16=None):
        _check(self.lib.fbalp_gelu_backward(dH.numel(), _p(dH), _p(Z), _p(dZ32), _p(dZ16), _stream()))

    def mse_grad(self, Y, T, scale, dY32=None, dY16=None, loss=None):
        _check(self.lib.fbalp_mse_grad(Y.shape[0], Y.shape[1], _p(Y), _p(T), float(scale), _p(dY32), _p(dY16),
                                       _p(loss), _stream()))

    def column_sum(self, X, out):
        _check(self.lib.fbalp_column_sum(X.shape[0], X.shape[1], _p(X), _p(out), _stream()))

    def adam(self, w, g, m, v, w16, lr, step, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.0):
        _check(self.lib.fbalp_adam_step(w.numel(), _p(w), _p(g), _p(m), _p(v), _p(w16), float(lr), float(beta1),
                                        float(beta2), float(eps), int(step), float(wd), _stream()))

    def to_bf16(self, x, y):
        _check(self.lib.fbalp_to_bf16(x.numel(), _p(x), _p(y), _stream()))


EPI_NONE, EPI_BIAS, EPI_BIAS_GELU = 0, 1, 2


def _pad8(n):
    return (n + 7) // 8 * 8


class MLP:
    """BF16 MLP with GELU hidden layers on the tensor-core kernels.

    Weights are FP32 masters ``W[l]`` of shape ``(out, in_padded)`` with BF16
    copies; inputs are padded to a multiple of 8 features so that every row is
    16-byte aligned for the vectorised tile loads.
    """

    def __init__(self, dims, *, device=None, seed=0):
        self.ops = TensorCoreOps()
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.dims = list(dims)
        self.pdims = [_pad8(d) for d in dims]
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W, self.b, self.W16 = [], [], []
        for l in range(len(dims) - 1):
            fan_in, fan_out = dims[l], dims[l + 1]
            w = torch.zeros(self.pdims[l + 1], self.pdims[l])
            w[:fan_out, :fan_in] = torch.randn(fan_out, fan_in, generator=g) * math.sqrt(2.0 / fan_in)
            if l == len(dims) - 2:
                w *= 0.1  # small output layer: predictions start near the mean
            self.W.append(w.to(self.device))
            self.b.append(torch.zeros(self.pdims[l + 1], device=self.device))
            self.W16.append(self.W[-1].to(BF16))
        self.m = [torch.zeros_like(t) for t in self.W + self.b]
        self.v = [torch.zeros_like(t) for t in self.W + self.b]
        self.step_count = 0
        self._cache = None

    @property
    def layers(self):
        return len(self.W)

    def parameters(self):
        return self.W + self.b

    def state_dict(self):
        return {"dims": self.dims, "W": [w.cpu() for w in self.W], "b": [b.cpu() for b in self.b]}

    def load_state_dict(self, sd):
        if list(sd["dims"]) != self.dims:
            raise ValueError("architecture mismatch")
        for l in range(self.layers):
            self.W[l].copy_(sd["W"][l].to(self.device))
            self.b[l].copy_(sd["b"][l].to(self.device))
            self.W16[l].copy_(self.W[l].to(BF16))

    def _input16(self, X):
        B = X.shape[0]
        xp = torch.zeros(B, self.pdims[0], dtype=F32, device=self.device)
        xp[:, :X.shape[1]] = X
        x16 = torch.empty(B, self.pdims[0], dtype=BF16, device=self.device)
        self.ops.to_bf16(xp, x16)
        return x16

    def forward(self, X, *, keep=False):
        """X: (B, d_in) FP32 -> (B, d_out_padded) FP32."""
        B = X.shape[0]
        h16 = self._input16(X)
        hs, zs = [h16], []
        out = None
        for l in range(self.layers):
            n_out = self.pdims[l + 1]
            last = l == self.layers - 1
            if last:
                out = torch.empty(B, n_out, dtype=F32, device=self.device)
                self.ops.gemm(h16, self.W16[l], B, n_out, self.pdims[l], bias=self.b[l], epilogue=EPI_BIAS,
                              out32=out)
            else:
                nxt = torch.empty(B, n_out, dtype=BF16, device=self.device)
                z = torch.empty(B, n_out, dtype=F32, device=self.device) if keep else None
                self.ops.gemm(h16, self.W16[l], B, n_out, self.pdims[l], bias=self.b[l], epilogue=EPI_BIAS_GELU,
                              out16=nxt, Z=z)
                zs.append(z)
                hs.append(nxt)
                h16 = nxt
        if keep:
            self._cache = (hs, zs)
        return out

    def backward(self, dY32, dY16):
        """Gradients of the loss given dL/dY (FP32 and BF16 copies,
        (B, d_out_padded))."""
        hs, zs = self._cache
        B = dY32.shape[0]
        grads_W = [None] * self.layers
        grads_b = [None] * self.layers
        dZ32 = dY32
        dZ16 = dY16
        for l in reversed(range(self.layers)):
            n_out, n_in = self.pdims[l + 1], self.pdims[l]
            gW = torch.empty(n_out, n_in, dtype=F32, device=self.device)
            # dW = dZ^T H_in : (n_out x B) (B x n_in)
            self.ops.gemm(dZ16, hs[l], n_out, n_in, B, transA=True, transB=True, out32=gW)
            gb = torch.empty(n_out, dtype=F32, device=self.device)
            self.ops.column_sum(dZ32, gb)
            grads_W[l], grads_b[l] = gW, gb
            if l > 0:
                dH = torch.empty(B, n_in, dtype=F32, device=self.device)
                # dH_in = dZ W : (B x n_out) (n_out x n_in)
                self.ops.gemm(dZ16, self.W16[l], B, n_in, n_out, transB=True, out32=dH)
                dZ32 = torch.empty_like(dH)
                dZ16 = torch.empty(B, n_in, dtype=BF16, device=self.device)
                self.ops.gelu_backward(dH, zs[l - 1], dZ32, dZ16)
        return grads_W, grads_b

    def adam_step(self, grads_W, grads_b, lr, wd=0.0):
        self.step_count += 1
        for l in range(self.layers):
            self.ops.adam(self.W[l], grads_W[l], self.m[l], self.v[l], self.W16[l], lr, self.step_count, wd=wd)
            self.ops.adam(self.b[l], grads_b[l], self.m[self.layers + l], self.v[self.layers + l], None, lr,
                          self.step_count)


# ------------------------------------------------------------------ codec
def state_features(medium, biomass, t_frac):
    """44 features: log1p(medium) (40), 10 * biomass (3), normalised time."""
    E = medium.shape[0]
    tcol = torch.full((E, 1), float(t_frac), dtype=F32, device=medium.device)
    return torch.cat([torch.log1p(medium.float().clamp_min(0)), 10.0 * biomass.float(), tcol], dim=1)


@dataclass
class Codec:
    """Feature and target standardisation (the reference's TemporalLPCodec,
    ``src/temporal_lp_data.py:62-175``, without its PCA rank reduction: the
    network predicts every flux and dual)."""
    f_mean: torch.Tensor
    f_std: torch.Tensor
    t_mean: torch.Tensor
    t_std: torch.Tensor
    omega: torch.Tensor      # per species median primal weight

    @staticmethod
    def fit(F, T, omegas, ranks=None):
        """Standardisation of the rows of ``F`` / ``T``; with ``ranks`` (a
        data-parallel job) over every rank's rows, and the primal weights
        averaged over the ranks."""
        from .distributed import allreduce_mean_, global_moments
        f_mean, f_std = global_moments(F, ranks)
        t_mean, t_std = global_moments(T, ranks)
        omegas = omegas.clone()
        allreduce_mean_([omegas], ranks)
        return Codec(f_mean, f_std.clamp_min(1e-3), t_mean, t_std.clamp_min(1e-6), omegas)

    def features(self, F):
        return (F - self.f_mean) / self.f_std

    def targets(self, T):
        return (T - self.t_mean) / self.t_std

    def decode(self, Y):
        return Y * self.t_std + self.t_mean

    def state_dict(self):
        return {k: getattr(self, k).cpu() for k in ("f_mean", "f_std", "t_mean", "t_std", "omega")}

    @staticmethod
    def from_state(sd, device):
        return Codec(**{k: v.to(device) for k, v in sd.items()})


def solution_layout(models):
    """Offsets of each species' x and y inside one target row."""
    out = []
    off = 0
    for m in models:
        n, r = m.S.shape[1], m.S.shape[0]
        out.append((off, n, off + n, r))
        off += n + r
    return out, off


def gather_targets(com, res):
    """One target row per environment: [x_0, y_0, x_1, y_1, x_2, y_2]."""
    E = com.E
    cols = []
    co = com.col_offsets
    eng = com.engine
    _, ro, _, _ = eng.layout(com.species_id)
    for s, m in enumerate(com.models):
        n, r = m.S.shape[1], m.S.shape[0]
        xs = res.x[int(co[s * E]):int(co[s * E]) + E * n].view(E, n)
        ys = res.y[int(ro[s * E]):int(ro[s * E]) + E * r].view(E, r)
        cols += [xs, ys]
    return torch.cat(cols, dim=1).float()


def temporal_base(prev, prev2):
    """Temporal base of a warm start (any layout, FP64): the previous
    solution extrapolated linearly from the last two, or the previous one."""
    return prev if prev2 is None else 2.0 * prev - prev2


@dataclass
class Rollouts:
    """Training pairs of one or more rollouts (device tensors)."""
    F: torch.Tensor        # (N, 44) state features
    T: torch.Tensor        # (N, width) certified solutions (FP32)
    ok: torch.Tensor       # (N,) every species certified
    omega: torch.Tensor    # (N, species) final primal weights


def collect(models, *, envs, steps, seed, dt=0.05, horizon_steps=960, config=None, device=None):
    """Roll the community forward with extrapolated warm starts and record
    (features, certified solution, status, primal weights) for every
    environment and step."""
    from .dfba import DeviceCommunity
    from . import synthetic as syn
    medium, biomass = syn.initial_environments(envs, seed=seed)
    com = DeviceCommunity(models, medium, biomass, config=config, warm_start="extrapolate", device=device)
    F, T, ok, om = [], [], [], []
    for k in range(steps):
        F.append(state_features(com.medium, com.biomass, k / horizon_steps))
        com.uptake_bounds()
        res = com.solve()
        T.append(gather_targets(com, res))
        ok.append((res.status == 0).view(len(models), envs).all(dim=0))
        om.append(res.omega.view(len(models), envs).float().t())
        com.integrate(res)
    com.close()
    return Rollouts(torch.cat(F), torch.cat(T), torch.cat(ok), torch.cat(om))


class LearnedWarmStart:
    """Trained network + codec producing flat warm-start arrays for a
    community: the network's prediction for environments without history,
    the temporal base of their last certified solutions otherwise."""

    def __init__(self, mlp: MLP, codec: Codec, models):
        self.mlp = mlp
        self.codec = codec
        self.models = models
        self.layout, self.width = solution_layout(models)

    def predict(self, features):
        Y = self.mlp.forward(self.codec.features(features))[:, :self.width]
        return self.codec.decode(Y)

    def _flat(self, P):
        xs, ys = [], []
        for s, (xo, n, yo, r) in enumerate(self.layout):
            xs.append(P[:, xo:xo + n].reshape(-1))
            ys.append(P[:, yo:yo + r].reshape(-1))
        return torch.cat(xs), torch.cat(ys)

    def propose(self, com, t_frac):
        """Warm start (x, y, omega) flat device arrays for the community's
        species-major batch, from its current state (``com.medium``,
        ``com.biomass``) or its last certified solutions (``com.prev``,
        ``com.prev2``)."""
        if com.prev is None:
            feats = state_features(com.medium, com.biomass, t_frac)
            x, y = self._flat(self.predict(feats).double())
            omega = torch.repeat_interleave(self.codec.omega.double(), com.E)
            return x, y, omega
        nc, nr = com.total_cols, com.total_rows
        p2 = com.prev2
        bx = temporal_base(com.prev.x[:nc], None if p2 is None else p2.x[:nc])
        by = temporal_base(com.prev.y[:nr], None if p2 is None else p2.y[:nr])
        return bx, by, com.prev.omega


def train(mlp: MLP, F, T, *, epochs=20, batch=4096, lr=1e-3, lr_final=1e-4, seed=0, log=None, ranks=None):
    """Full-batch-shuffled Adam on the MSE of standardised targets.  With
    ``ranks`` (data-parallel): every rank takes the same number of steps on
    its own rows and applies the gradient averaged over the ranks."""
    from .distributed import allreduce_mean_, min_int
    ops = mlp.ops
    n = F.shape[0]
    width = T.shape[1]
    gen = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    per_epoch = min_int(max(1, n // batch), ranks)
    steps_total = epochs * per_epoch
    step = 0
    loss_acc = torch.zeros(1, dtype=torch.float64, device=mlp.device)
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen).to(mlp.device)
        loss_acc.zero_()
        count = 0
        for i in range(0, per_epoch * batch, batch):
            idx = perm[i:i + batch]
            X = F[idx]
            Y = mlp.forward(X, keep=True)
            Tp = torch.zeros_like(Y)
            Tp[:, :width] = T[idx]
            dY = torch.empty_like(Y)
            dY16 = torch.empty(Y.shape, dtype=BF16, device=mlp.device)
            ops.mse_grad(Y, Tp, 2.0 / (batch * width), dY32=dY, dY16=dY16, loss=loss_acc)
            gW, gb = mlp.backward(dY, dY16)
            allreduce_mean_(gW + gb, ranks)
            frac = step / max(1, steps_total - 1)
            cur = lr * (lr_final / lr) ** frac
            mlp.adam_step(gW, gb, cur)
            step += 1
            count += batch * width
        if ranks is not None and ranks.world > 1:
            losses.append(ranks.sum(float(loss_acc.item())) / ranks.sum(float(count)))
        else:
            losses.append(float(loss_acc.item()) / max(1, count))
        if log:
            log(f"epoch {ep}: mse {losses[-1]:.4e}")
    if ops.error_flag():
        raise RuntimeError("a tensor-core GEMM wait timed out during training")
    return losses


# ------------------------------------------------------------ drop-in backend
def signed_log(values):
    """``sign(v) log(1 + |v|)`` with infinities clipped to +-1e13 (the
    reference's feature transform, ``src/temporal_lp_data.py:15-17``)."""
    v = np.nan_to_num(np.asarray(values, dtype=np.float64), nan=0.0, posinf=1e13, neginf=-1e13)
    return np.sign(v) * np.log1p(np.abs(v))


MAX_REQUEST_FEATURES = 128


@dataclass
class RequestMember:
    """The network of one species matrix: request features -> [x; y]."""
    mlp: MLP
    index: np.ndarray        # int64 positions in [lower, upper, c, rhs] used as features
    f_mean: torch.Tensor
    f_std: torch.Tensor
    t_mean: torch.Tensor
    t_std: torch.Tensor
    n: int
    m: int
    omega: float             # median primal weight of the training solutions

    def features(self, lower, upper, cost, rhs):
        """Feature rows of a batch ((k, n), (k, n), (k, n), (k, m) arrays)."""
        full = np.concatenate([lower, upper, cost, rhs], axis=1)
        return signed_log(full[:, self.index])

    def predict(self, feats):
        X = torch.as_tensor(feats, dtype=F32, device=self.mlp.device)
        Y = self.mlp.forward((X - self.f_mean) / self.f_std)[:, :self.n + self.m]
        return (Y * self.t_std + self.t_mean).double()


def select_request_features(full, limit=MAX_REQUEST_FEATURES):
    """Feature positions of signed-log request rows ``full`` (k, d): the
    columns that vary over the rows, one representative of identical
    columns, at most ``limit`` (the largest spreads), ascending; a batch with
    no varying entry keeps position 0."""
    spread = full.std(axis=0)
    cand = np.flatnonzero(spread > 1e-12)
    _, first = np.unique(full[:, cand].T, axis=0, return_index=True)
    cand = cand[np.sort(first)]
    if cand.size > limit:
        cand = np.sort(cand[np.argsort(-spread[cand], kind="stable")[:limit]])
    if cand.size == 0:
        cand = np.array([0], dtype=np.int64)
    return cand.astype(np.int64)


def fit_request_member(lower, upper, cost, rhs, X, Y, omega, *, hidden=(512, 512), epochs=20, batch=1024,
                       seed=0, device=None, log=None):
    """Train the network of one species matrix on (request -> certified
    solution) pairs: rows of ``lower``/``upper``/``cost`` (k, n), ``rhs``
    (k, m), solutions ``X`` (k, n), ``Y`` (k, m), primal weights ``omega``.
    Features are the signed-log entries of ``[lower, upper, c, rhs]`` that
    vary over the training rows, duplicates removed, at most 128 (the
    largest spreads), as the reference's codec selects them
    (``src/temporal_lp_data.py:62-175``); targets are standardised."""
    full = signed_log(np.concatenate([lower, upper, cost, rhs], axis=1))
    cand = select_request_features(full)
    dev = torch.device(device) if device is not None else torch.device("cuda")
    F = torch.as_tensor(full[:, cand], dtype=F32, device=dev)
    T = torch.as_tensor(np.concatenate([X, Y], axis=1), dtype=F32, device=dev)
    f_mean, f_std = F.mean(0), F.std(0).clamp_min(1e-3)
    t_mean, t_std = T.mean(0), T.std(0).clamp_min(1e-6)
    n, m = X.shape[1], Y.shape[1]
    net = MLP([int(cand.size), *hidden, n + m], device=dev, seed=seed)
    losses = train(net, (F - f_mean) / f_std, (T - t_mean) / t_std, epochs=epochs,
                   batch=min(batch, F.shape[0]), seed=seed, log=log)
    member = RequestMember(net, cand.astype(np.int64), f_mean, f_std, t_mean, t_std, n, m,
                           float(np.median(np.asarray(omega, dtype=np.float64))))
    return member, losses


class RequestWarmStart:
    """Learned warm start of the drop-in backend (``B200LPBackend(mode=
    'mlp', warm_start_model=...)``), the counterpart of the reference's
    ``TemporalLPModel`` / ``TemporalLPSession`` behind
    ``TemporalGpuLPBackend(mode='mlp')`` (``src/temporal_gpu_lp.py:136-168``,
    ``src/temporal_lp_model.py:221-285``).

    ``members`` maps a species matrix's content key (``problem.matrix_key``)
    to its trained network.  For every request of a batch, ``propose``
    returns the temporal base of the environment's last certified solutions
    of the same matrix (the previous one extrapolated linearly from the last
    two, as the dFBA loop's warm start) when it has any, else the network's
    prediction from the request's features, else the cold start.  Proposals
    are pending until ``commit``: the backend commits after every row of a
    call is built, with the call's certified solutions, so a call that
    raises leaves every environment's history as it was (the reference's
    propose/commit transaction).  A failed row clears its environment's
    history."""

    def __init__(self, members: dict):
        self.members = dict(members)
        self._history: dict = {}   # env -> [(key, x, y, omega)] oldest first, at most two
        self.last_sources: list = []

    def reset(self, environment_ids=None):
        if environment_ids is None:
            self._history.clear()
        else:
            for env in environment_ids:
                self._history.pop(env, None)

    def propose(self, ids, problems, species, eng, keys=None):
        """Flat warm-start arrays (x, y, omega) in the engine's batch layout
        (host numpy, FP64)."""
        from .problem import matrix_key
        if keys is None:
            keys = [matrix_key(p[0], p[5]) for p in problems]
        co, ro, tc, tr = eng.layout(species)
        wx = np.zeros(tc)
        wy = np.zeros(tr)
        wo = np.ones(len(ids))
        sources = ["cold"] * len(ids)
        by_key: dict = {}
        for i, (env, key) in enumerate(zip(ids, keys)):
            hist = [h for h in self._history.get(env, []) if h[0] == key]
            n, m = problems[i][4].shape[0], problems[i][1].shape[0]
            if hist:
                x1, y1, o1 = hist[-1][1:]
                if len(hist) > 1:
                    x0, y0, _ = hist[-2][1:]
                    x1, y1 = temporal_base(x1, x0), temporal_base(y1, y0)
                wx[co[i]:co[i] + n] = x1
                wy[ro[i]:ro[i] + m] = y1
                wo[i] = o1
                sources[i] = "temporal"
            elif key in self.members:
                by_key.setdefault(key, []).append(i)
        for key, rows in by_key.items():
            mem = self.members[key]
            lo = np.stack([problems[i][2] for i in rows])
            up = np.stack([problems[i][3] for i in rows])
            c = np.stack([problems[i][4] for i in rows])
            b = np.stack([problems[i][1] for i in rows])
            pred = mem.predict(mem.features(lo, up, c, b)).cpu().numpy()
            for r, i in enumerate(rows):
                wx[co[i]:co[i] + mem.n] = pred[r, :mem.n]
                wy[ro[i]:ro[i] + mem.m] = pred[r, mem.n:]
                wo[i] = mem.omega
                sources[i] = "network"
        self.last_sources = sources
        return wx, wy, wo

    def commit(self, ids, certified, keys):
        """Advance the history of every environment of a finished call:
        ``certified`` maps an environment to its (x, y, omega), ``keys``
        gives each environment's matrix key."""
        for env, key in zip(ids, keys):
            if env in certified:
                x, y, om = certified[env]
                hist = [h for h in self._history.get(env, []) if h[0] == key][-1:]
                hist.append((key, x, y, om))
                self._history[env] = hist
            else:
                self._history.pop(env, None)


def species_key(model):
    """The drop-in's content key of a species' FBA matrix (the key
    ``B200LPBackend`` computes for its requests)."""
    from .problem import matrix_key, normalize
    zeros = np.zeros(model.S.shape[0])
    p = normalize(model.cost, dict(A_eq=model.S, b_eq=zeros, bounds=np.column_stack([model.lower, model.upper])))
    return matrix_key(p[0], p[5])


def collect_request_pairs(models, *, envs, steps, seed, config=None, device=None):
    """Per species, (lower bounds, certified x, y, omega) rows of every
    certified (environment, step) of a rollout with extrapolated warm
    starts: the drop-in's training pairs (its requests differ only in their
    lower bounds)."""
    from . import synthetic as syn
    from .dfba import DeviceCommunity
    medium, biomass = syn.initial_environments(envs, seed=seed)
    com = DeviceCommunity(models, medium, biomass, config=config, warm_start="extrapolate", device=device)
    co = com.col_offsets.cpu().numpy()
    _, ro, _, _ = com.engine.layout(com.species_id)
    out = [dict(lower=[], x=[], y=[], omega=[]) for _ in models]
    for _ in range(steps):
        com.uptake_bounds()
        lower = com.lower.cpu().numpy()
        res = com.solve()
        x, y = res.x.cpu().numpy(), res.y.cpu().numpy()
        ok = (res.status == 0).cpu().numpy()
        om = res.omega.cpu().numpy()
        for s, mdl in enumerate(models):
            m, n = mdl.S.shape
            c0, r0 = int(co[s * envs]), int(ro[s * envs])
            sel = ok[s * envs:(s + 1) * envs]
            out[s]["lower"].append(lower[c0:c0 + envs * n].reshape(envs, n)[sel])
            out[s]["x"].append(x[c0:c0 + envs * n].reshape(envs, n)[sel])
            out[s]["y"].append(y[r0:r0 + envs * m].reshape(envs, m)[sel])
            out[s]["omega"].append(om[s * envs:(s + 1) * envs][sel])
        com.integrate(res)
    com.close()
    return [{k: np.concatenate(v) for k, v in d.items()} for d in out]


def fit_request_warm_start(models, *, envs, steps, seeds, epochs=20, hidden=(512, 512), config=None, device=None,
                           log=None):
    """Train one network per species on the engine's own rollouts (seeds
    disjoint from the evaluated environments) and return the drop-in's
    ``RequestWarmStart`` and the per-species losses."""
    parts = [collect_request_pairs(models, envs=envs, steps=steps, seed=sd, config=config, device=device)
             for sd in seeds]
    members, losses = {}, []
    for s, mdl in enumerate(models):
        d = {k: np.concatenate([p[s][k] for p in parts]) for k in ("lower", "x", "y", "omega")}
        k = d["lower"].shape[0]
        member, ls = fit_request_member(d["lower"], np.broadcast_to(mdl.upper, (k, mdl.S.shape[1])),
                                        np.broadcast_to(mdl.cost, (k, mdl.S.shape[1])),
                                        np.zeros((k, mdl.S.shape[0])), d["x"], d["y"], d["omega"],
                                        hidden=hidden, epochs=epochs, device=device, log=log)
        members[species_key(mdl)] = member
        losses.append(ls)
    return RequestWarmStart(members), losses
