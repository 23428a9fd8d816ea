"""NumPy restatement of the engine's restarted Halpern PDHG (test
infrastructure only; the parity reference for the CUDA kernels).

Problem (minimisation form, HiGHS dual signs, as in
``src/gpu_pdhg_corrector.py:1-15``)::

    min c.x  s.t.  A[:neq] x = b[:neq],  A[neq:] x <= b[neq:],  l <= x <= u

Preprocessing (per species, shared by every instance of that species):
  * ``ruiz_iters`` rounds of Ruiz equilibration (row/column infinity norms,
    square-root updates), then one Pock-Chambolle step (alpha = 1: row/column
    absolute sums, square roots).  ``A~ = Dr A Dc``, ``x = Dc x~``,
    ``y = Dr y~``.  The reference uses only the Pock-Chambolle diagonal metric
    (``src/gpu_pdhg_corrector.py:183-200``); Ruiz scaling is this engine's
    addition.
  * ``eta = step_safety / ||A~||_2`` with ``||A~||_2`` from ``power_iters``
    power iterations on ``A~^T A~`` from a fixed deterministic start vector.

Iteration (primal-first PDHG operator ``T``, reflected Halpern anchoring;
Lu & Yang "restarted Halpern PDHG", cuPDLPx 2025), ``tau = eta/omega``,
``sigma = eta*omega``::

    xn = clip(x - tau (c - A^T y), l, u)
    yn = P_Y(y + sigma (b - A (2 xn - x)))      P_Y: y_i <= 0 on rows >= neq
    w  = (k+1)/(k+2)
    x  = w ((1+rho) xn - rho x) + (1-w) xa
    y  = w ((1+rho) yn - rho y) + (1-w) ya

Every ``check_every`` iterations, at the candidate ``(xn, yn)``: FP64 KKT
metrics in original units; stop when converged; otherwise the restart rule on
the fixed-point residual ``r = sqrt(omega |xn-x|^2 + |yn-y|^2/omega)``::

    restart if r <= 0.2 r_restart
            or (r <= 0.8 r_restart and r > r_prev)
            or k >= 0.36 * it

On restart the primal weight becomes
``exp(theta log(|yn-ya|/|xn-xa|) + (1 - theta) log omega)`` with ``theta =
OMEGA_SMOOTHING`` (0.5, the engine's default ``primal_weight_smoothing``;
when both distances exceed 1e-10) and ``x = xa = xn``, ``y = ya = yn``, ``k = 0``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.sparse import csr_matrix

BETA_SUFFICIENT = 0.2
BETA_NECESSARY = 0.8
BETA_ARTIFICIAL = 0.36
OMEGA_SMOOTHING = 0.5
STALL_FLOOR = 1.0

STATUS_OPTIMAL = 0
STATUS_ITERATION_LIMIT = 1
STATUS_NUMERICAL = 2
STATUS_HANDOFF = 5


def power_start(n):
    """Deterministic start vector: a multiplicative hash of the index mapped
    to [0.5, 1.5) (identical integer arithmetic in the C++ preprocessor)."""
    j = np.arange(n, dtype=np.uint64)
    h = (j * np.uint64(2654435761)) % np.uint64(1 << 32)
    return h.astype(np.float64) / 4294967296.0 + 0.5


@dataclass
class Prepared:
    A: csr_matrix          # scaled matrix A~ (FP64)
    dr: np.ndarray
    dc: np.ndarray
    eta: float
    sigma_max: float
    neq: int


def prepare(S, neq=None, *, ruiz_iters=10, power_iters=256, step_safety=0.99):
    S = csr_matrix(S, dtype=np.float64)
    S.sum_duplicates()
    S.sort_indices()
    m, n = S.shape
    neq = m if neq is None else int(neq)
    dr = np.ones(m)
    dc = np.ones(n)
    rows = np.repeat(np.arange(m), np.diff(S.indptr))
    cols = S.indices
    av = np.abs(S.data)
    for _ in range(ruiz_iters):
        cur = av * dr[rows] * dc[cols]
        rmax = np.zeros(m)
        np.maximum.at(rmax, rows, cur)
        cmax = np.zeros(n)
        np.maximum.at(cmax, cols, cur)
        fr = np.where(rmax > 0, np.sqrt(rmax), 1.0)
        fc = np.where(cmax > 0, np.sqrt(cmax), 1.0)
        dr = dr / fr
        dc = dc / fc
    cur = av * dr[rows] * dc[cols]
    rsum = np.zeros(m)
    np.add.at(rsum, rows, cur)
    csum = np.zeros(n)
    np.add.at(csum, cols, cur)
    dr = dr / np.where(rsum > 0, np.sqrt(rsum), 1.0)
    dc = dc / np.where(csum > 0, np.sqrt(csum), 1.0)
    A = csr_matrix((S.data * dr[rows] * dc[cols], S.indices.copy(), S.indptr.copy()), shape=(m, n))
    v = power_start(n)
    v /= np.linalg.norm(v)
    lam = 0.0
    AT = A.T.tocsr()
    for _ in range(power_iters):
        wv = AT @ (A @ v)
        lam = np.linalg.norm(wv)
        if lam <= 0:
            break
        v = wv / lam
    smax = float(np.sqrt(lam)) if lam > 0 else 0.0
    eta = step_safety / smax if smax > 0 else 1.0
    return Prepared(A=A, dr=dr, dc=dc, eta=eta, sigma_max=smax, neq=neq)


def kkt_metrics(P: Prepared, lower, upper, cost, rhs, xn, yn):
    """FP64 metrics at a scaled point, evaluated in ORIGINAL units with the
    exact FP64 bounds / objective / right-hand side."""
    A, dr, dc, neq = P.A, P.dr, P.dc, P.neq
    x = xn * dc
    y = yn * dr
    ro = (A @ xn) / dr - rhs                  # A x - b
    pr_eq = np.max(np.abs(ro[:neq]), initial=0.0)
    pr_ub = np.max(ro[neq:], initial=0.0)
    bviol = max(np.max(lower - x, initial=0.0), np.max(x - upper, initial=0.0))
    primal = max(0.0, pr_eq, pr_ub, bviol)
    r = cost - (A.T @ yn) / dc                # c - A^T y
    finl = np.isfinite(lower)
    finu = np.isfinite(upper)
    dual = max(0.0, np.max(y[neq:], initial=0.0),
               np.max(np.where(~finl, r, 0.0), initial=0.0),
               np.max(np.where(~finu, -r, 0.0), initial=0.0))
    pobj = float(cost @ x)
    term = np.where(r > 0, np.where(finl, r * np.where(finl, lower, 0.0), 0.0),
                    np.where(r < 0, np.where(finu, r * np.where(finu, upper, 0.0), 0.0), 0.0))
    dobj = float(rhs @ y + term.sum())
    target = np.where(r >= 0, lower, upper)
    bgap = np.abs(r * (x - np.where(np.isfinite(target), target, x))).sum()
    rgap = np.abs(y[neq:] * ro[neq:]).sum()
    kgap = (bgap + rgap) / max(1.0, abs(pobj))
    rel_gap = abs(pobj - dobj) / (1.0 + abs(pobj) + abs(dobj))
    xinf = float(np.max(np.abs(x), initial=0.0))
    cinf = float(np.max(np.abs(cost), initial=0.0))
    return dict(primal_residual=primal, dual_violation=dual, relative_kkt_gap=kgap,
                objective=pobj, dual_objective=dobj, relative_gap=rel_gap, x_inf=xinf, c_inf=cinf)


def converged(mt, tol_primal, tol_dual, tol_gap):
    return (mt["primal_residual"] <= tol_primal * (1.0 + mt["x_inf"])
            and mt["dual_violation"] <= tol_dual * (1.0 + mt["c_inf"])
            and mt["relative_gap"] <= tol_gap and mt["relative_kkt_gap"] <= tol_gap)


def solve(P: Prepared, lower, upper, cost, rhs=None, *, x0=None, y0=None, omega0=1.0,
          dtype=np.float64, max_iters=100000, check_every=64, tol_primal=1e-9, tol_dual=1e-9,
          tol_gap=1e-7, rho=1.0, restarts=True, stop_on_converge=True, final_status=STATUS_OPTIMAL,
          stall_checks=None, floor_tol=1e-7, fallback_iters=0, trace=None):
    """Run the engine's algorithm for one instance; return dict with scaled
    and original-unit iterates, status, iterations and metrics."""
    A, dr, dc = P.A, P.dr, P.dc
    m, n = A.shape
    rhs = np.zeros(m) if rhs is None else np.asarray(rhs, float)
    ls = lower / dc
    us = upper / dc
    cs = cost * dc
    bs = rhs * dr
    Af = A.astype(dtype)
    ATf = A.T.tocsr().astype(dtype)
    lsf, usf, csf, bsf = (v.astype(dtype) for v in (ls, us, cs, bs))
    ineq = np.arange(m) >= P.neq
    x = np.zeros(n) if x0 is None else np.asarray(x0, float) / dc
    y = np.zeros(m) if y0 is None else np.asarray(y0, float) / dr
    x = np.clip(x.astype(dtype), lsf, usf)
    y = np.where(ineq, np.minimum(y, 0.0), y).astype(dtype)
    xa, ya = x.copy(), y.copy()
    omega = float(omega0)
    k = 0
    r_restart = np.inf
    r_prev = np.inf
    status = STATUS_ITERATION_LIMIT
    mt = None
    it = 0
    xn, yn = x, y
    mt = kkt_metrics(P, lower, upper, cost, rhs, x.astype(float), y.astype(float))
    if converged(mt, tol_primal, tol_dual, tol_gap) or max_iters == 0:
        status = final_status if converged(mt, tol_primal, tol_dual, tol_gap) else STATUS_ITERATION_LIMIT
        return dict(x=np.clip(x.astype(float) * dc, lower, upper), y=y.astype(float) * dr, xs=x, ys=y,
                    status=status, iterations=0, metrics=mt, omega=omega)
    best_err = np.inf
    stall = 0
    fell_back = False
    if stall_checks is None:
        stall_checks = 8 if final_status == STATUS_OPTIMAL else 6
    for it in range(1, max_iters + 1):
        tau = dtype(P.eta / omega)
        sig = dtype(P.eta * omega)
        g = ATf @ y
        xn = np.clip(x - tau * (csf - g), lsf, usf).astype(dtype)
        xb = (xn + xn - x).astype(dtype)
        h = Af @ xb
        yn = (y + sig * (bsf - h)).astype(dtype)
        yn = np.where(ineq, np.minimum(yn, 0), yn).astype(dtype)
        w = dtype((k + 1.0) / (k + 2.0))
        if rho == 1.0:
            xnew = (w * xb + (1 - w) * xa).astype(dtype)
            ynew = (w * (yn + yn - y) + (1 - w) * ya).astype(dtype)
        else:
            xnew = (w * ((1 + rho) * xn - rho * x) + (1 - w) * xa).astype(dtype)
            ynew = (w * ((1 + rho) * yn - rho * y) + (1 - w) * ya).astype(dtype)
        k += 1
        full = (it % check_every == 0) or it == max_iters
        # termination-only tests at 8, 16, 32, ... below check_every
        is_check = full or (8 <= it < check_every and (it & (it - 1)) == 0)
        if is_check:
            dx = (xn.astype(float) - x.astype(float))
            dy = (yn.astype(float) - y.astype(float))
            r = np.sqrt(omega * (dx @ dx) + (dy @ dy) / omega)
            mt = kkt_metrics(P, lower, upper, cost, rhs, xn.astype(float), yn.astype(float))
            if trace is not None:
                trace.append(dict(it=it, r=r, omega=omega, **mt))
            if not np.isfinite(r) or not all(np.isfinite(v) for v in mt.values()):
                status = STATUS_NUMERICAL
                break
            if stop_on_converge and converged(mt, tol_primal, tol_dual, tol_gap):
                status = final_status
                break
            if it == max_iters:
                break
            if not full:
                x, y = xnew, ynew
                continue
            err = max(mt["primal_residual"] / (1 + mt["x_inf"]), mt["dual_violation"] / (1 + mt["c_inf"]),
                      mt["relative_gap"], mt["relative_kkt_gap"])
            if err < 0.5 * best_err:
                best_err, stall = err, 0
            else:
                stall += 1
            if stall_checks > 0 and stall >= stall_checks:
                if final_status == STATUS_HANDOFF and best_err <= STALL_FLOOR:
                    status = final_status
                    break
                if (final_status == STATUS_OPTIMAL and err <= floor_tol
                        and mt["primal_residual"] <= floor_tol * (1 + mt["x_inf"])
                        and mt["dual_violation"] <= floor_tol * (1 + mt["c_inf"])):
                    status = final_status
                    break
            if (fallback_iters > 0 and not fell_back and it >= fallback_iters
                    and (x0 is not None or y0 is not None)):
                # cold fallback of a warm start that has not converged
                fell_back = True
                omega = 1.0
                x = np.clip(np.zeros(n, dtype), lsf, usf).astype(dtype)
                y = np.zeros(m, dtype)
                xa, ya = x.copy(), y.copy()
                k = 0
                r_restart = r_prev = best_err = np.inf
                stall = 0
                continue
            if restarts and (r <= BETA_SUFFICIENT * r_restart
                             or (r <= BETA_NECESSARY * r_restart and r > r_prev)
                             or k >= BETA_ARTIFICIAL * it):
                ddx = xn.astype(float) - xa.astype(float)
                ddy = yn.astype(float) - ya.astype(float)
                nx = np.sqrt(ddx @ ddx)
                ny = np.sqrt(ddy @ ddy)
                if nx > 1e-10 and ny > 1e-10:
                    omega = float(np.exp(OMEGA_SMOOTHING * np.log(ny / nx)
                                         + (1 - OMEGA_SMOOTHING) * np.log(omega)))
                xnew, ynew = xn.copy(), yn.copy()
                xa, ya = xn.copy(), yn.copy()
                k = 0
                r_restart = r
                r_prev = np.inf
            else:
                r_prev = r
        x, y = xnew, ynew
    xo = xn.astype(float) * dc
    if final_status == STATUS_OPTIMAL:  # the final FP64 phase reports x inside its bounds
        xo = np.clip(xo, lower, upper)
    yo = yn.astype(float) * dr
    return dict(x=xo, y=yo, xs=xn, ys=yn, status=status, iterations=it, metrics=mt, omega=omega)


def bf16_round(x):
    """FP32 values rounded to the nearest BF16 (ties to even), as FP32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = (b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32)


def solve_recentred(P: Prepared, lower, upper, cost, rhs=None, *, x0=None, y0=None, omega0=1.0,
                    max_iters=20000, check_every=64, tol_primal=1e-9, tol_dual=1e-9, tol_gap=1e-7, rho=1.0,
                    restarts=True, stall_checks=8, floor_tol=1e-7, fallback_iters=0, handoff_stall_checks=32,
                    trace=None):
    """The engine's re-centred FP32 phase (the first phase of its mixed
    schedule).

    Iterates are FP32 differences from an FP64 base ``(xh, yh)`` (scaled
    space).  At the start, after every restart and after a cold fallback the
    base moves to the evaluated candidate and the FP32 problem becomes the
    correction LP ``min d.dx s.t. A~ dx = r, ls - xh <= dx <= us - xh``
    (``yh + dy <= 0`` on inequality rows) with ``d = c~ - A~^T yh`` and
    ``r = b~ - A~ xh`` computed in FP64 and rounded to FP32 once.  The FP32
    passes use the scaled matrix rounded to BF16 (the engine stages it as
    packed 16-bit index / BF16 value words): the re-centring corrects the
    rounding of the matrix like the rounding of the iterates, and the
    convergence tests use the FP64 matrix.  The Halpern
    anchor is the base, so the differences restart from zero.  Convergence
    tests evaluate the FP64 candidate ``xh + dxn`` (projected onto the exact
    scaled bounds), ``yh + dyn``.  After ``stall_checks`` full tests without
    halving the KKT error a point meeting ``floor_tol`` is accepted; after
    ``handoff_stall_checks`` such tests the solve ends with
    ``STATUS_HANDOFF`` (the FP64 phase continues; 0 = never).
    """
    f32 = np.float32
    A, dr, dc = P.A, P.dr, P.dc
    m, n = A.shape
    rhs = np.zeros(m) if rhs is None else np.asarray(rhs, float)
    ls, us, cs, bs = lower / dc, upper / dc, cost * dc, rhs * dr
    AT = A.T.tocsr()
    Af = A.astype(f32)
    ATf = AT.astype(f32)
    Af.data = bf16_round(Af.data)
    ATf.data = bf16_round(ATf.data)
    ineq = np.arange(m) >= P.neq

    def evaluate(xc, yc):
        xc = np.minimum(np.maximum(xc, ls), us)
        mt = kkt_metrics(P, lower, upper, cost, rhs, xc, yc)
        d = (cs - AT @ yc).astype(f32)
        r = (bs - A @ xc).astype(f32)
        return xc, mt, d, r

    def recentre(xh, yh, d, r):
        lp = (ls - xh).astype(f32)
        up = (us - xh).astype(f32)
        yl = np.where(ineq, -yh, 0.0).astype(f32)
        return d, r, lp, up, yl

    xh = np.zeros(n) if x0 is None else np.asarray(x0, float) / dc
    xh = np.where(np.isfinite(xh), xh, 0.0)
    xh = np.minimum(np.maximum(xh, ls), us)
    yh = np.zeros(m) if y0 is None else np.asarray(y0, float) / dr
    yh = np.where(np.isfinite(yh), yh, 0.0)
    yh = np.where(ineq, np.minimum(yh, 0.0), yh)
    omega = float(omega0)
    xh, mt, d, r = evaluate(xh, yh)
    xo, yo = xh, yh
    if converged(mt, tol_primal, tol_dual, tol_gap) or max_iters == 0:
        st = STATUS_OPTIMAL if converged(mt, tol_primal, tol_dual, tol_gap) else STATUS_ITERATION_LIMIT
        return dict(x=np.clip(xo * dc, lower, upper), y=yo * dr, status=st, iterations=0, metrics=mt,
                    omega=omega)
    d, r, lp, up, yl = recentre(xh, yh, d, r)
    dx = np.zeros(n, f32)
    dy = np.zeros(m, f32)
    k = 0
    r_restart = r_prev = best_err = np.inf
    stall = 0
    fell_back = False
    status = STATUS_ITERATION_LIMIT
    it = 0
    for it in range(1, max_iters + 1):
        tau = f32(P.eta / omega)
        sig = f32(P.eta * omega)
        w = f32((k + 1.0) / (k + 2.0))
        g = ATf @ dy
        dxn = np.minimum(np.maximum(dx - tau * (d - g), lp), up).astype(f32)
        xb = (dxn + dxn - dx).astype(f32)
        h = Af @ xb
        dyn = (dy + sig * (r - h)).astype(f32)
        dyn = np.where(ineq, np.minimum(dyn, yl), dyn).astype(f32)
        if rho == 1.0:
            dxnew = (w * xb).astype(f32)
            dynew = (w * (dyn + dyn - dy)).astype(f32)
        else:
            dxnew = (w * ((1 + f32(rho)) * dxn - f32(rho) * dx)).astype(f32)
            dynew = (w * ((1 + f32(rho)) * dyn - f32(rho) * dy)).astype(f32)
        k += 1
        full = (it % check_every == 0) or it >= max_iters
        is_check = full or (8 <= it < check_every and (it & (it - 1)) == 0)
        if not is_check:
            dx, dy = dxnew, dynew
            continue
        ddx = dxn.astype(float) - dx.astype(float)
        ddy = dyn.astype(float) - dy.astype(float)
        rr = np.sqrt(omega * (ddx @ ddx) + (ddy @ ddy) / omega)
        xc, mt, dcand, rcand = evaluate(xh + dxn.astype(float), yh + dyn.astype(float))
        yc = yh + dyn.astype(float)
        xo, yo = xc, yc
        if trace is not None:
            trace.append(dict(it=it, r=rr, omega=omega, **mt))
        if not np.isfinite(rr) or not all(np.isfinite(v) for v in mt.values()):
            status = STATUS_NUMERICAL
            break
        if converged(mt, tol_primal, tol_dual, tol_gap):
            status = STATUS_OPTIMAL
            break
        if it >= max_iters:
            status = STATUS_ITERATION_LIMIT
            break
        if not full:
            dx, dy = dxnew, dynew
            continue
        err = max(mt["primal_residual"] / (1 + mt["x_inf"]), mt["dual_violation"] / (1 + mt["c_inf"]),
                  mt["relative_gap"], mt["relative_kkt_gap"])
        if err < 0.5 * best_err:
            best_err, stall = err, 0
        else:
            stall += 1
        if (stall_checks > 0 and stall >= stall_checks and err <= floor_tol
                and mt["primal_residual"] <= floor_tol * (1 + mt["x_inf"])
                and mt["dual_violation"] <= floor_tol * (1 + mt["c_inf"])):
            status = STATUS_OPTIMAL
            break
        if handoff_stall_checks > 0 and stall >= handoff_stall_checks:
            status = STATUS_HANDOFF
            break
        if fallback_iters > 0 and not fell_back and it >= fallback_iters and (x0 is not None or y0 is not None):
            fell_back = True
            omega = 1.0
            xh, _, d0, r0 = evaluate(np.minimum(np.maximum(np.zeros(n), ls), us), np.zeros(m))
            yh = np.zeros(m)
            xo, yo = xh, yh
            d, r, lp, up, yl = recentre(xh, yh, d0, r0)
            dx = np.zeros(n, f32)
            dy = np.zeros(m, f32)
            k = 0
            r_restart = r_prev = best_err = np.inf
            stall = 0
            continue
        if restarts and (rr <= BETA_SUFFICIENT * r_restart or (rr <= BETA_NECESSARY * r_restart and rr > r_prev)
                         or k >= BETA_ARTIFICIAL * it):
            nx = np.sqrt(float(dxn.astype(float) @ dxn.astype(float)))
            ny = np.sqrt(float(dyn.astype(float) @ dyn.astype(float)))
            if nx > 1e-10 and ny > 1e-10:
                omega = float(np.exp(OMEGA_SMOOTHING * np.log(ny / nx) + (1 - OMEGA_SMOOTHING) * np.log(omega)))
            xh, yh = xc, yc
            d, r, lp, up, yl = recentre(xh, yh, dcand, rcand)
            dx = np.zeros(n, f32)
            dy = np.zeros(m, f32)
            k = 0
            r_restart = rr
            r_prev = np.inf
            continue
        r_prev = rr
        dx, dy = dxnew, dynew
    x_out = xo * dc
    if status != STATUS_HANDOFF:
        x_out = np.clip(x_out, lower, upper)
    return dict(x=x_out, y=yo * dr, status=status, iterations=it, metrics=mt, omega=omega)


def solve_mixed(P: Prepared, lower, upper, cost, rhs=None, *, x0=None, y0=None, omega0=1.0, max_iters=20000,
                check_every=64, tol_primal=1e-9, tol_dual=1e-9, tol_gap=1e-7, fallback_iters=4096, **kw):
    """The engine's default mixed schedule: the re-centred FP32 phase; an
    instance it hands off (a stall above the floor tolerance) continues in
    FP64 from the handed-off point.  Iterations of both phases are summed."""
    kw.setdefault("handoff_stall_checks", 4 * kw.get("stall_checks", 8))
    r = solve_recentred(P, lower, upper, cost, rhs, x0=x0, y0=y0, omega0=omega0, max_iters=max_iters,
                        check_every=check_every, tol_primal=tol_primal, tol_dual=tol_dual, tol_gap=tol_gap,
                        fallback_iters=fallback_iters, **kw)
    if r["status"] != STATUS_HANDOFF:
        return r
    r2 = solve(P, lower, upper, cost, rhs, x0=r["x"], y0=r["y"], omega0=r["omega"], max_iters=max_iters,
               check_every=check_every, tol_primal=tol_primal, tol_dual=tol_dual, tol_gap=tol_gap,
               fallback_iters=fallback_iters)
    r2["iterations"] += r["iterations"]
    return r2
