"""GPU parity of the engine (through the C ABI) against the CPU oracle and
HiGHS golden optima."""
import numpy as np
import pytest
from scipy.sparse import csr_matrix

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import certificate, dfba, pdhg
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]

OBJ_TOL = 1e-6  # relative objective tolerance against HiGHS


def engine(mats, **opt):
    import torch  # noqa: F401
    from co_cultivation_metabolic_atlas_b200.engine import EngineOptions, LPEngine
    return LPEngine(mats, options=EngineOptions(**opt))


def cfg(**kw):
    from co_cultivation_metabolic_atlas_b200.engine import SolveConfig
    return SolveConfig(**kw)


def flat(rows):
    return np.concatenate([np.asarray(r, float).ravel() for r in rows])


def run_single(a, neq, lowers, uppers, costs, rhss=None, config=None, **opt):
    eng = engine([(csr_matrix(np.asarray(a, float)) if not hasattr(a, "tocsr") else a, neq)], **opt)
    k = len(lowers)
    eng.set_instances(np.zeros(k, np.int32), flat(lowers), flat(uppers), flat(costs),
                      None if rhss is None else flat(rhss))
    res = eng.solve(config=config or cfg())
    n = eng.shapes[0][1]
    m = eng.shapes[0][0]
    out = dict(status=res.status.cpu().numpy(), obj=res.objective.cpu().numpy(),
               x=res.x.cpu().numpy()[:k * n].reshape(k, n),
               y=res.y.cpu().numpy()[:k * m].reshape(k, m) if m else np.zeros((k, 0)),
               iters=res.iterations.cpu().numpy(), metrics=res.metrics.cpu().numpy(),
               omega=res.omega.cpu().numpy())
    eng.close()
    return out


# --- the reference's known-answer LPs, through the C ABI ---

@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_kat_inequality_dual_sign(precision):
    r = run_single([[1.0]], 0, [[0.0]], [[2.0]], [[-1.0]], [[1.0]], config=cfg(precision=precision))
    assert r["status"].tolist() == [0]
    np.testing.assert_allclose(r["x"], [[1.0]], atol=1e-8)
    np.testing.assert_allclose(r["y"], [[-1.0]], atol=1e-8)


def test_kat_independent_instances():
    r = run_single([[1.0]], 0, [[0.0], [0.0]], [[2.0], [2.0]], [[-1.0], [-1.0]], [[1.0], [0.5]],
                   config=cfg(precision="fp64"))
    assert r["status"].tolist() == [0, 0]
    np.testing.assert_allclose(r["x"].ravel(), [1.0, 0.5], atol=1e-8)
    np.testing.assert_allclose(r["y"].ravel(), [-1.0, -1.0], atol=3e-7)


def test_kat_box_only_infinite_bound():
    r = run_single([[0.0, 1.0]], 1, [[-np.inf, 0.0]], [[2.0, np.inf]], [[-1.0, 0.0]], [[0.0]],
                   config=cfg(precision="fp64"))
    assert r["status"].tolist() == [0]
    np.testing.assert_allclose(r["x"], [[2.0, 0.0]], atol=1e-10)


def test_kat_infeasible_fails_closed():
    r = run_single([[1.0], [-1.0]], 0, [[-np.inf]], [[np.inf]], [[0.0]], [[0.0, -1.0]],
                   config=cfg(precision="fp64", max_iterations=40, check_every=5))
    assert r["status"].tolist() == [1]
    assert r["iters"].tolist() == [40]


def test_warm_start_at_optimum_needs_no_iterations():
    import torch
    eng = engine([(csr_matrix([[1.0]]), 1)])
    eng.set_instances([0, 0], np.zeros(2), np.full(2, 3.0), np.ones(2), np.array([1.0, 2.0]))
    res = eng.solve(warm_x=np.array([1.0, 2.0]), warm_y=np.array([1.0, 1.0]), config=cfg(precision="fp64"))
    torch.cuda.synchronize()
    assert res.status.cpu().tolist() == [0, 0]
    assert res.iterations.cpu().tolist() == [0, 0]
    eng.close()


def test_invalid_instance_is_flagged_and_others_solve():
    lo = [[0.0], [3.0], [np.nan]]
    up = [[2.0], [2.0], [1.0]]
    r = run_single([[1.0]], 0, lo, up, [[-1.0]] * 3, [[1.0]] * 3, config=cfg(precision="fp64"))
    assert r["status"].tolist() == [0, 3, 3]
    assert np.isnan(r["obj"][1]) and np.isnan(r["x"][2]).all()


# --- iterate parity with the oracle restatement ---

@pytest.mark.parametrize("restarts,iters,staged", [(False, 37, True), (False, 200, True), (True, 640, True),
                                                   (True, 640, False)])
def test_fp64_iterates_match_oracle(restarts, iters, staged):
    model, lower, upper = syn.single_species_workload(3, m=120, n=260)
    P = pdhg.prepare(model.S)
    config = cfg(precision="fp64", max_iterations=iters, check_every=64, tol_primal=0.0,
                 tol_dual=0.0, tol_gap=0.0, restarts=restarts)
    r = run_single(model.S, 120, lower, upper, [model.cost] * 3, config=config, stage_matrix=staged)
    for i in range(3):
        ref = pdhg.solve(P, lower[i], upper[i], model.cost, max_iters=iters, check_every=64,
                         tol_primal=0.0, tol_dual=0.0, tol_gap=0.0, restarts=restarts)
        assert r["status"][i] == 1 and r["iters"][i] == iters
        scale = max(1.0, np.abs(ref["x"]).max())
        np.testing.assert_allclose(r["x"][i], np.clip(ref["x"], lower[i], upper[i]), rtol=0,
                                   atol=1e-9 * scale)
        np.testing.assert_allclose(r["y"][i], ref["y"], rtol=0, atol=1e-9 * max(1.0, np.abs(ref["y"]).max()))
        assert r["omega"][i] == pytest.approx(ref["omega"], rel=1e-9)


# --- the seeded workloads against HiGHS ---

@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_single_species_batch_matches_highs(golden_dir, precision):
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    r = run_single(model.S, 1200, lower, upper, [model.cost] * 8, config=cfg(precision=precision))
    assert (r["status"] == 0).all(), r["status"]
    fun = g["fun"]
    assert np.all(np.abs(r["obj"] - fun) <= OBJ_TOL * np.maximum(1.0, np.abs(fun)))
    for i in range(8):
        cert = certificate.certificate(model.S, np.zeros(1200), lower[i], upper[i], model.cost, 1200,
                                       r["x"][i], r["y"][i])
        assert cert["certificate_passed"], cert
        assert cert["objective"] == pytest.approx(fun[i], rel=OBJ_TOL, abs=OBJ_TOL)


def test_uneven_three_species_batch_in_one_launch(golden_dir):
    g = np.load(golden_dir / "highs_community.npz")
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4)
    eng = engine([(m.S, m.S.shape[0]) for m in models])
    order = [(s, e) for e in range(4) for s in range(3)]  # species interleaved
    lows = {s: dfba.uptake_lower_bounds(models[s], medium, biomass, 0.05) for s in range(3)}
    sid = np.array([s for s, _ in order], np.int32)
    eng.set_instances(sid, flat([lows[s][e] for s, e in order]),
                      flat([models[s].upper for s, _ in order]), flat([models[s].cost for s, _ in order]))
    res = eng.solve(config=cfg(precision="mixed"))
    status = res.status.cpu().numpy()
    obj = res.objective.cpu().numpy()
    x = res.x.cpu().numpy()
    co, ro, _, _ = eng.layout(sid)
    y = res.y.cpu().numpy()
    assert (status == 0).all(), status
    for i, (s, e) in enumerate(order):
        fun = float(g[f"s{s}_fun"][e])
        assert abs(obj[i] - fun) <= OBJ_TOL * max(1.0, abs(fun))
        mdl = models[s]
        n, m = mdl.S.shape[1], mdl.S.shape[0]
        cert = certificate.certificate(mdl.S, np.zeros(m), lows[s][e], mdl.upper, mdl.cost, m,
                                       x[co[i]:co[i] + n], y[ro[i]:ro[i] + m])
        assert cert["certificate_passed"], cert
    eng.close()


def test_spilled_arrays_give_identical_results():
    """Array placement (shared memory, global slab) and matrix staging do not
    change the FP32 arithmetic: the FP32 phase is bit for bit the same."""
    model, lower, upper = syn.single_species_workload(4, m=300, n=650)
    config = cfg(precision="fp32", fp32_tol_gap=1e-5)
    a = run_single(model.S, 300, lower, upper, [model.cost] * 4, config=config)
    b = run_single(model.S, 300, lower, upper, [model.cost] * 4, config=config, max_dynamic_smem=8192)
    c = run_single(model.S, 300, lower, upper, [model.cost] * 4, config=config, stage_matrix=False)
    for other in (b, c):
        np.testing.assert_array_equal(a["x"], other["x"])
        np.testing.assert_array_equal(a["y"], other["y"])
        np.testing.assert_array_equal(a["iters"], other["iters"])
    assert (a["status"] == 5).all()


@pytest.mark.parametrize("opt", [dict(max_dynamic_smem=8192), dict(stage_matrix=False), dict(warps_per_block=32)])
def test_fp64_layouts_agree(opt):
    """The staged unscaled FP64 path (default), the generic path (global
    matrix, spilled arrays) and 32-warp blocks reach the same optima."""
    model, lower, upper = syn.single_species_workload(4, m=300, n=650)
    a = run_single(model.S, 300, lower, upper, [model.cost] * 4, config=cfg(precision="mixed"))
    d = run_single(model.S, 300, lower, upper, [model.cost] * 4, config=cfg(precision="mixed"), **opt)
    assert (a["status"] == 0).all() and (d["status"] == 0).all()
    np.testing.assert_allclose(a["obj"], d["obj"], rtol=1e-8, atol=1e-8)


def test_repeat_solves_are_deterministic():
    model, lower, upper = syn.single_species_workload(6, m=300, n=650)
    a = run_single(model.S, 300, lower, upper, [model.cost] * 6)
    b = run_single(model.S, 300, lower, upper, [model.cost] * 6)
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["iters"], b["iters"])


def test_mixed_precision_keeps_an_accurate_fp64_warm_start():
    """A warm start already at FP32-floor accuracy skips the FP32 phase and
    reaches the FP64 phase unrounded: re-solving from a certified solution
    takes no iterations and returns it bit for bit."""
    model, lower, upper = syn.single_species_workload(3, m=300, n=650)
    eng = engine([(model.S, 300)])
    eng.set_instances(np.zeros(3, np.int32), flat(lower), flat(upper), flat([model.cost] * 3))
    first = eng.solve(config=cfg(precision="mixed"))
    x0 = first.x[:eng.total_cols].clone()
    y0 = first.y[:eng.total_rows].clone()
    again = eng.solve(warm_x=x0, warm_y=y0, warm_omega=first.omega, config=cfg(precision="mixed"))
    assert again.status.cpu().tolist() == [0, 0, 0]
    assert again.iterations.cpu().tolist() == [0, 0, 0]
    np.testing.assert_array_equal(again.x[:eng.total_cols].cpu().numpy(), x0.cpu().numpy())
    eng.close()


# --- the re-centred FP32 phase (default mixed schedule) ---

def test_recentred_iterates_match_oracle():
    """A fixed number of re-centred FP32 iterations (restarts included)
    follows the oracle's restatement to FP32 accuracy."""
    model, lower, upper = syn.single_species_workload(3, m=120, n=260)
    P = pdhg.prepare(model.S)
    iters = 320
    config = cfg(precision="mixed", max_iterations=iters, check_every=64, tol_primal=0.0, tol_dual=0.0,
                 tol_gap=0.0, fp64_stall_checks=0)
    r = run_single(model.S, 120, lower, upper, [model.cost] * 3, config=config)
    for i in range(3):
        ref = pdhg.solve_recentred(P, lower[i], upper[i], model.cost, max_iters=iters, check_every=64,
                                   tol_primal=0.0, tol_dual=0.0, tol_gap=0.0, stall_checks=0,
                                   handoff_stall_checks=0)
        assert r["status"][i] == 1 and r["iters"][i] == iters
        scale = max(1.0, np.abs(ref["x"]).max())
        np.testing.assert_allclose(r["x"][i], ref["x"], rtol=0, atol=1e-5 * scale)
        np.testing.assert_allclose(r["y"][i], ref["y"], rtol=0, atol=1e-5 * max(1.0, np.abs(ref["y"]).max()))


def test_recentred_reaches_fp64_tolerances_in_fp32(golden_dir):
    """The default mixed schedule certifies the three species' LPs in its
    FP32 phase (no FP64 iterations) with the oracle's iteration counts."""
    import torch
    g = np.load(golden_dir / "highs_community.npz")
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4)
    for s, mdl in enumerate(models):
        lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
        eng = engine([(mdl.S, mdl.S.shape[0])])
        eng.set_instances(np.zeros(4, np.int32), lo.ravel(), np.tile(mdl.upper, 4), np.tile(mdl.cost, 4))
        res = eng.solve(config=cfg())
        it32 = eng.phase_iterations().cpu().numpy()
        torch.cuda.synchronize()
        st = res.status.cpu().numpy()
        it = res.iterations.cpu().numpy()
        obj = res.objective.cpu().numpy()
        eng.close()
        assert (st == 0).all(), st
        np.testing.assert_array_equal(it, it32)  # nothing was handed to the FP64 phase
        P = pdhg.prepare(mdl.S)
        ref = pdhg.solve_recentred(P, lo[0], mdl.upper, mdl.cost)
        assert abs(int(it[0]) - ref["iterations"]) <= 64
        fun = g[f"s{s}_fun"]
        assert np.all(np.abs(obj - fun) <= OBJ_TOL * np.maximum(1.0, np.abs(fun)))


@pytest.mark.parametrize("values_phase, second", [(1, "fp32 values"), (0, "pdhg_persistent<double>")])
def test_recentred_handoff_continues_in_the_second_phase(golden_dir, values_phase, second):
    """Instances the re-centred phase hands off (forced by a one-test stall
    rule and short test period) finish in the second phase from the
    compacted work list -- the re-centred kernel with FP32 matrix values by
    default, the FP64 kernel with fp32_values_phase=0; every objective still
    matches HiGHS."""
    import torch
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    eng = engine([(model.S, 1200)])
    eng.set_instances(np.zeros(8, np.int32), flat(lower), flat(upper), flat([model.cost] * 8))
    res = eng.solve(config=cfg(fp64_stall_checks=1, check_every=16, fp32_values_phase=values_phase))
    kernels = eng.phase_kernels()
    assert second in (kernels[1] or ""), kernels
    it32 = eng.phase_iterations().cpu().numpy()
    torch.cuda.synchronize()
    st = res.status.cpu().numpy()
    it = res.iterations.cpu().numpy()
    obj = res.objective.cpu().numpy()
    eng.close()
    assert (st == 0).all(), st
    assert (it > it32).any(), "no instance reached the second phase"
    fun = g["fun"]
    assert np.all(np.abs(obj - fun) <= OBJ_TOL * np.maximum(1.0, np.abs(fun)))


def test_plain_mixed_schedule_still_available(golden_dir):
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(4)
    r = run_single(model.S, 1200, lower[:4], upper[:4], [model.cost] * 4, config=cfg(recentre=False))
    assert (r["status"] == 0).all()
    fun = g["fun"][:4]
    assert np.all(np.abs(r["obj"] - fun) <= OBJ_TOL * np.maximum(1.0, np.abs(fun)))


def test_recentred_streamed_matrix_gives_identical_results():
    """The re-centred phase with the matrix streamed from L2 (the variant for
    species whose matrix does not fit shared memory) computes exactly what
    the staged variant computes."""
    models = syn.community_models()
    medium, biomass = syn.initial_environments(3)
    for s in (0, 2):
        mdl = models[s]
        lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
        a = run_single(mdl.S, mdl.S.shape[0], lo, [mdl.upper] * 3, [mdl.cost] * 3)
        b = run_single(mdl.S, mdl.S.shape[0], lo, [mdl.upper] * 3, [mdl.cost] * 3, stage_matrix=False)
        assert (a["status"] == 0).all() and (b["status"] == 0).all()
        np.testing.assert_array_equal(a["iters"], b["iters"])
        np.testing.assert_array_equal(a["x"], b["x"])
        np.testing.assert_array_equal(a["y"], b["y"])


def test_large_species_solve_in_the_streamed_recentred_phase():
    """Scale workload species (3,000 x 6,000 class, fixed exchange bounds,
    duplicated reversible columns) exceed shared memory for the staged
    matrix; the streamed re-centred phase certifies them with HiGHS's
    objectives."""
    import torch
    from oracle import highs
    models = syn.community_models(syn.LARGE_SIZES, fixed_fraction=0.2, duplicate_fraction=0.05)
    sid, bounds = syn.scale_batch(models, 6, mix=(1, 1, 1), seed=2)
    eng = engine([(m.S, m.S.shape[0]) for m in models])
    lo = np.concatenate([b[0].ravel() for b in bounds])
    up = np.concatenate([b[1].ravel() for b in bounds])
    cost = np.concatenate([np.tile(m.cost, len(b[0])) for m, b in zip(models, bounds)])
    eng.set_instances(sid, lo, up, cost)
    res = eng.solve(config=cfg())
    torch.cuda.synchronize()
    st, obj = res.status.cpu().numpy(), res.objective.cpu().numpy()
    eng.close()
    assert (st == 0).all(), st
    k = 0
    for s, (mdl, (lw, uw)) in enumerate(zip(models, bounds)):
        for i in range(len(lw)):
            hst, fun, _, _ = highs.solve_one(mdl.S, lw[i], uw[i], mdl.cost, method="highs-ipm")
            assert hst == 0
            assert abs(obj[k] - fun) <= OBJ_TOL * max(1.0, abs(fun))
            k += 1


def test_iteration_hints_and_instance_data_rebinding():
    """Hints >= the test period skip the early termination tests (an instance
    that would stop at iteration 8 stops at the first full test instead, with
    the same optimum); re-pointing the batch at new arrays of the same layout
    solves exactly what set_instances with those arrays solves."""
    import torch
    model, lower, upper = syn.single_species_workload(4, m=300, n=650)
    eng = engine([(model.S, 300)])
    eng.set_instances(np.zeros(4, np.int32), flat(lower), flat(upper), flat([model.cost] * 4))
    first = eng.solve(config=cfg())
    x0, y0 = first.x[:eng.total_cols].clone(), first.y[:eng.total_rows].clone()
    lo2 = lower.copy()
    lo2[:, :model.n_exchange] *= 0.999
    lo2_d = torch.as_tensor(flat(lo2), device="cuda")
    eng.set_instance_data(lo2_d, flat(upper), flat([model.cost] * 4))
    rebound = eng.solve(config=cfg())
    plain = eng.solve(warm_x=x0, warm_y=y0, warm_omega=first.omega, config=cfg())
    eng.set_iteration_hints(torch.full((4,), 1000, dtype=torch.int32, device="cuda"))
    hinted = eng.solve(warm_x=x0, warm_y=y0, warm_omega=first.omega, config=cfg())
    eng.set_iteration_hints(None)
    torch.cuda.synchronize()
    ip, ih = plain.iterations.cpu().numpy(), hinted.iterations.cpu().numpy()
    assert (plain.status.cpu().numpy() == 0).all() and (hinted.status.cpu().numpy() == 0).all()
    assert np.all(ih >= np.minimum(ip, 64)) and np.all(ih % 64 == 0)
    np.testing.assert_allclose(hinted.objective.cpu().numpy(), plain.objective.cpu().numpy(), rtol=1e-7, atol=1e-8)
    ref = run_single(model.S, 300, lo2, upper, [model.cost] * 4)
    np.testing.assert_array_equal(rebound.iterations.cpu().numpy(), ref["iters"])
    np.testing.assert_array_equal(rebound.x[:eng.total_cols].cpu().numpy().reshape(4, -1), ref["x"])
    eng.close()


def test_graph_captured_dfba_steps_equal_eager_steps():
    """dFBA steps replayed from CUDA graphs (uptake bounds, the engine's
    launches, Euler updates) give bit-for-bit the states of eager steps."""
    import torch
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    models = syn.community_models()
    medium, biomass = syn.initial_environments(24, seed=5)
    a = DeviceCommunity(models, medium, biomass, warm_start="extrapolate")
    b = DeviceCommunity(models, medium, biomass, warm_start="extrapolate")
    for _ in range(3):
        a.step()
        b.step()
    b.capture()
    its_a, its_b = [], []
    for _ in range(7):
        its_a.append(a.step().iterations.clone())
        its_b.append(b.step().iterations.clone())
    torch.cuda.synchronize()
    for x, y in zip(its_a, its_b):
        assert torch.equal(x, y)
    assert torch.equal(a.medium, b.medium) and torch.equal(a.biomass, b.biomass)
    assert torch.equal(a.result.x, b.result.x)
    a.close()
    b.close()


def test_patched_entries_solve_per_instance_matrices(golden_dir):
    """Per-instance matrix entries: every instance solves its own matrix
    (shared matrix plus its deltas at two patched positions, one of them not
    a structural nonzero); objectives match HiGHS on each instance's full
    matrix, and the same LPs without deltas match the shared matrix."""
    import torch
    from oracle import highs
    model, lower, upper = syn.single_species_workload(4, m=120, n=260)
    S = model.S.tocsr()
    r0, c0 = 5, int(S.indices[S.indptr[5]])          # an existing entry
    zr = np.flatnonzero(np.asarray(S[:, model.biomass].todense()).ravel() == 0)[0]
    rows, cols = [r0, int(zr)], [c0, model.biomass]  # and a structural zero
    deltas = np.array([[0.5, -0.3], [-0.25, 0.1], [0.0, 0.0], [1.0, 0.2]])
    eng = engine([(S, 120)])
    eng.set_instances(np.zeros(4, np.int32), flat(lower), flat(upper), flat([model.cost] * 4))
    eng.set_patches(0, rows, cols)
    eng.set_patch_values(torch.as_tensor(deltas, device="cuda"))
    res = eng.solve(config=cfg())
    torch.cuda.synchronize()
    st, obj = res.status.cpu().numpy(), res.objective.cpu().numpy()
    eng.close()
    assert (st == 0).all(), st
    for i in range(4):
        Si = S.tolil(copy=True)
        for (r, c), d in zip(zip(rows, cols), deltas[i]):
            Si[r, c] = Si[r, c] + d
        hst, fun, _, _ = highs.solve_one(Si.tocsr(), lower[i], upper[i], model.cost)
        assert hst == 0
        assert abs(obj[i] - fun) <= OBJ_TOL * max(1.0, abs(fun)), (i, obj[i], fun)
