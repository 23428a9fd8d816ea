"""Benchmark: HiGHS-certified FBA LPs/s on the 4,096-environment three-species
dFBA workload (one step = 12,288 LPs of uneven size, solved in one persistent
launch per precision phase, then the Euler update), warm start vs cold.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]
    python bench.py --profile fba|cooperative|mlp [--envs E] [--steps K]

``--profile`` runs a short, untimed driver of one workload for an external
profiler (ncu) instead of the benchmark: warm-started dFBA steps of the FBA
community (per-step phase instance-iterations and times printed), steps of
the cooperative community (the last one inside the NVTX range
``coop_step``), or inference and training passes of the warm-start network
(random weights; TFLOP/s of the GEMMs printed).

Prints one JSON line (rank 0).  Roofline model of the dominant kernel
(the re-centred PDHG phase), a design that streams everything from HBM:
w (3 n + 3 m + 2 n_medium) bytes per instance-iteration (w = 4 bytes per
FP32 value) plus, per species and iteration of its longest instance, the
matrix and its transpose, 2 (nnz (w + 4) + 4 (m + 1)) bytes; their sum over
the phase's launch divided by its CUDA-event time, against the measured
copy bandwidth.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "HiGHS-certified FBA LPs/s (1e-6 rel obj); warm-start vs cold PDHG, same B200"
UNIT = "LPs/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("product", "reference"), default="product")
    ap.add_argument("--envs", type=int, default=4096, help="environments per GPU")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=("mixed", "fp64", "fp32"))
    ap.add_argument("--cpu-sample", type=int, default=48,
                    help="reference arm: LPs per step in its bounded CPU HiGHS sample (a third per species)")
    ap.add_argument("--highs-check", type=int, default=1536,
                    help="product arm: LPs of one step checked against HiGHS (a third per species); their CPU "
                         "time is the cpu_baseline")
    ap.add_argument("--drop-in", type=int, default=1,
                    help="1: also time one step's LPs through B200LPBackend.solve_batch (host preparation included)")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = the same number of steps as the timed region")
    ap.add_argument("--no-cold", action="store_true")
    ap.add_argument("--warm", default="extrapolate", choices=("previous", "extrapolate"),
                    help="temporal base of the warm start (the product arm without --learned)")
    ap.add_argument("--learned", type=int, default=1,
                    help="1: train the learned warm start and measure it as the product arm (the temporal base "
                         "alone and cold PDHG are measured beside it)")
    ap.add_argument("--graphs", type=int, default=1,
                    help="1: capture the dFBA step in CUDA graphs after the warm-up and replay them when timed")
    ap.add_argument("--learn-seeds", type=int, default=2)
    ap.add_argument("--learn-steps", type=int, default=16)
    ap.add_argument("--learn-epochs", type=int, default=10)
    ap.add_argument("--workload", default="fba", choices=("fba", "cooperative"),
                    help="fba: the per-species FBA step (headline); cooperative: the three-stage shared-medium "
                         "community LP per environment")
    ap.add_argument("--coop-sample", type=int, default=6, help="environments in the cooperative CPU sample")
    ap.add_argument("--profile", default=None, choices=("fba", "cooperative", "mlp"),
                    help="run a short profiling driver of one workload instead of the benchmark")
    ap.add_argument("--warps", type=int, default=16, help="warps per CTA of the PDHG kernels")
    ap.add_argument("--coop-growth-cap", type=float, default=0.005,
                    help="coexistence growth upper bound (the reference simulator's 0.005 /h; <= 0: the solver "
                         "default 10)")
    return ap.parse_args()


def workload_config(args, lps):
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    return {"workload": f"community dFBA step: {args.envs} envs x 3 species "
                        f"({', '.join(f'{m}x{n}' for m, n in syn.COMMUNITY_SIZES)}), {lps} LPs/step, dt=0.05 h",
            "envs_per_gpu": args.envs, "lps_per_step": lps, "seed": args.seed,
            "precision": args.precision, "warps_per_cta": args.warps,
            "l2": "inputs larger than L2 (bounds+objective of one step > 600 MB), no flush"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(parts)
            except ValueError:
                pass
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- peaks
def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


PROFILE_FOR_KERNEL = {"pdhg_recentred_pair": "pdhg_recentred_pair_community_small.txt",
                      "pdhg_recentred<staged>": "pdhg_recentred_community_small.txt"}


def profiled_figure(kernel, key):
    """A per-instance-iteration figure (``key: value ...`` line) from the
    committed ncu summary of a smaller case of the same step for ``kernel``
    (profiles/), or None."""
    name = PROFILE_FOR_KERNEL.get(kernel)
    p = ROOT / "profiles" / name if name else None
    if p is None or not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ----------------------------------------------------------------------------- CPU HiGHS
def cpu_highs_sample(models, lowers, per_species, seed, cores=None):
    """HiGHS (scipy linprog highs-ds, one thread per LP) over all host cores on
    a seeded sample of ``per_species`` LPs per species.  Returns (LPs/s, cores,
    wall seconds, [(species, env, fun)])."""
    from oracle import highs
    cores = cores or len(os.sched_getaffinity(0))
    rng = np.random.default_rng(seed + 99)
    S_list, lo, up, c, tags = [], [], [], [], []
    for s, mdl in enumerate(models):
        envs = rng.choice(lowers[s].shape[0], min(per_species, lowers[s].shape[0]), replace=False)
        for e in envs:
            S_list.append(mdl.S)
            lo.append(lowers[s][e])
            up.append(mdl.upper)
            c.append(mdl.cost)
            tags.append((s, int(e)))
    res, wall = highs.solve_batch(S_list, lo, up, c, workers=cores)
    funs = [(t[0], t[1], r[1] if r[0] == 0 else None) for t, r in zip(tags, res)]
    return len(res) / wall, cores, wall, funs


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from oracle import dfba
    models = syn.community_models(seed=args.seed)
    medium, biomass = syn.initial_environments(args.envs, seed=args.seed)
    lowers = [dfba.uptake_lower_bounds(m, medium, biomass, 0.05) for m in models]
    per = max(4, args.cpu_sample // 3)
    rates, walls = [], []
    cores = None
    for k in range(args.warmup + args.steps):
        rate, cores, wall, _ = cpu_highs_sample(models, lowers, per, args.seed + k)
        if k >= args.warmup:
            rates.append(rate)
            walls.append(wall)
    value = statistics.mean(rates)
    lps = args.envs * len(models)
    # one step of this arm is the bounded sample (3 * per LPs); the time a
    # whole 12,288-LP step would take at this rate is reported beside it
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
            "projected_full_step_ms": 1e3 * lps / value,
            "step": f"a bounded sample of {3 * per} of the step's {lps} LPs",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; no public dataset)", "config": workload_config(args, lps),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{3 * per} LPs per step (seeded, {per} per species) of the step's "
                                       f"{lps} LPs; scipy.optimize.linprog(method='highs-ds'), one HiGHS "
                                       f"thread per LP, thread pool over all cores (the reference's "
                                       f"ParallelCpuLP pattern)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- product arm
def timed_trajectory(com, args, barrier, pdhg_launches):
    """Warm-up, (graph capture,) then ``args.steps`` timed dFBA steps.  The
    whole region is timed with CUDA events on the stream; each step's PDHG
    launches are bracketed by the engine's timing slots (external event
    nodes inside the captured graphs), read two steps behind so the host
    never drains the queue.  Returns (ms, certified, iterations, launches,
    per-step PDHG kernel ms)."""
    import torch
    for _ in range(args.warmup):
        com.step()
    graphs = bool(args.graphs and args.warmup >= 2)
    if graphs:
        com.capture()  # the timed steps replay CUDA graphs of whole dFBA steps
    else:
        com.engine.timing_slots(3)
    torch.cuda.synchronize()
    barrier()
    stream = torch.cuda.current_stream()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    certified, iters, kernel_ms, slots = [], [], [], []
    launches = 0

    def harvest(slot):
        t32, t64 = com.engine.slot_times(slot)
        kernel_ms.append(t32 + t64)

    start.record(stream)
    for j in range(args.steps):
        if not graphs:
            com.engine.use_timing_slot(j % 3)
        st = com.step()
        slots.append(com.last_replay_slot() if graphs else j % 3)
        certified.append(st.certified.clone())
        iters.append(st.iterations.clone())
        launches += pdhg_launches
        if j >= 2:
            harvest(slots[j - 2])
    stop.record(stream)
    torch.cuda.synchronize()
    for j in range(max(0, args.steps - 2), args.steps):
        harvest(slots[j])
    if not graphs:
        com.engine.use_timing_slot(-1)
    barrier()
    ms = start.elapsed_time(stop)
    cert = int(sum(int(c.item()) for c in certified))
    it = torch.stack(iters).cpu().numpy()  # (steps, lps)
    return ms, cert, it, launches, kernel_ms


def streaming_bytes(models, species_id, it, w=4):
    """Algorithmic bytes of one launch of the PDHG phase in the streaming
    model: per instance-iteration w (3 n + 3 m + 2 n_medium), plus per
    species and iteration of its longest instance the matrix and its
    transpose, 2 (nnz (w + 4) + 4 (m + 1))."""
    per_inst = np.array([w * (3 * m.S.shape[1] + 3 * m.S.shape[0] + 2 * len(m.medium_columns))
                         for m in models], dtype=np.float64)
    total = float(np.sum(it.astype(np.float64) * per_inst[species_id]))
    for s, m in enumerate(models):
        its = it[species_id == s]
        total += float(its.max() if its.size else 0) * 2 * (m.S.nnz * (w + 4) + 4 * (m.S.shape[0] + 1))
    return total


def certificate_summary(res, lps):
    """Distribution of the kernel's FP64 certificate fields over every LP of
    a step (primal residual, dual violation, relative KKT gap)."""
    mt = res.metrics.cpu().numpy()
    st = res.status.cpu().numpy()
    out = {"lps": int(lps), "optimal": int(np.sum(st == 0))}
    for k, name in enumerate(("primal", "dual", "kkt_gap")):
        v = mt[:, k]
        out[name] = {"max": float(np.max(v)), "p99": float(np.percentile(v, 99)), "median": float(np.median(v))}
    out["gate_passed"] = int(np.sum((st == 0) & (mt[:, 0] <= 1e-5) & (mt[:, 1] <= 1e-7) & (mt[:, 2] <= 1e-7)))
    return out


def drop_in_measure(models, lower_host, envs, device):
    """The reference-facing drop-in (``B200LPBackend.solve_batch``) on one
    step's LPs as ``linprog``-kwargs requests: a first call builds the engine,
    a second call (warm-started from the first) is reported with its host
    preparation, GPU solve and total seconds."""
    from co_cultivation_metabolic_atlas_b200.backend import B200LPBackend
    reqs, ids = [], []
    for s, m in enumerate(models):
        zeros = np.zeros(m.S.shape[0])
        for e in range(envs):
            reqs.append((m.cost, dict(A_eq=m.S, b_eq=zeros, bounds=np.column_stack([lower_host[s][e], m.upper]),
                                      method="highs-ds")))
            ids.append((s, e))
    be = B200LPBackend(mode="previous", device=device)
    be.solve_batch(reqs, environment_ids=ids)
    rows = be.solve_batch(reqs, environment_ids=ids)
    h = be.history[-1]
    be.close()
    return {"requests": len(reqs), "accepted": int(sum(r.success for r in rows)),
            "host_preparation_seconds": h["host_preparation_seconds"], "solve_seconds": h["solve_seconds"],
            "total_seconds": h["total_seconds"], "lps_per_s": len(reqs) / h["total_seconds"],
            "api": "B200LPBackend.solve_batch(requests) with scipy-linprog kwargs, warm-started from the previous "
                   "call (mode='previous')"}


def run_product(args):
    import torch

    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    from co_cultivation_metabolic_atlas_b200.engine import SolveConfig

    from co_cultivation_metabolic_atlas_b200.distributed import Ranks

    ranks = Ranks("nccl")
    world, rank, local, dev = ranks.world, ranks.rank, ranks.local_rank, ranks.device
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum

    models = syn.community_models(seed=args.seed)
    medium, biomass = syn.initial_environments(args.envs, seed=ranks.environment_seed(args.seed))
    cfg = SolveConfig(precision=args.precision)
    lps = args.envs * len(models)
    # kernels of this project per step: the PDHG launches (re-centred FP32 +
    # FP64 hand-off phase in the mixed schedule); the network runs only at an
    # environment's first step, which is a warm-up step
    pdhg_launches = 2 if args.precision == "mixed" else 1

    # --- learned warm start: networks trained on the engine's own rollouts
    # (seeds disjoint from the evaluated environments) ---
    ws = None
    learned_info = None
    if args.learned:
        from co_cultivation_metabolic_atlas_b200 import train_warmstart as tw
        t0 = time.perf_counter()
        data = tw.build_dataset(models, envs=args.envs, steps=args.learn_steps,
                                seeds=ranks.training_seeds(args.seed, args.learn_seeds),
                                config=cfg, device=dev, log=lambda *_: None)
        # data-parallel over the ranks' own rollouts (one network for the job)
        ws, losses = tw.fit(models, data, epochs=args.learn_epochs, device=dev, log=lambda *_: None, ranks=ranks)
        torch.cuda.synchronize()
        learned_info = {"training_pairs": int(data.F.shape[0]), "final_train_mse_standardised": losses[-1],
                        "train_seconds": time.perf_counter() - t0,
                        "model": "MLP 44 -> 4 x 512 GELU -> x,y of 3 species, BF16 tcgen05 kernels; seeds an "
                                 "environment's first solve, the temporal base seeds the later ones",
                        "training": f"data-parallel over {world} rank(s)"}
        del data

    from co_cultivation_metabolic_atlas_b200.engine import EngineOptions
    options = EngineOptions(warps_per_block=args.warps)

    def trajectory(warm, learned=None):
        com = DeviceCommunity(models, medium, biomass, config=cfg, warm_start=warm, learned=learned, device=dev,
                              options=options)
        first = None
        if args.warmup:
            # the first (history-free) step: the network's seed or a cold start
            com.step()
            first = com.prev.iterations.float().mean().item()
            args_w = argparse.Namespace(**{**vars(args), "warmup": args.warmup - 1})
        else:
            args_w = args
        ms, cert, it, launches, kms = timed_trajectory(com, args_w, barrier, pdhg_launches)
        return com, ms, cert, it, launches, kms, first

    headline = "learned" if ws is not None else args.warm
    with ClockSampler(local) as clocks:
        com, ms, cert, it, launches, kernel_ms, first_its = trajectory(headline, learned=ws)
    clock_summary = clocks.summary()
    ms_max = max_over_ranks(ms)
    cert_all = sum_over_ranks(cert)
    value = cert_all / (ms_max / 1e3)

    # --- roofline of the dominant kernel over the timed steps themselves:
    # streaming-model bytes of every timed step's PDHG launches over their
    # CUDA-event durations (graph event nodes) ---
    peak, peak_kind = hbm_peak()
    w = 4 if args.precision != "fp64" else 8
    sid = com.species_id
    step_bytes = [streaming_bytes(models, sid, it[j], w) for j in range(it.shape[0])]
    kernel_total_ms = float(sum(kernel_ms))
    achieved = sum(step_bytes) / (kernel_total_ms / 1e3) / 1e9
    inst_its = int(it.sum())
    first_kernel, fp64_kernel = com.engine.phase_kernels()
    tpi = profiled_figure(first_kernel, "dram_bytes_per_instance_iteration")
    traffic = None if tpi is None else tpi * inst_its / it.shape[0]
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{peak_kind} copy bandwidth",
                "kernel": first_kernel, "fp64_phase_kernel": fp64_kernel, "algorithmic_bytes": sum(step_bytes) / len(step_bytes),
                "kernel_ms": kernel_total_ms / len(kernel_ms), "kernel_share_of_step": kernel_total_ms / ms,
                "instance_iterations_per_launch": inst_its / it.shape[0],
                "measured_on": f"the {args.steps} timed steps (CUDA events around each step's PDHG launches)"}
    wf = profiled_figure(first_kernel, "shared_wavefronts_per_instance_iteration")
    sm_mhz = clock_summary.get("sm_mhz") or 1965.0
    if wf is not None:
        sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
        onchip_peak = sm_count * 128.0 * sm_mhz * 1e6 / 1e9
        onchip = wf * 128.0 * inst_its / (kernel_total_ms / 1e3) / 1e9
        roofline["shared_memory"] = {"achieved": onchip, "peak": onchip_peak, "unit": "GB/s", "frac": onchip / onchip_peak,
                                     "wavefronts_per_instance_iteration": wf,
                                     "model": "ncu shared-memory wavefronts per instance-iteration x 128 B, over "
                                              "SMs x 128 B/clk at the sampled SM clock"}

    # --- the last timed step's certificate distribution over all its LPs,
    # and HiGHS on a sample of its LPs (objective check + CPU baseline) ---
    res = com.prev
    cert_dist = certificate_summary(res, lps)
    cpu = None
    highs_check = None
    lower_host = None
    if rank == 0:
        # the bounds the last step was solved with are the state's uptake
        # bounds before its Euler update: recompute them from the previous
        # state is not possible, so solve one more eager step and check it
        com.uptake_bounds()
        res = com.solve()
        torch.cuda.synchronize()
        lower = com.lower.cpu().numpy()
        co = com.col_offsets.cpu().numpy()
        lower_host = []
        for s, m in enumerate(models):
            n = m.S.shape[1]
            base = int(co[s * args.envs])
            lower_host.append(lower[base:base + args.envs * n].reshape(args.envs, n))
        per = max(4, args.highs_check // 3)
        rate, cores, wall, funs = cpu_highs_sample(models, lower_host, per, args.seed)
        obj = res.objective.cpu().numpy()
        status = res.status.cpu().numpy()
        errs = []
        agree = 0
        for s, e, fun in funs:
            i = s * args.envs + e
            if fun is None or status[i] != 0:
                continue
            err = abs(obj[i] - fun) / max(1.0, abs(fun))
            errs.append(err)
            agree += err <= 1e-6
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{len(funs)} LPs ({per} per species, seeded) of one step's {lps}; "
                         f"scipy.optimize.linprog(method='highs-ds'), one HiGHS thread per LP, thread "
                         f"pool over all cores (ParallelCpuLP pattern); {wall:.1f} s wall"}
        highs_check = {"sampled": len(funs), "within_1e-6": int(agree),
                       "max_rel_obj_err": max(errs) if errs else None,
                       "step_certificates": certificate_summary(res, lps)}
    com.close()
    com = None

    # --- the same trajectory without the network (temporal base only) and cold ---
    extrap = None
    if ws is not None:
        com_e, ms_e, cert_e, it_e, _, _, first_e = trajectory(args.warm)
        com_e.close()
        extrap = {"value": sum_over_ranks(cert_e) / (max_over_ranks(ms_e) / 1e3),
                  "mean_iterations": float(np.mean(it_e)), "warm_start": args.warm,
                  "first_step_mean_iterations": first_e}
    cold = None
    cold_iters = None
    cold_first = None
    if not args.no_cold:
        com_c, ms_c, cert_c, it_c, _, _, cold_first = trajectory("cold")
        cold = sum_over_ranks(cert_c) / (max_over_ranks(ms_c) / 1e3)
        cold_iters = float(np.mean(it_c))
        com_c.close()
    # --- e2e through the public engine API with host buffers ---
    e2e = run_e2e(args, models, medium, biomass, cfg, dev, barrier, max_over_ranks, sum_over_ranks, ws)
    drop_in = None
    if rank == 0 and args.drop_in and lower_host is not None:
        drop_in = drop_in_measure(models, lower_host, args.envs, dev)

    if rank == 0:
        warm_desc = {"previous": "previous-step solution",
                     "extrapolate": "extrapolated from the last two step solutions"}[args.warm]
        if ws is not None:
            warm_desc = ("learned: MLP prediction from the medium state at an environment's first step, then the "
                         "temporal base (" + warm_desc + ")")
        if learned_info is not None:
            learned_info.update(value=value, mean_iterations=float(np.mean(it)),
                                first_step_mean_iterations=first_its,
                                first_step_iterations_vs_cold=(first_its / cold_first) if cold_first else None)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "cuda_graphs": bool(args.graphs and args.warmup >= 3),
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "fp32+fp64" if args.precision == "mixed" else args.precision,
                "data": "synthetic (seeded generator; no public dataset)",
                "config": workload_config(args, lps),
                "warm_start": warm_desc, "parallelism": f"env-sharded x{world}",
                "certified_fraction": cert / (lps * args.steps),
                "env_steps_per_s": world * args.envs * args.steps / (ms_max / 1e3),
                "iterations": {"mean": float(np.mean(it)), "p50": float(np.median(it)),
                               "p99": float(np.percentile(it, 99)), "max": int(np.max(it))},
                "cold_value": cold, "warm_vs_cold": (value / cold) if cold else None,
                "cold_mean_iterations": cold_iters, "cold_first_step_mean_iterations": cold_first,
                "without_network": extrap, "network_gain": (value / extrap["value"]) if extrap else None,
                "learned": learned_info, "learned_vs_cold": (value / cold) if (ws is not None and cold) else None,
                "roofline": roofline, "cpu_baseline": cpu, "highs_check": highs_check,
                "timed_step_certificates": cert_dist, "e2e": e2e, "drop_in": drop_in,
                "gpu_launches": launches, "clocks": clock_summary}
        print(json.dumps(line), flush=True)
    ranks.close()


class _HostDrivenState:
    """What a warm-start proposal reads of a community (state and the last
    two results), fed from host copies in the end-to-end arm."""

    def __init__(self, E, total_cols, total_rows):
        self.E = E
        self.total_cols, self.total_rows = total_cols, total_rows
        self.medium = self.biomass = None
        self.prev = self.prev2 = None


def run_e2e(args, models, medium, biomass, cfg, dev, barrier, max_over_ranks, sum_over_ranks, ws=None):
    """Same metric through the public ``LPEngine`` API with HOST inputs: every
    step copies that step's lower bounds (the only per-step input of a dFBA
    step; upper bounds and objectives are bound once) and, for the learned
    warm start, the medium state from pinned host memory, proposes the warm
    start, solves, and reads status, objectives, metrics and fluxes back."""
    import torch

    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    from co_cultivation_metabolic_atlas_b200.engine import EngineOptions
    com = DeviceCommunity(models, medium, biomass, config=cfg, warm_start=args.warm, device=dev,
                          options=EngineOptions(warps_per_block=args.warps))
    K = args.e2e_steps if args.e2e_steps > 0 else args.steps
    host_lower, host_state = [], []
    for _ in range(args.warmup + K):
        host_state.append((com.medium.cpu().pin_memory(), com.biomass.cpu().pin_memory()))
        com.uptake_bounds()
        host_lower.append(com.lower.cpu().pin_memory())
        res = com.solve()
        com.integrate(res)
    up_h = com.upper.cpu().pin_memory()
    c_h = com.cost.cpu().pin_memory()
    eng = com.engine
    lo_d, up_d, c_d = eng._bound[0], eng._bound[1], eng._bound[2]
    out = [eng.allocate_result() for _ in range(3)]
    wx = torch.empty(eng.total_cols, dtype=torch.float64, device=dev)
    wy = torch.empty(max(1, eng.total_rows), dtype=torch.float64, device=dev)
    x_h = torch.empty(eng.total_cols, dtype=torch.float64).pin_memory()
    st_h = torch.empty(eng.count, dtype=torch.int32).pin_memory()
    ob_h = torch.empty(eng.count, dtype=torch.float64).pin_memory()
    mt_h = torch.empty((eng.count, 8), dtype=torch.float64).pin_memory()
    state = _HostDrivenState(com.E, eng.total_cols, eng.total_rows)
    med_d = torch.empty_like(com.medium)
    bio_d = torch.empty_like(com.biomass)
    hist = []

    # upper bounds and objectives do not change between dFBA steps: bound once
    up_d.copy_(up_h)
    c_d.copy_(c_h)

    def one(k, o):
        lo_d.copy_(host_lower[k], non_blocking=True)
        eng.set_iteration_hints(hist[-1].iterations if hist else None)
        if ws is not None:
            med_d.copy_(host_state[k][0], non_blocking=True)
            bio_d.copy_(host_state[k][1], non_blocking=True)
            state.medium, state.biomass = med_d, bio_d
            state.prev = hist[-1] if hist else None
            state.prev2 = hist[-2] if len(hist) > 1 else None
            px, py, po = ws.propose(state, k / 960)
            kw = dict(warm_x=px, warm_y=py, warm_omega=po)
        elif not hist:
            kw = {}
        elif args.warm == "extrapolate" and len(hist) >= 2:
            torch.sub(hist[-1].x[:eng.total_cols] * 2.0, hist[-2].x[:eng.total_cols], out=wx)
            torch.sub(hist[-1].y[:eng.total_rows] * 2.0, hist[-2].y[:eng.total_rows], out=wy[:eng.total_rows])
            kw = dict(warm_x=wx, warm_y=wy[:eng.total_rows], warm_omega=hist[-1].omega)
        else:
            kw = dict(warm_x=hist[-1].x[:eng.total_cols], warm_y=hist[-1].y[:eng.total_rows],
                      warm_omega=hist[-1].omega)
        r = eng.solve(config=cfg, out=o, **kw)
        x_h.copy_(r.x[:eng.total_cols], non_blocking=True)
        st_h.copy_(r.status, non_blocking=True)
        ob_h.copy_(r.objective, non_blocking=True)
        mt_h.copy_(r.metrics, non_blocking=True)
        hist.append(r)
        del hist[:-2]
        return r

    for k in range(args.warmup):
        one(k, out[k % 3])
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    cert = 0
    for k in range(args.warmup, args.warmup + K):
        one(k, out[k % 3])
        torch.cuda.synchronize()
        st = st_h.numpy()
        mt = mt_h.numpy()
        cert += int(np.sum((st == 0) & (mt[:, 0] <= 1e-5) & (mt[:, 1] <= 1e-7) & (mt[:, 2] <= 1e-7)))
    wall = time.perf_counter() - t0
    barrier()
    com.close()
    value = sum_over_ranks(cert) / max_over_ranks(wall)
    h2d = eng.total_cols * 8 + (0 if ws is None else (med_d.numel() + bio_d.numel()) * 8)
    d2h = eng.total_cols * 8 + eng.count * (4 + 8 + 64)
    return {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": K, "warm_start": "learned" if ws is not None else args.warm,
            "api": "LPEngine.solve over the C ABI (fbalp_engine_solve) with pinned host buffers"}


# ----------------------------------------------------------------------------- cooperative LP
COOP_METRIC = "certified cooperative community stage LPs/s (max-min growth + parsimonious exchange per env-step)"


def coop_config(args, st, stages):
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    return {"workload": f"cooperative dFBA step: {args.envs} envs, one joint LP per env and stage over 3 species "
                        f"({', '.join(f'{m}x{n}' for m, n in syn.COMMUNITY_SIZES)}) + {st.n_medium_rows} shared "
                        f"medium rows: stage 1 {st.m1}x{st.n1}, stage 3 {st.m3}x{st.n3}; {stages} stage LPs/env-step, "
                        f"dt=0.05 h",
            "envs_per_gpu": args.envs, "seed": args.seed, "community_seed": syn.COOPERATIVE_SEED,
            "l2": "inputs larger than L2 (per-stage bounds of one step > 400 MB), no flush"}


def coop_cpu_sample(com_state, members, sample, seed, cap, cores=None):
    """The oracle's exact-CPU cooperative solve (HiGHS, the reference's
    stage sequence) on ``sample`` environments of one state, one HiGHS
    thread per environment over all cores.  Returns (stage LPs/s, cores,
    wall, {env: solution})."""
    from concurrent.futures import ThreadPoolExecutor

    from co_cultivation_metabolic_atlas_b200 import cooperative as coop
    from oracle import cooperative as oc
    X, C, lo, up = com_state
    st = coop.CommunityStructure(members)
    growth = [(s, int(st.growth_cols[s]), float(st.growth_coef[s])) for s in range(st.n_species)]
    orig = {int(c): o for c, o in zip(st.relax_cols, st.relax_orig)}
    blocks = [m.S for m in members]
    rng = np.random.default_rng(seed + 7)
    envs = rng.choice(X.shape[0], min(sample, X.shape[0]), replace=False)
    cores = cores or len(os.sched_getaffinity(0))

    def one(i):
        return int(i), oc.solve(blocks, growth, st.exchange_terms, st.global_objective, lo[i], up[i],
                                dict(enumerate(X[i])), dict(zip(st.metabolites, C[i])), 0.05,
                                original_lower=orig, maximum_coexistence_growth=cap)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=min(cores, len(envs))) as pool:
        sols = dict(pool.map(one, envs))
    wall = time.perf_counter() - t0
    lps = sum(len(s.stages) for s in sols.values())
    return lps / wall, min(cores, len(envs)), wall, sols


def run_cooperative(args):
    import torch

    from co_cultivation_metabolic_atlas_b200 import cooperative as coop
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from co_cultivation_metabolic_atlas_b200.distributed import Ranks

    ranks = Ranks("nccl")
    world, rank, local, dev = ranks.world, ranks.rank, ranks.local_rank, ranks.device
    models = syn.community_models(seed=syn.COOPERATIVE_SEED)
    medium, biomass = syn.initial_environments(args.envs, seed=ranks.environment_seed(args.seed))
    cap = args.coop_growth_cap if args.coop_growth_cap > 0 else None
    stages = 2

    def trajectory(warm):
        com = coop.CooperativeCommunity(models, medium, biomass, dt=0.05, device=dev,
                                        maximum_coexistence_growth=cap, warm_start="extrapolate" if warm else False)
        warm_its = []
        for _ in range(args.warmup):
            r = com.step()
            warm_its.append(torch.stack([r.stages[k]["iterations"] for k in ("max_min", "parsimonious_exchange")]))
        torch.cuda.synchronize()
        ranks.barrier()
        stream = torch.cuda.current_stream()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        oks, iters = [], {"max_min": [], "parsimonious_exchange": []}
        start.record(stream)
        for _ in range(args.steps):
            r = com.step()
            oks.append(r.ok.sum())
            for k in iters:
                iters[k].append(r.stages[k]["iterations"])
        stop.record(stream)
        torch.cuda.synchronize()
        ranks.barrier()
        ms = ranks.max(start.elapsed_time(stop))
        ok_envs = int(sum(int(o.item()) for o in oks))
        its = {k: torch.cat(v).cpu().numpy() for k, v in iters.items()}
        first = warm_its[0].cpu().numpy() if warm_its else None
        return com, ms, ok_envs, its, first

    with ClockSampler(local) as clocks:
        com, ms_max, ok_envs, it, first_its = trajectory(True)
    st = com.solver.structure
    value = ranks.sum(ok_envs * stages) / (ms_max / 1e3)
    state = (com.biomass.cpu().numpy(), com.shared_medium().cpu().numpy(),
             com.live_bounds().cpu().numpy(), com.upper.cpu().numpy())
    res = com.step()
    torch.cuda.synchronize()
    com_c, ms_c, ok_c, it_c, _ = trajectory(False)
    cold = {"value": ranks.sum(ok_c * stages) / (ms_c / 1e3), "ms_per_step": ms_c / args.steps,
            "certified_fraction": ok_c / (args.envs * args.steps),
            "iterations": {k: {"mean": float(np.mean(v)), "p99": float(np.percentile(v, 99)), "max": int(np.max(v))}
                           for k, v in it_c.items()}}

    # roofline of the dominant kernel on one more cold step (the warm steps
    # may need no iteration at all): each stage's re-centred launch timed by
    # the engine's events
    peak, peak_kind = hbm_peak()
    res_c = com_c.step()
    torch.cuda.synchronize()
    kernel_ms, alg_bytes, inst_its = 0.0, 0.0, 0
    for key, eng, (m, n, nnz) in (("max_min", com_c.solver.engine1, (st.m1, st.n1, st.template1.nnz)),
                                  ("parsimonious_exchange", com_c.solver.engine3, (st.m3, st.n3, st.template3.nnz))):
        t32, _ = eng.phase_times()
        its = res_c.stages[key]["iterations"].cpu().numpy().astype(np.int64)
        kernel_ms += t32
        inst_its += int(its.sum())
        alg_bytes += float(its.sum()) * 4 * (3 * n + 3 * m + 2 * n) + float(its.max()) * 2 * (nnz * 8 + 4 * (m + 1))
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "peak_kind": f"{peak_kind} copy bandwidth", "kernel": "pdhg_recentred",
                "algorithmic_bytes": alg_bytes, "kernel_ms": kernel_ms, "instance_iterations": inst_its,
                "measured_on": "one cold step (both stages' launches)"}
    com_c.close()

    # CPU baseline: the exact-CPU cooperative solve on a sample of the same
    # state, and the GPU's stage-1 optima against it
    cpu = check = None
    if rank == 0:
        rate, cores, wall, sols = coop_cpu_sample(state, st.members, args.coop_sample, args.seed, cap)
        nu = res.coexistence.cpu().numpy()
        errs = [abs(nu[i] - sol.coexistence) / max(1.0, abs(sol.coexistence))
                for i, sol in sols.items() if sol.status == "optimal"]
        cpu = {"value": rate, "unit": "LPs/s", "cores": cores, "kind": "port",
               "sample": f"{len(sols)} environments of one step (seeded), the oracle's restatement of the "
                         f"reference's exact-CPU cooperative solve (scipy linprog 'highs', stages 1 and 3), one "
                         f"environment per thread; {wall:.1f} s wall"}
        check = {"sampled": len(sols), "max_rel_coexistence_err": max(errs) if errs else None}

    # e2e: the public solve with pinned host inputs of recorded steps and the
    # fluxes read back every step
    K = args.e2e_steps if args.e2e_steps > 0 else min(args.steps, 3)
    rec = []
    for _ in range(K + 1):
        rec.append(tuple(t.cpu().pin_memory() for t in (com.biomass, com.shared_medium(),
                                                        com.live_bounds())))
        com.step()
    # the upper bounds do not change between steps: bound once on the
    # device, as the FBA arm binds its upper bounds and objectives
    up_d = com.upper.cpu().pin_memory().to(dev)
    flux_h = torch.empty(args.envs, st.n_fluxes, dtype=torch.float64).pin_memory()
    ok_h = torch.empty(args.envs, dtype=torch.bool).pin_memory()
    solver = com.solver
    b0, m0, l0 = rec[0]
    solver.solve(b0, m0, 0.05, l0, up_d)
    torch.cuda.synchronize()
    ranks.barrier()
    t0 = time.perf_counter()
    e2e_ok = 0
    for b, mdm, lo in rec[1:]:
        r = solver.solve(b, mdm, 0.05, lo, up_d)
        flux_h.copy_(r.fluxes, non_blocking=True)
        ok_h.copy_(r.ok, non_blocking=True)
        torch.cuda.synchronize()
        e2e_ok += int(ok_h.sum())
    wall = time.perf_counter() - t0
    ranks.barrier()
    e2e = {"value": ranks.sum(e2e_ok * stages) / ranks.max(wall), "unit": "LPs/s",
           "h2d_bytes_per_step": int(8 * args.envs * (st.n_species + len(st.metabolites) + st.n_fluxes)),
           "d2h_bytes_per_step": int(args.envs * (8 * st.n_fluxes + 1)), "steps": K,
           "api": "CooperativeSolver.solve with pinned host biomass, shared-medium concentrations and live lower "
                  "bounds each step (upper bounds bound once); fluxes and status read back"}
    com.close()
    if rank == 0:
        line = {"metric": COOP_METRIC, "value": value, "unit": "LPs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
                "data": "synthetic (seeded generator; no public dataset)",
                "config": dict(coop_config(args, st, stages), parallelism=f"env-sharded x{world}",
                               growth_cap=cap if cap is not None else 10.0),
                "certified_fraction": ok_envs / (args.envs * args.steps),
                "env_steps_per_s": world * args.envs * args.steps / (ms_max / 1e3),
                "iterations": {k: {"mean": float(np.mean(v)), "p99": float(np.percentile(v, 99)),
                                   "max": int(np.max(v))} for k, v in it.items()},
                "first_step_mean_iterations": (None if first_its is None else
                                               {"max_min": float(first_its[0].mean()),
                                                "parsimonious_exchange": float(first_its[1].mean())}),
                "warm_start": "first-order extrapolation of the last two steps' stage solutions (reference "
                              "units), rescaled to the new biomass",
                "cold": cold, "warm_vs_cold": value / cold["value"] if cold["value"] else None,
                "roofline": roofline, "cpu_baseline": cpu, "highs_check": check, "e2e": e2e,
                "gpu_launches": stages * args.steps, "clocks": clocks.summary()}
        print(json.dumps(line), flush=True)
    ranks.close()


def run_reference_cooperative(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from co_cultivation_metabolic_atlas_b200 import cooperative as coop
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from oracle import dfba
    models = syn.community_models(seed=syn.COOPERATIVE_SEED)
    members = coop.synthetic_members(models)
    st = coop.CommunityStructure(members)
    medium, biomass = syn.initial_environments(args.envs, seed=args.seed)
    lower = np.concatenate([dfba.uptake_lower_bounds(m, medium, biomass, 0.05) for m in models], axis=1)
    upper = np.repeat(np.concatenate([m.upper for m in models])[None], args.envs, 0)
    shared = np.zeros((args.envs, len(st.metabolites)))
    for k, name in enumerate(st.metabolites):
        if int(name[1:4]) < coop.SECONDARY_OFFSET:
            shared[:, k] = medium[:, int(name[1:4])]
    state = (biomass, shared, lower, upper)
    cap = args.coop_growth_cap if args.coop_growth_cap > 0 else None
    rates, cores = [], None
    for k in range(args.warmup + args.steps):
        rate, cores, _, _ = coop_cpu_sample(state, members, args.coop_sample, args.seed + k, cap)
        if k >= args.warmup:
            rates.append(rate)
    value = statistics.mean(rates)
    line = {"impl": "reference", "metric": COOP_METRIC, "value": value, "unit": "LPs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * 2 * args.envs / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": coop_config(args, st, 2),
            "cpu_baseline": {"value": value, "unit": "LPs/s", "cores": cores, "kind": "port",
                             "sample": f"{args.coop_sample} environments per step of the initial state, the "
                                       f"exact-CPU cooperative solve (HiGHS), one environment per thread"},
            "e2e": {"value": value, "unit": "LPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- profiling driver
def run_profile(args):
    """Short untimed runs of one workload for an external profiler."""
    import torch

    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    from co_cultivation_metabolic_atlas_b200.engine import EngineOptions, SolveConfig

    models = syn.community_models()
    if args.profile == "mlp":
        from co_cultivation_metabolic_atlas_b200.train_warmstart import HIDDEN, N_FEATURES
        from co_cultivation_metabolic_atlas_b200.warmstart import BF16, MLP, solution_layout
        _, width = solution_layout(models)
        net = MLP([N_FEATURES, *HIDDEN, width], seed=0)
        g = torch.Generator(device="cuda").manual_seed(0)
        X = torch.randn(args.envs, N_FEATURES, device="cuda", generator=g)
        T = torch.randn(args.envs, net.pdims[-1], device="cuda", generator=g)
        # 2 B sum(in * out) per forward pass (padded widths: the FLOPs the
        # kernels issue); backward: dW for every layer, dH for all but the first
        mac = [net.pdims[l] * net.pdims[l + 1] for l in range(net.layers)]
        fwd = 2.0 * args.envs * sum(mac)
        train = fwd + 2.0 * args.envs * (sum(mac) + sum(mac[1:]))
        dY32 = torch.empty_like(T)
        dY16 = torch.empty(T.shape, dtype=BF16, device="cuda")
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        for k in range(args.steps):
            ev[0].record()
            net.forward(X)
            ev[1].record()
            Y = net.forward(X, keep=True)
            net.ops.mse_grad(Y, T, 2.0 / Y.numel(), dY32, dY16, loss)
            gW, gb = net.backward(dY32, dY16)
            net.adam_step(gW, gb, 1e-4)
            ev[2].record()
            torch.cuda.synchronize()
            if net.ops.error_flag():
                raise RuntimeError("tensor-core kernel reported a timeout")
            t_inf, t_train = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
            print(f"step {k}: inference {t_inf:.3f} ms ({fwd / t_inf / 1e9:.1f} TFLOP/s), "
                  f"training step {t_train:.3f} ms ({train / t_train / 1e9:.1f} TFLOP/s)")
        return
    if args.profile == "cooperative":
        from co_cultivation_metabolic_atlas_b200.cooperative import CooperativeCommunity
        models = syn.community_models(seed=syn.COOPERATIVE_SEED)
        medium, biomass = syn.initial_environments(args.envs)
        com = CooperativeCommunity(models, medium, biomass)
        for k in range(args.steps):
            last = k == args.steps - 1
            if last:
                torch.cuda.nvtx.range_push("coop_step")
            res = com.step()
            torch.cuda.synchronize()
            if last:
                torch.cuda.nvtx.range_pop()
            its = {name: float(v["iterations"].float().mean()) for name, v in res.stages.items()}
            print(f"step {k}: certified {int(res.ok.sum())}/{args.envs}, mean iterations {its}")
        com.close()
        return
    medium, biomass = syn.initial_environments(args.envs)
    com = DeviceCommunity(models, medium, biomass, config=SolveConfig(precision=args.precision),
                          options=EngineOptions(warps_per_block=args.warps), warm_start=args.warm)
    for k in range(args.steps):
        st = com.step()
        if args.precision == "mixed":
            phase = com.engine.phase_iterations()
            t32, t64 = com.engine.phase_times()
            print(f"step {k}: first-phase instance-iterations {int(phase.sum().item())}, "
                  f"first phase {t32:.3f} ms, FP64 phase {t64:.3f} ms")
    torch.cuda.synchronize()
    print("certified", int(st.certified.item()), "of", st.lps)
    com.close()


def spawn_ranks(n):
    """``--gpus N`` without a ``torchrun`` environment: run this command as
    N ranks under ``torch.distributed.run`` on this node and return its
    exit code (rank 0 prints the line)."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and not args.profile:
        sys.exit(spawn_ranks(args.gpus))
    if args.profile:
        run_profile(args)
    elif args.workload == "cooperative":
        (run_reference_cooperative if args.impl == "reference" else run_cooperative)(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
