"""Profiling driver: run a few warm-started dFBA steps of the synthetic
community so that an external profiler can capture the PDHG phase kernels.

    python -m co_cultivation_metabolic_atlas_b200.profile_step --envs 512 --steps 3
    python -m co_cultivation_metabolic_atlas_b200.profile_step --cooperative --envs 1024 --steps 4

``--cooperative`` steps the cooperative community LP instead (stage 1 and
stage 3 per step, certificate in the reference's units).

    python -m co_cultivation_metabolic_atlas_b200.profile_step --mlp --envs 4096 --steps 5

``--mlp`` runs the learned warm start's network instead (44 state features,
four GELU layers of 512, one output per flux and dual of the three species;
random-initialised weights): per step one inference pass and one training
step (forward, MSE gradient, backward, Adam) over ``--envs`` states, timed
with CUDA events and reported as tensor-core TFLOP/s of the GEMMs.
"""

from __future__ import annotations

import argparse

import torch

from . import synthetic as syn
from .dfba import DeviceCommunity
from .engine import EngineOptions, SolveConfig


def run_mlp(models, states, steps):
    from .train_warmstart import HIDDEN, N_FEATURES
    from .warmstart import BF16, MLP, solution_layout
    _, width = solution_layout(models)
    net = MLP([N_FEATURES, *HIDDEN, width], seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn(states, N_FEATURES, device="cuda", generator=g)
    T = torch.randn(states, net.pdims[-1], device="cuda", generator=g)
    # 2 B sum(in * out) per forward pass (padded widths: the FLOPs the
    # kernels issue); backward: dW for every layer, dH for all but the first
    mac = [net.pdims[l] * net.pdims[l + 1] for l in range(net.layers)]
    fwd = 2.0 * states * sum(mac)
    train = fwd + 2.0 * states * (sum(mac) + sum(mac[1:]))
    dY32 = torch.empty_like(T)
    dY16 = torch.empty(T.shape, dtype=BF16, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for k in range(steps):
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--envs", type=int, default=512)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--warps", type=int, default=16)
    ap.add_argument("--warm", default="extrapolate", choices=("cold", "previous", "extrapolate"))
    ap.add_argument("--cooperative", action="store_true")
    ap.add_argument("--mlp", action="store_true")
    args = ap.parse_args()
    models = syn.community_models()
    if args.mlp:
        run_mlp(models, args.envs, args.steps)
        return
    if args.cooperative:
        from .cooperative import CooperativeCommunity
        models = syn.community_models(seed=syn.COOPERATIVE_SEED)
        medium, biomass = syn.initial_environments(args.envs)
        com = CooperativeCommunity(models, medium, biomass)
        for k in range(args.steps):
            # the last step is marked for profilers (NVTX range "coop_step")
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


if __name__ == "__main__":
    main()
