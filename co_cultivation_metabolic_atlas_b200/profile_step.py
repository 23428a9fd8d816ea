"""Profiling driver: run a few warm-started dFBA steps of the synthetic
community so that an external profiler can capture the PDHG phase kernels.

    python -m co_cultivation_metabolic_atlas_b200.profile_step --envs 512 --steps 3
    python -m co_cultivation_metabolic_atlas_b200.profile_step --cooperative --envs 1024 --steps 4

``--cooperative`` steps the cooperative community LP instead (stage 1 and
stage 3 per step, certificate in the reference's units).
"""

from __future__ import annotations

import argparse

import torch

from . import synthetic as syn
from .dfba import DeviceCommunity
from .engine import EngineOptions, SolveConfig


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--envs", type=int, default=512)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--warps", type=int, default=16)
    ap.add_argument("--warm", default="extrapolate", choices=("cold", "previous", "extrapolate"))
    ap.add_argument("--cooperative", action="store_true")
    args = ap.parse_args()
    models = syn.community_models()
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
