"""Throughput of the batched ensemble: the 256 cases of ensemble_cases() (grid
side U[64, 400], Ma U[2, 8], ...) advanced together in one context, either
one CUDA graph per step or (--persistent) one persistent cooperative kernel
for all timed steps; particle-steps/s summed over the cases, CUDA events on
the context's stream.

    python -m dsmc_erlend_b200.ensemble_bench [--cases 256] [--steps 200]
        [--warmup 20] [--autotune] [--precision fp32|fp64] [--persistent]
        [--ctas-per-sm N]

Prints one JSON line.  The full protocol is 5000 steps per case; the timed
window here is a bounded slice of it after the cold start and warm-up.
"""
from __future__ import annotations

import argparse
import json
import time

from . import Engine
from .abi import FP32, FP64
from .ensemble import ensemble_cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--persistent", action="store_true")
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    args = ap.parse_args()

    import torch

    prec = FP32 if args.precision == "fp32" else FP64
    cases = ensemble_cases(args.cases, args.seed, precision=prec)
    for p in cases:
        p.first_sampling_step = 0  # every timed step samples
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        t0 = time.perf_counter()
        eng = Engine(cases, stream=stream.cuda_stream)
        eng.InitialConditions()
        eng.synchronize()
        init_s = time.perf_counter() - t0
        shapes = None
        if args.autotune:
            shapes = eng.autotune(steps_per_trial=2)
            eng.InitialConditions()
        if args.persistent:
            eng.set_step_mode(True, args.ctas_per_sm)
        mode = eng.step_mode()
        eng.step(args.warmup)
        eng.synchronize()
        before = sum(eng.counters(i)["particle_steps"] for i in range(len(cases)))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        status = eng.synchronize()
        ms = e0.elapsed_time(e1)
        after = sum(eng.counters(i)["particle_steps"] for i in range(len(cases)))
        eng.close()
    ps = after - before
    print(json.dumps({
        "metric": "particle-steps/s on 1 B200 (batched ensemble)",
        "value": ps / (ms / 1e3), "unit": "particle-steps/s", "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "particles_mean": ps / args.steps, "cases": len(cases), "status": status,
        "config": {"workload": f"{len(cases)} cases of ensemble_cases(seed={args.seed}): "
                               "grid side U[64,400], Ma U[2,8], angle U[-30,30], "
                               "n log-U[1e16,1e18], box U[2,6], walls S/D/CLL, NPCFree U[5,20]",
                   "precision": args.precision, "sampling": "every timed step"},
        "launch": ("persistent" if mode["persistent"] else "graph per step"),
        "step_mode": mode, "cold_start_s": init_s, "launch_shapes": shapes}))


if __name__ == "__main__":
    main()
