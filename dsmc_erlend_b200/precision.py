"""What FP32 particle state costs in accuracy: the large single instance run
with FP32 positions and velocities (hit times, inflow counts, cell indices
and moment accumulators in FP64) against the same case run all in FP64.

    python -m dsmc_erlend_b200.precision [--steps 20000] [--sample-from 10000]
        [--walls diffuse cll] [--grid 1000]

For every wall model it runs three cases of identical parameters: FP64 with
key A, FP32 with key A and FP64 with key B.  DSMC is a Monte Carlo method:
the FP32 and FP64 runs share their random streams but part ways at the first
rounding that changes a cell index or a collision decision, after which they
are independent samples of the same flow.  So the FP32 error is reported
next to the FP64 run-to-run difference (key A against key B), the noise
floor of the comparison.  Each line gives the relative L2 error of n, ux,
uy and T outside the wall cells (dsmc_erlend_b200.fields.field_errors, the
fields Printing derives: src/Sampling.cpp:114-143).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import Engine
from .abi import FP32, FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, large_case
from .fields import field_errors, macroscopic

WALLS = {"diffuse": WALL_DIFFUSE, "cll": WALL_CLL, "specular": WALL_SPECULAR}


def run_field(p, stream=None) -> tuple[dict, float]:
    """Runs case p for p.n_step steps from the cold start; its macroscopic
    field and the device-synchronised wall time."""
    t = time.perf_counter()
    eng = Engine(p, stream=stream)
    eng.InitialConditions()
    eng.step(int(p.n_step))
    eng.synchronize()
    secs = time.perf_counter() - t
    d = eng.derived[0]
    f = macroscopic(eng.fields(), d.weight, d.dv, d.molecule_mass,
                    eng.counters()["sample_step"])
    eng.close()
    return f, secs


def compare(p, key_a: int = 1, key_b: int = 2) -> dict:
    """FP32 (key A) and FP64 (key B) against FP64 (key A): per-field
    relative L2 errors outside the wall cells."""
    f64a, s64 = run_field(p.copy(precision=FP64, seed=key_a))
    f32a, s32 = run_field(p.copy(precision=FP32, seed=key_a))
    f64b, _ = run_field(p.copy(precision=FP64, seed=key_b))
    from . import setup

    u = setup(p).u_free
    return {"fp32_vs_fp64": field_errors(f32a, f64a, p, u),
            "fp64_vs_fp64_other_key": field_errors(f64b, f64a, p, u),
            "seconds": {"fp64": s64, "fp32": s32}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--sample-from", type=int, default=10000)
    ap.add_argument("--walls", nargs="+", default=["diffuse", "cll"])
    ap.add_argument("--grid", type=int, default=1000)
    args = ap.parse_args()
    for w in args.walls:
        p = large_case(wall_model=WALLS[w])
        p.nx = p.ny = args.grid
        p.n_step = args.steps
        p.first_sampling_step = args.sample_from
        r = compare(p)
        r.update({"wall": w, "grid": args.grid, "steps": args.steps,
                  "sample_from": args.sample_from,
                  "case": "1000x1000 (or --grid), NPCFree 20, angle 10, Dt 1e-6, "
                          "diffuse Tw 300 K or CLL (0.8, 0.8)"})
        print(json.dumps({k: (v if not isinstance(v, dict) else
                              {kk: float(np.round(vv, 6)) for kk, vv in v.items()})
                          for k, v in r.items()}), flush=True)


if __name__ == "__main__":
    main()
