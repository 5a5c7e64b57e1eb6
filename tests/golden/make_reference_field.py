"""Generates tests/golden/reference_case_field.npz: the sampled field of the
plain reference case (100x100 cells, NPCFree 10, specular walls, Dt 1e-5 s,
4000 steps sampled after step 2000) from the UNMODIFIED reference solver - its
own sources, its own multiply-with-carry RNG, its own time loop - built as
oracle/_ref/dsmc_ref_baseline by `make -C oracle ref`.

Independent seeds are run in parallel and their moments summed (replica
statistics), so the fixture's own sampling noise is small next to the 2%
field tolerance of the statistical test.

    python tests/golden/make_reference_field.py [--seeds 256]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
EXE = ROOT / "oracle" / "_ref" / "dsmc_ref_baseline"

K_B = 1.380662e-23
N_A = 6.022045e23


def fields_from_moments(m: np.ndarray, sample_step: int, weight: float, dv: float,
                        mass: float) -> dict:
    """Printing()'s derived quantities (src/Sampling.cpp:114-143)."""
    np_ = m[:, 0]
    n = weight * np_ / sample_step / dv
    with np.errstate(invalid="ignore", divide="ignore"):
        u = m[:, 1:4] / np_[:, None]
        vv = m[:, [4, 8, 12]] / np_[:, None]
        t = mass * (vv - u * u) / K_B
    u[np_ == 0] = 0
    t[np_ == 0] = 0
    return {"n": n, "ux": u[:, 0], "uy": u[:, 1], "tx": t[:, 0], "ty": t[:, 1],
            "t": t.mean(axis=1), "count": np_}


def run_one(seed: int) -> tuple[np.ndarray, int]:
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as tf:
        path = tf.name
    try:
        subprocess.run([str(EXE), "100", "100", "10", "0", "4000", "1", "0", "0", "0", "1e-5",
                        str(seed), "2000", path], check=True, capture_output=True)
        raw = np.fromfile(path, dtype=np.float64)
    finally:
        os.unlink(path)
    return raw[:-1].reshape(-1, 17), int(raw[-1])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=256)
    args = ap.parse_args()
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        results = list(ex.map(run_one, range(1, args.seeds + 1)))
    moments = sum(r[0] for r in results)
    sample_step = sum(r[1] for r in results)
    dx = 40.0 / 100
    dv = dx * dx * 0.1
    weight = dv * 1e17 / 10
    mass = 0.040 / N_A
    f = fields_from_moments(moments, sample_step, weight, dv, mass)
    np.savez_compressed(HERE / "reference_case_field.npz",
                        **{k: v.astype(np.float32) for k, v in f.items()},
                        seeds=np.arange(1, args.seeds + 1), sample_step=sample_step)
    print("wrote", HERE / "reference_case_field.npz", "samples", sample_step)


if __name__ == "__main__":
    main()
