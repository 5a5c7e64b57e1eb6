"""Generates the golden fixtures of tests/golden/ from the reference solver's
own routines (oracle/_ref/libdsmc_ref.so, compiled from the reference sources
by `make -C oracle ref`).

    python tests/golden/make_golden.py

Per wall model, a small seeded case is run for 8 time steps under the
engine's stream contract; the fixture keeps, at several points, the particle
count, counters, cell starts and SHA-256 digests of the bit patterns of every
state array and of the 17 moments per cell.  A restatement that reproduces the
digests reproduces the reference's arithmetic bit for bit.  The reference's
Printing() output for the final field is kept verbatim (DSMC2D_Field.*).
"""
from __future__ import annotations

import hashlib
import json
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from dsmc_erlend_b200.abi import WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR  # noqa: E402
from oracle.cpu import RefEngine  # noqa: E402
from tests.helpers import small_case  # noqa: E402

SNAPSHOTS = (0, 1, 3, 8)
WALLS = {"specular": WALL_SPECULAR, "diffuse": WALL_DIFFUSE, "cll": WALL_CLL}


def golden_case(wall: int):
    return small_case(wall, seed=900 + wall, nx=20, ny=16, npc_free=6.0, first_sampling_step=1)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def snapshot(eng) -> dict:
    st = eng.particles()
    return {
        "counters": eng.counters(),
        "cell_starts_digest": hashlib.sha256(eng.cell_starts().astype(np.int32).tobytes()).hexdigest(),
        "state_digest": {k: digest(v) for k, v in st.items()},
        "fields_digest": digest(eng.fields()),
        "first": {k: float(v[0]) if len(v) else None for k, v in st.items()},
    }


def main():
    out = {"snapshots": list(SNAPSHOTS), "cases": {}}
    for name, wall in WALLS.items():
        p = golden_case(wall)
        ref = RefEngine(p)
        d = ref.derived()
        assert ref.init_cold() == 0
        snaps = {0: snapshot(ref)}
        for s in range(1, max(SNAPSHOTS) + 1):
            assert ref.step() == 0
            if s in SNAPSHOTS:
                snaps[s] = snapshot(ref)
        out["cases"][name] = {"params": p.as_dict(), "derived": d.as_dict(),
                              "snapshots": {str(k): v for k, v in snaps.items()}}
        with tempfile.TemporaryDirectory() as tmp:
            ref.write_field(tmp)
            for f in ("DSMC2D_Field.plt", "DSMC2D_Field.json"):
                shutil.copy(Path(tmp) / name / f, HERE / f"printing_{name}_{f}")
    (HERE / "reference_steps.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "reference_steps.json")


if __name__ == "__main__":
    main()
