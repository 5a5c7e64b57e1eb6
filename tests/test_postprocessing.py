"""The reference's post-processing reads this engine's field files unchanged:
postprocessing/compare_runs.py (load_run, check_settings, extract_profile, as
its own tests/test_compare_runs.py exercises them) on fields written by
dsmc_write_field for two wall models of the same case.

The script is imported from the reference's source tree, so the test runs
where that tree is present and is skipped elsewhere; it needs no GPU (the
moments come from the oracle, which reproduces the engine's bit for bit).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

from dsmc_erlend_b200.abi import Derived, Params
from dsmc_erlend_b200.engine import write_field
from oracle.cpu import OracleEngine
from oracle.paths import REFERENCE_SOURCES

REFERENCE = REFERENCE_SOURCES / "postprocessing"
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def compare_runs():
    if not (REFERENCE / "compare_runs.py").exists():
        pytest.skip("the reference's post-processing scripts are not present")
    sys.path.insert(0, str(REFERENCE))
    import compare_runs as cr

    return cr


def _write(wall: str, out: Path):
    g = json.loads((GOLDEN / "reference_steps.json").read_text())
    case = g["cases"][wall]
    p, d = Params(), Derived()
    for k, v in case["params"].items():
        setattr(p, k, v)
    for k, v in case["derived"].items():
        setattr(d, k, v)
    o = OracleEngine(p, d)
    o.init_cold()
    o.step(8)
    cells = o.fields()
    write_field(p, d, o.counters()["sample_step"], cells, str(out))
    return p, d, cells, o.counters()["sample_step"]


def test_compare_runs_reads_engine_fields(engine_lib, compare_runs, tmp_path):
    runs = {}
    for wall in ("specular", "diffuse"):
        p, d, cells, ss = _write(wall, tmp_path)
        run = compare_runs.load_run(tmp_path / wall)
        runs[wall] = (run, p, d, cells, ss)
        data = run["data"]
        assert data.shape == (p.nx * p.ny, 8)
        # Column 2 is the number density W CountNP / SampleStep / DV of the
        # cell, x-major like the engine's fields.
        n = d.weight * cells[:, 0] / ss / d.dv
        assert np.allclose(data[:, 2], n, rtol=1e-9, atol=0)
        assert compare_runs.run_label(run) == wall.capitalize()
    compare_runs.check_settings(runs["specular"][0], runs["diffuse"][0])
    for axis, target in (("y", -5.0), ("x", 3.0)):
        coords, values, actual = compare_runs.extract_profile(runs["diffuse"][0], axis, target)
        assert len(coords) > 10 and np.isfinite(values["density"]).any()
        assert abs(actual - target) <= max(runs["diffuse"][1].x2 - runs["diffuse"][1].x1,
                                           runs["diffuse"][1].y2 - runs["diffuse"][1].y1)
