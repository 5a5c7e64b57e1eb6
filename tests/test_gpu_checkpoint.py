"""Checkpoint and restart (no counterpart in the reference, whose run cannot
resume): a run interrupted by dsmc_checkpoint_save and resumed in a fresh
context by dsmc_checkpoint_load continues bit-identically to the run that
was never interrupted: same particles in the same slots, same cell starts,
same moments and counters (the drag impulse sums to within rounding, their
atomic order being free).  Also the drag window counters against the oracle
and the --restart / --checkpoint / --print-period flags of the CLI."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import FP32, FP64, WALL_DIFFUSE
from dsmc_erlend_b200.ensemble import ensemble_cases
from helpers import small_case

pytestmark = pytest.mark.gpu

CLI = Path(__file__).resolve().parents[1] / "dsmc_erlend_b200" / "lib" / "dsmc"


def _state(e: Engine, i: int = 0):
    c = e.counters(i)
    imp = (c.pop("drag_impulse_total"), c.pop("drag_impulse_window"))
    return e.particles(i), e.cell_starts(i), e.fields(i), c, imp


def _assert_same(a, b, what):
    pa, sa, fa, ca, ia = a
    pb, sb, fb, cb, ib = b
    for k in pa:
        assert np.array_equal(pa[k], pb[k]), f"{what}: {k}"
    assert np.array_equal(sa, sb), f"{what}: cell starts"
    assert np.array_equal(fa, fb), f"{what}: moments"
    assert ca == cb, what
    for x, y in zip(ia, ib):
        assert abs(x - y) <= 1e-12 * max(1e-300, abs(y)), what


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_resume_is_bit_identical(cuda, engine_lib, tmp_path, precision):
    p = small_case(WALL_DIFFUSE, seed=31, precision=precision, first_sampling_step=5)
    whole = Engine(p)
    whole.InitialConditions()
    whole.step(24)
    want = _state(whole)
    whole.close()

    first = Engine(p)
    first.InitialConditions()
    first.step(11)
    ck = tmp_path / "run.ckpt"
    first.checkpoint_save(ck)
    first.close()
    second = Engine(p)
    second.checkpoint_load(ck)
    assert second.counters()["step"] == 11
    second.step(13)
    _assert_same(_state(second), want, "resumed")
    second.close()


def test_ensemble_resume(cuda, engine_lib, tmp_path):
    cases = ensemble_cases(n=5, seed=8, precision=FP32, grid_range=(24, 48))
    for p in cases:
        p.first_sampling_step = 2
    whole = Engine(cases)
    whole.InitialConditions()
    whole.step(9)
    want = [_state(whole, i) for i in range(len(cases))]
    whole.close()
    a = Engine(cases)
    a.InitialConditions()
    a.step(4)
    a.checkpoint_save(tmp_path / "ens.ckpt")
    a.close()
    b = Engine(cases)
    b.checkpoint_load(tmp_path / "ens.ckpt")
    b.step(5)
    for i in range(len(cases)):
        _assert_same(_state(b, i), want[i], f"case {i}")
    b.close()


def test_checkpoint_of_other_case_is_refused(cuda, engine_lib, tmp_path):
    p = small_case(seed=3)
    e = Engine(p)
    e.InitialConditions()
    e.step(2)
    e.checkpoint_save(tmp_path / "a.ckpt")
    e.close()
    other = Engine(small_case(seed=4))
    with pytest.raises(RuntimeError):
        other.checkpoint_load(tmp_path / "a.ckpt")
    (tmp_path / "junk.ckpt").write_bytes(b"not a checkpoint")
    with pytest.raises(RuntimeError):
        other.checkpoint_load(tmp_path / "junk.ckpt")
    other.close()


def test_drag_report_window(cuda, engine_lib):
    p = small_case(WALL_DIFFUSE, seed=5, first_sampling_step=6)
    e = Engine(p)
    e.InitialConditions()
    e.step(5)
    with pytest.raises(RuntimeError):  # no sampling time yet
        e.drag_report()
    e.step(20)
    r = e.drag_report()
    c = e.counters()
    assert r["box_collisions"] == c["drag_collision_count"] > r["box_collisions_window"] > 0
    assert r["sampling_time"] == pytest.approx(18 * p.dt, rel=1e-12)  # steps 7..24
    assert r["mean_force"] == pytest.approx(c["drag_impulse_window"] / r["sampling_time"])
    assert 0.0 < r["cd"] < r["cd_total"]
    e.close()


def test_cli_checkpoint_restart_and_print_period(cuda, engine_lib, tmp_path):
    common = ["--nx", "40", "--ny", "30", "--npc", "6", "--wall", "specular", "--dt", "4e-5",
              "--first-sampling-step", "10", "--seed", "77"]
    full = subprocess.run([str(CLI), *common, "--steps", "60", "--results",
                           str(tmp_path / "full"), "--print-period", "20", "--drag"],
                          capture_output=True, text=True, timeout=300)
    assert full.returncode == 0, full.stderr
    assert "Drag coefficient Cd" in full.stdout
    assert (tmp_path / "full" / "step_20" / "specular" / "DSMC2D_Field.plt").exists()
    assert (tmp_path / "full" / "step_40" / "specular" / "DSMC2D_Field.plt").exists()
    half = subprocess.run([str(CLI), *common, "--steps", "30", "--results",
                           str(tmp_path / "half"), "--checkpoint", str(tmp_path / "c.ckpt")],
                          capture_output=True, text=True, timeout=300)
    assert half.returncode == 0, half.stderr
    rest = subprocess.run([str(CLI), *common, "--steps", "60", "--results",
                           str(tmp_path / "rest"), "--restart", str(tmp_path / "c.ckpt")],
                          capture_output=True, text=True, timeout=300)
    assert rest.returncode == 0, rest.stderr
    a = (tmp_path / "full" / "specular" / "DSMC2D_Field.plt").read_bytes()
    b = (tmp_path / "rest" / "specular" / "DSMC2D_Field.plt").read_bytes()
    assert a == b
