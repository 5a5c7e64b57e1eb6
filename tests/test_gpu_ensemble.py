"""The batched ensemble: cases of uneven grid, particle count and wall model
advanced together in one context (one CUDA graph per step) give, case by
case, bit-identical results to the same case run alone (each case owns its
Philox key and its slot and cell ranges)."""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import FP32, FP64
from dsmc_erlend_b200.ensemble import ensemble_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_ensemble_cases_equal_single_runs(cuda, engine_lib, precision):
    cases = ensemble_cases(n=12, seed=99, precision=precision, grid_range=(24, 72))
    for p in cases:
        p.first_sampling_step = 3
    steps = 12
    ens = Engine(cases)
    ens.InitialConditions()
    ens.step(steps)
    ens.synchronize()
    for i, p in enumerate(cases):
        solo = Engine(p)
        solo.InitialConditions()
        solo.step(steps)
        solo.synchronize()
        a, b = ens.particles(i), solo.particles()
        for k in a:
            assert np.array_equal(a[k], b[k]), f"case {i}: {k}"
        assert np.array_equal(ens.cell_starts(i), solo.cell_starts())
        assert np.array_equal(ens.fields(i), solo.fields())
        ca, cb = ens.counters(i), solo.counters()
        for k in ("drag_impulse_total", "drag_impulse_window"):  # atomic sum order
            x, y = ca.pop(k), cb.pop(k)
            assert abs(x - y) <= 1e-12 * max(abs(y), 1e-300), (i, k)
        assert ca == cb, i
        solo.close()
    ens.close()


def test_ensemble_generator_ranges():
    cases = ensemble_cases(n=256, seed=2024)
    sides = np.array([p.nx for p in cases])
    assert sides.min() >= 64 and sides.max() <= 400 and all(p.nx == p.ny for p in cases)
    ang = np.array([p.attack_angle for p in cases])
    assert ang.min() >= -30 and ang.max() <= 30
    ma = np.array([p.ma_free for p in cases])
    assert ma.min() >= 2 and ma.max() <= 8
    n = np.array([p.n_free for p in cases])
    assert n.min() >= 1e16 and n.max() <= 1e18
    box = np.array([p.box_width for p in cases])
    assert box.min() >= 2 and box.max() <= 6
    npc = np.array([p.npc_free for p in cases])
    assert npc.min() >= 5 and npc.max() <= 20
    walls = {p.wall_model for p in cases}
    assert walls == {0, 1, 2}
    assert len({p.seed for p in cases}) == 256


def test_autotuned_launch_shapes_keep_results(cuda, engine_lib):
    """The autotuner changes grid shapes only: a run with the tuned shapes is
    bit-identical to a run with the default ones."""
    cases = ensemble_cases(n=6, seed=31, precision=FP32, grid_range=(32, 96))
    tuned = Engine(cases)
    tuned.InitialConditions()
    shapes = tuned.autotune(steps_per_trial=2)
    assert shapes and all(1 <= v <= mx for v, mx in shapes.values())
    tuned.InitialConditions()
    tuned.step(15)
    plain = Engine(cases)
    plain.set_launch_config({k: 1 for k in shapes})  # the smallest grids
    small = plain.launch_config()
    assert all(v == 1 for v, _ in small.values())
    plain.InitialConditions()
    plain.step(15)
    for i in range(len(cases)):
        a, b = tuned.particles(i), plain.particles(i)
        for k in a:
            assert np.array_equal(a[k], b[k]), (i, k)
        assert np.array_equal(tuned.fields(i), plain.fields(i))
    tuned.close()
    plain.close()
