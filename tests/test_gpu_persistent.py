"""The persistent step: ONE cooperative kernel for all steps of a dsmc_step
call (dsmc_set_step_mode(DSMC_STEP_PERSISTENT)) gives, case by case, the
same particles, cell lists, counters and moments as the step graph, for an
ensemble of uneven grids, particle counts and wall models, whatever the grid
size of the persistent launch and however the steps are split into calls.
Its grid-barrier waits are bounded: a barrier that cannot complete returns
DSMC_ERR_TIMEOUT and the context stays usable."""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import ERR_TIMEOUT, FP32, FP64
from dsmc_erlend_b200.ensemble import ensemble_cases

pytestmark = pytest.mark.gpu


def assert_same(a: Engine, b: Engine, what: str):
    for i in range(a.n_cases):
        pa, pb = a.particles(i), b.particles(i)
        for k in pa:
            assert np.array_equal(pa[k], pb[k]), f"{what} case {i}: {k}"
        assert np.array_equal(a.cell_starts(i), b.cell_starts(i)), f"{what} case {i}"
        assert np.array_equal(a.fields(i), b.fields(i)), f"{what} case {i}: moments"
        ca, cb = a.counters(i), b.counters(i)
        for k in ("drag_impulse_total", "drag_impulse_window"):  # atomic sum order
            x, y = ca.pop(k), cb.pop(k)
            assert abs(x - y) <= 1e-12 * max(abs(y), 1e-300), (what, i, k)
        assert ca == cb, (what, i)


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_persistent_steps_equal_graph_steps(cuda, engine_lib, precision):
    cases = ensemble_cases(n=10, seed=7, precision=precision, grid_range=(24, 96))
    for p in cases:
        p.first_sampling_step = 4
    graph = Engine(cases)
    pers = Engine(cases)
    pers.set_step_mode(True)
    mode = pers.step_mode()
    print("persistent launch:", mode)
    assert mode["persistent"] and 1 <= mode["ctas_per_sm"] == mode["max_ctas_per_sm"]
    graph.InitialConditions()
    pers.InitialConditions()
    # Calls of odd and even lengths: the buffer side alternates inside a launch.
    for n in (1, 6, 3, 14):
        graph.step(n)
        pers.step(n)
        graph.synchronize()
        pers.synchronize()
        assert_same(pers, graph, f"after {n}")
    graph.close()
    pers.close()


def test_persistent_grid_size_does_not_change_results(cuda, engine_lib):
    cases = ensemble_cases(n=5, seed=3, precision=FP32, grid_range=(32, 80))
    for p in cases:
        p.first_sampling_step = 2
    runs = []
    for ctas in (0, 1):
        e = Engine(cases)
        e.set_step_mode(True, ctas)
        if ctas:
            assert e.step_mode()["ctas_per_sm"] == ctas
        e.InitialConditions()
        e.step(12)
        e.synchronize()
        runs.append(e)
    assert_same(runs[0], runs[1], "grid")
    for e in runs:
        e.close()


def test_mode_switch_mid_run(cuda, engine_lib):
    """Graph steps, then persistent steps, then graph steps again continue
    one run: the same as graph steps throughout."""
    cases = ensemble_cases(n=4, seed=11, precision=FP64, grid_range=(24, 64))
    for p in cases:
        p.first_sampling_step = 3
    ref = Engine(cases)
    ref.InitialConditions()
    ref.step(15)
    mix = Engine(cases)
    mix.InitialConditions()
    mix.step(5)
    mix.set_step_mode(True)
    mix.step(5)
    mix.set_step_mode(False)
    mix.step(5)
    ref.synchronize()
    mix.synchronize()
    assert_same(mix, ref, "mixed")
    ref.close()
    mix.close()


def test_grid_barrier_wait_is_bounded(cuda, engine_lib):
    """A barrier that one more CTA would have to reach gives up after its
    bound (20 ms here) and reports DSMC_ERR_TIMEOUT; the context then steps
    normally."""
    cases = ensemble_cases(n=2, seed=5, precision=FP32, grid_range=(24, 40))
    e = Engine(cases)
    assert e.grid_sync_probe(20_000_000) == ERR_TIMEOUT
    e.set_step_mode(True)
    e.InitialConditions()
    e.step(3)
    e.synchronize()
    assert all(e.counters(i)["step"] == 3 for i in range(2))
    e.close()
