"""dsmc_get_fields_noalloc: the field read-out for callers that cannot
allocate device memory when they read results (an application whose device
memory is reserved by its own pool, a monitor that must not stall the device
the way cudaFree does).  It stages the moments in one static device array
instead of a temporary buffer.

Its output must equal dsmc_get_fields' (the allocating entry point) on two
calls in a row with different contents - the static array keeps the previous
call's data, so the second call shows that nothing stale leaks through - and
a case larger than the array must be refused without touching memory.  This
file is collected last so a run stopping at the first failure has run every
other test already.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import WALL_CLL, default_params

pytestmark = pytest.mark.gpu

MAX_CELLS = 65536  # DSMC_FIELDS_NOALLOC_MAX_CELLS
ERR_TOO_LARGE = 63


def _noalloc(lib, eng: Engine, case: int, ncell: int):
    out = np.full((ncell, 17), np.nan)
    status = lib.dsmc_get_fields_noalloc(eng._h, case, out.ctypes.data_as(C.c_void_p))
    return status, out


def test_noalloc_fields_equal_allocating_entry_point(cuda, engine_lib):
    # Two cases of different size in one context: the second call reads a
    # smaller field than the first, so stale staging data would show up.
    p0 = default_params().copy(nx=120, ny=90, npc_free=8.0, wall_model=WALL_CLL,
                               first_sampling_step=0, attack_angle=5.0, seed=71)
    p1 = p0.copy(nx=64, ny=40, seed=72, attack_angle=-12.0)
    eng = Engine([p0, p1])
    eng.InitialConditions()
    eng.step(15)
    eng.synchronize()
    for call, case in enumerate((0, 1)):
        if call:
            eng.step(7)  # new contents between the two calls
            eng.synchronize()
        p = eng.params[case]
        ncell = p.nx * p.ny
        want = eng.GatherGlobalField(case)
        status, got = _noalloc(engine_lib, eng, case, ncell)
        assert status == 0
        assert np.array_equal(got, want), f"call {call + 1}: fields differ"
        assert want[:, 0].sum() > 0  # the case sampled particles
    eng.close()


def test_noalloc_refuses_cases_above_the_static_maximum(cuda, engine_lib):
    p = default_params().copy(nx=300, ny=300, npc_free=1.0, seed=3)
    assert p.nx * p.ny > MAX_CELLS
    eng = Engine(p)
    eng.InitialConditions()
    status, out = _noalloc(engine_lib, eng, 0, p.nx * p.ny)
    assert status == ERR_TOO_LARGE
    assert np.isnan(out).all()  # the host buffer was not touched
    eng.close()
