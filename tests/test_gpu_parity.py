"""Parity of the sm_100a kernels with the CPU oracle (the restatement of the
reference routines, oracle/dsmc_oracle.c) on the same seeded inputs.

Integer results (impact flags, counts, cell starts, removal order, collision
counts) must be identical; FP64 values agree to the last bits of CUDA's
log/cos/sin/pow/hypot against the host libm (tolerances in helpers.py);
specular impacts and free flight use only IEEE arithmetic and are bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine, setup
from dsmc_erlend_b200.abi import (RNG_MOVE, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR,
                                  default_params)
from oracle.cpu import OracleEngine
from tests.helpers import WALLS, assert_close, assert_state_close, small_case

pytestmark = pytest.mark.gpu

# Known answers of the reference tests (tests/GeometryTests.cpp:48-70):
# (x, y, dx, dy, tHit, nx, ny) for impacts, None for misses, box 6x6 at 0.
INTERSECT_6X6 = [
    (-4, 0, 2, 0, (0.5, -1, 0)),
    (4, 0, -2, 0, (0.5, 1, 0)),
    (0, -4, 0, 2, (0.5, 0, -1)),
    (0, 4, 0, -2, (0.5, 0, 1)),
    (-10, 0, 20, 0, (0.35, -1, 0)),
    (-4, 0, 1, 0, (1.0, -1, 0)),
    (-3, 0, 1, 0, (0.0, -1, 0)),
    (-4, -4, 2, 2, (0.5, -1, 0)),
    (-4, 2, 4, -1, (0.25, -1, 0)),
    (-4, 0, -1, 0, None),
    (-3, 0, -1, 0, None),
    (-4, 3, 8, 0, None),
    (-4, 2, 2, 2, None),
    (4, 4, 0, 0, None),
    (-4, 0, 0.5, 0, None),
]
# Translated rectangle (GeometryTests.cpp:64-69): box 4x2 at (2, -1).
INTERSECT_4X2 = [(-1, -1, 2, 0, (0.5, -1, 0)), (2, 1, 0, -2, (0.5, 0, 1))]


def _intersect_gpu(torch, p, rows):
    dev = "cuda"
    cols = [torch.tensor([float(r[i]) for r in rows], dtype=torch.float64, device=dev)
            for i in range(4)]
    n = len(rows)
    hit = torch.zeros(n, dtype=torch.int32, device=dev)
    t, nx, ny = (torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(3))
    from dsmc_erlend_b200._lib import check, load
    import ctypes as C

    check(load().dsmc_k_intersect(C.byref(p), n, *[c.data_ptr() for c in cols], hit.data_ptr(),
                                  t.data_ptr(), nx.data_ptr(), ny.data_ptr(), None))
    torch.cuda.synchronize()
    return hit.cpu().numpy(), t.cpu().numpy(), nx.cpu().numpy(), ny.cpu().numpy()


def test_intersect_known_answers(cuda, engine_lib):
    for (bx, by, bw, bh), table in (((0, 0, 6, 6), INTERSECT_6X6), ((2, -1, 4, 2), INTERSECT_4X2)):
        p = default_params().copy(box_x=bx, box_y=by, box_width=bw, box_height=bh)
        hit, t, nx, ny = _intersect_gpu(cuda, p, table)
        for i, row in enumerate(table):
            exp = row[4]
            if exp is None:
                assert hit[i] == 0, f"row {row}: unexpected impact"
            else:
                assert hit[i] == 1, f"row {row}: expected impact"
                assert abs(t[i] - exp[0]) < 1e-12
                assert nx[i] == exp[1] and ny[i] == exp[2]


def test_intersect_matches_oracle_random(cuda, engine_lib):
    rng = np.random.default_rng(3)
    p = default_params().copy(box_x=0.3, box_y=-0.2, box_width=3.7, box_height=2.9)
    o = OracleEngine(p)
    n = 20000
    rows = np.column_stack([rng.uniform(-4, 4, n), rng.uniform(-4, 4, n),
                            rng.normal(0, 2, n), rng.normal(0, 2, n)])
    rows[::7, 2] = 0.0  # axis-parallel segments
    rows[::11, 3] = 0.0
    hit, t, nx, ny = _intersect_gpu(cuda, p, rows.tolist())
    for i in range(n):
        h, tt, a, b = o.intersect(*rows[i])
        assert bool(hit[i]) == h
        if h:
            assert t[i] == tt and nx[i] == a and ny[i] == b  # IEEE only: bit-exact


@pytest.mark.parametrize("wall", ["specular", "diffuse", "cll"])
def test_wall_scatter_matches_oracle(cuda, engine_lib, wall):
    import ctypes as C
    from dsmc_erlend_b200._lib import check, load

    rng = np.random.default_rng(11)
    p = default_params().copy(wall_model=WALLS[wall], cll_normal=0.3, cll_tangential=0.7)
    d = setup(p)
    o = OracleEngine(p, d)
    n = 4096
    v = rng.normal(0, 500, (n, 3))
    normals = np.array([(-1, 0), (1, 0), (0, -1), (0, 1)], dtype=np.float64)[rng.integers(0, 4, n)]
    v[:, 0] = np.where(normals[:, 0] != 0, -normals[:, 0] * np.abs(v[:, 0]), v[:, 0])
    v[:, 1] = np.where(normals[:, 1] != 0, -normals[:, 1] * np.abs(v[:, 1]), v[:, 1])
    ent = np.arange(n, dtype=np.uint32) * 7 + 3
    tv = cuda.tensor(v.ravel(), device="cuda")
    tnx = cuda.tensor(normals[:, 0].copy(), device="cuda")
    tny = cuda.tensor(normals[:, 1].copy(), device="cuda")
    te = cuda.tensor(ent.astype(np.int64), device="cuda").to(cuda.int32)
    check(load().dsmc_k_scatter(C.byref(p), C.byref(d), n, tv.data_ptr(), tnx.data_ptr(),
                                tny.data_ptr(), RNG_MOVE, 5, te.data_ptr(), None))
    cuda.cuda.synchronize()
    got = tv.cpu().numpy().reshape(n, 3)
    want = np.empty_like(got)
    for i in range(n):
        s, w = o.scatter(v[i], normals[i, 0], normals[i, 1], RNG_MOVE, 5, int(ent[i]))
        assert s == 0
        want[i] = w
    if wall == "specular":
        assert np.array_equal(got, want)
    else:
        assert_close(got, want, 1e-13, 1e-10, f"{wall} scatter")
    # Outgoing velocity always points away from the face (Boundary.cpp:280).
    assert np.all(got[:, 0] * normals[:, 0] + got[:, 1] * normals[:, 1] >= 0)


def _pair(p, **kw):
    """The engine and the oracle, each with the constants of its own Setup
    (both restate the reference's, Gamma included, bit for bit)."""
    g = Engine(p)
    o = OracleEngine(p)
    assert g.derived[0].as_dict() == OracleEngine.setup(p)[1].as_dict()
    return g, o


def _compare(g: Engine, o: OracleEngine, what: str, fields: bool = True):
    cg, co = g.counters(), o.counters()
    for k in ("np", "step", "sample_step", "collisions_last_step", "drag_collision_count",
              "drag_collision_count_window", "particle_steps"):
        assert cg[k] == co[k], f"{what}: {k} {cg[k]} != {co[k]}"
    for k in ("drag_impulse_total", "drag_impulse_window"):  # atomic sums: order differs
        assert abs(cg[k] - co[k]) <= 1e-9 * max(1e-30, abs(co[k])), f"{what}: {k}"
    np.testing.assert_array_equal(g.cell_starts(), o.cell_starts(), err_msg=what)
    assert_state_close(g.particles(), o.particles(), what)
    if fields:
        assert_close(g.fields(), o.fields(), 1e-11, 1e-6, f"{what} fields")


def test_cold_start_matches_oracle(cuda, engine_lib):
    p = small_case(WALL_CLL, seed=21)
    g, o = _pair(p)
    g.InitialConditions()
    assert o.init_cold() == 0
    g.synchronize()
    _compare(g, o, "after InitialConditions")
    # Positions come from IEEE arithmetic on the shared draws: bit-exact.
    pg, po = g.particles(), o.particles()
    assert np.array_equal(pg["x"], po["x"]) and np.array_equal(pg["y"], po["y"])


@pytest.mark.parametrize("wall", ["specular", "diffuse", "cll"])
def test_steps_match_oracle(cuda, engine_lib, wall):
    p = small_case(WALLS[wall], seed=100 + WALLS[wall])
    g, o = _pair(p)
    g.InitialConditions()
    assert o.init_cold() == 0
    for s in range(12):
        g.step(1)
        assert o.step() == 0
        g.synchronize()
        _compare(g, o, f"{wall} step {s + 1}")


def test_stages_match_oracle(cuda, engine_lib):
    """Each stage function against the oracle's, including the removal order
    of BoundaryConditions (swap-with-last) before the sort."""
    p = small_case(WALL_DIFFUSE, seed=5)
    g, o = _pair(p)
    g.InitialConditions()
    o.init_cold()
    for s in range(4):
        g.MoveParticles()
        assert o.stage("move") == 0
        assert_state_close(g.particles(), o.particles(), f"step {s} after MoveParticles")
        g.BoundaryConditions()
        assert o.stage("boundary") == 0
        pg, po = g.particles(), o.particles()
        assert len(pg["x"]) == len(po["x"])
        assert_state_close(pg, po, f"step {s} after BoundaryConditions")
        g.Indexing()
        assert o.stage("index") == 0
        np.testing.assert_array_equal(g.cell_starts(), o.cell_starts())
        assert_state_close(g.particles(), o.particles(), f"step {s} after Indexing")
        g.CollideParticles()
        assert o.stage("collide") == 0
        g.Sampling()
        assert o.stage("sample") == 0
        g.end_step()
        assert o.stage("end_step") == 0
        g.synchronize()
        _compare(g, o, f"stage-wise step {s}")


def test_upload_sorts_like_indexing(cuda, engine_lib):
    """A random, unsorted population is put in cell order exactly as
    Indexing's lists order it (stable in particle order)."""
    rng = np.random.default_rng(8)
    p = small_case(WALL_SPECULAR, seed=1)
    g, o = _pair(p)
    n = 5000
    st = {"x": rng.uniform(-19.9, 19.9, n), "y": rng.uniform(-19.9, 19.9, n),
          "vx": rng.normal(0, 300, n), "vy": rng.normal(0, 300, n), "vz": rng.normal(0, 300, n)}
    # Duplicate cells heavily so the stable order matters.
    st["x"][::3] = st["x"][1::3][: len(st["x"][::3])]
    g.set_particles(st)
    assert o.set_particles(st) == 0
    np.testing.assert_array_equal(g.cell_starts(), o.cell_starts())
    pg, po = g.particles(), o.particles()
    for k in pg:
        assert np.array_equal(pg[k], po[k]), k


@pytest.mark.parametrize("wall", ["diffuse", "cll"])
def test_fp32_state_keeps_the_sort_invariant(cuda, engine_lib, wall):
    """FP32 storage: after the cold start and after every step the particles
    lie in their cells' slot ranges (cells recomputed on the host from the
    stored FP32 positions with the reference's Indexing arithmetic), none is
    inside the box, and none outside the domain."""
    from dsmc_erlend_b200.abi import FP32

    p = small_case(WALLS[wall], seed=61, precision=FP32, nx=64, ny=48, npc_free=12.0)
    d = setup(p)
    g = Engine(p)
    g.InitialConditions()
    for s in range(25):
        if s:
            g.step(1)
        g.synchronize()
        st = g.particles()
        starts = g.cell_starts()
        k = np.floor((st["x"] - p.x1) / d.dx).astype(np.int64)
        l = np.floor((st["y"] - p.y1) / d.dy).astype(np.int64)
        assert k.min() >= 0 and k.max() < p.nx and l.min() >= 0 and l.max() < p.ny
        cells = k * p.ny + l
        assert np.all(np.diff(cells) >= 0), f"step {s}: not in cell order"
        np.testing.assert_array_equal(np.searchsorted(cells, np.arange(p.nx * p.ny + 1)),
                                      starts)
        inside = (np.abs(st["x"] - p.box_x) < p.box_width / 2) & \
                 (np.abs(st["y"] - p.box_y) < p.box_height / 2)
        assert not inside.any(), f"step {s}: {inside.sum()} particles inside the box"


def test_upload_then_steps_match(cuda, engine_lib):
    """From one shared state, full steps agree (in-range fast path and the
    out-of-range lists both exercised)."""
    p = small_case(WALL_SPECULAR, seed=44)
    g, o = _pair(p)
    o.init_cold()
    st = o.particles()
    g.set_particles(st)
    o.set_particles(st)
    g.synchronize()
    _compare(g, o, "after upload", fields=False)
    for s in range(6):
        g.step(1)
        o.step()
        g.synchronize()
        _compare(g, o, f"uploaded step {s + 1}", fields=False)


def test_field_readback_paths_agree(cuda, engine_lib):
    """The field read-back gives the same bits whatever the destination: a
    fresh array, a caller's pageable buffer (staged through pinned chunks when
    larger than one), a caller's pinned buffer, and the device-side gather."""
    import torch

    p = small_case(WALL_DIFFUSE, seed=5, nx=300, ny=300, npc_free=2.0, first_sampling_step=0)
    g = Engine(p)
    g.InitialConditions()
    g.step(3)
    fresh = g.GatherGlobalField()
    assert fresh.nbytes > 8 << 20  # more than one staging chunk
    pageable = np.full_like(fresh, np.nan)
    assert g.GatherGlobalField(out=pageable) is pageable
    pinned = torch.empty(fresh.shape, dtype=torch.float64, pin_memory=True)
    g.GatherGlobalField(out=pinned.numpy())
    dev = torch.empty(fresh.shape, dtype=torch.float64, device="cuda")
    g.fields_to_device(0, dev.data_ptr())
    g.synchronize()
    for other in (pageable, pinned.numpy(), dev.cpu().numpy()):
        assert np.array_equal(fresh.view(np.uint64), other.view(np.uint64))
    assert np.isfinite(fresh).any() and (fresh[:, 0] > 0).any()
    with pytest.raises(ValueError):
        g.GatherGlobalField(out=np.empty((10, 17)))
    g.close()


def test_step_read_records_every_step(cuda, engine_lib):
    """dsmc_step_read's records equal dsmc_get_counters read after each step
    (the FP64 drag sums to rounding: their atomic additions have no fixed
    order)."""
    import ctypes as C

    import torch

    from dsmc_erlend_b200.abi import Counters

    cases = [small_case(WALL_DIFFUSE, seed=31), small_case(WALL_SPECULAR, seed=32)]
    n_steps = 6
    a = Engine(cases)
    b = Engine(cases)
    a.InitialConditions()
    b.InitialConditions()
    ring = torch.zeros(n_steps * len(cases) * C.sizeof(Counters), dtype=torch.uint8,
                       pin_memory=True)
    a.step_read(n_steps, ring.data_ptr())
    a.synchronize()
    recs = (Counters * (n_steps * len(cases))).from_address(ring.data_ptr())
    for k in range(n_steps):
        b.step(1)
        b.synchronize()
        for i in range(len(cases)):
            want = b.counters(i)
            got = recs[k * len(cases) + i].as_dict()
            for key, v in want.items():
                if isinstance(v, float):
                    assert got[key] == pytest.approx(v, rel=1e-12, abs=1e-300), (k, i, key)
                else:
                    assert got[key] == v, (k, i, key)
    assert recs[-1].step == n_steps and recs[-1].particle_steps > 0
    a.close()
    b.close()
