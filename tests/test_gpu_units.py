"""The single-routine entry points of the C ABI against the oracle, and the
population edits behind the reference-named GenerateNewParticles and
RemoveParticlesInsideBox.

  dsmc_k_inject    GenerateNewParticles (src/Boundary.cpp:60-92)
  dsmc_k_collide   BinaryCollisionsInCell (src/Collision.cpp:21-44)
  dsmc_k_elastic   ElasticCollision (src/Collision.cpp:7-19)
  dsmc_append_particles_device, dsmc_remove_inside_box, dsmc_collide_list

Counts and positions drawn with IEEE arithmetic only are bit-exact; velocities
that pass through log/cos/sin/pow are held to TRANSCENDENTAL_ULP units in
the last place of the speeds they are made of (the larger of the value and
the case's thermal speed sqrt(k T / m); tests/helpers.ulp_of_scale).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine, setup
from dsmc_erlend_b200._lib import check, load
from dsmc_erlend_b200.abi import (RNG_USER, WALL_DIFFUSE, WALL_SPECULAR, default_params)
from oracle.cpu import OracleEngine
from tests.helpers import assert_ulp, assert_ulp_of_scale, small_case

pytestmark = pytest.mark.gpu

# CUDA's log, cos, sin and pow are within 1-2 ulp of the correctly rounded
# value, as is the host libm; a Maxwellian or isotropic draw passes through
# one or two of them and a product or sum, so the two sides agree to a few
# ulp of the speeds involved.  A particle that collides again carries its
# difference into the next collision, so the lists of many collisions get a
# wider bound.
TRANSCENDENTAL_ULP = 8
CHAINED_ULP = 32
K_B = 1.380662e-23


def thermal_speed(t: float, p=None) -> float:
    m = (p.molar_mass if p is not None else 0.040) / 6.022045e23
    return float(np.sqrt(K_B * t / m))

RECTS = [(-20.1, -20.0, -20.0, 20.0), (-3.0, 1.0, 2.5, 4.0), (-20.0, -20.0, 20.0, 20.0)]


def _dev(torch, a, dtype=None):
    return torch.tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype)


@pytest.mark.parametrize("rect", RECTS)
@pytest.mark.parametrize("n_gas,move", [(1e17, 1), (3e15, 0), (2e16, 1)])
def test_k_inject_matches_oracle(cuda, engine_lib, rect, n_gas, move):
    torch = cuda
    p = small_case(WALL_DIFFUSE, seed=77)
    d = setup(p)
    cap = 200000
    bufs = [torch.empty(cap, dtype=torch.float64, device="cuda") for _ in range(5)]
    o = OracleEngine(p)
    o.set_particles({k: np.zeros(0) for k in ("x", "y", "vx", "vy", "vz")}, raw=True)
    total = 0
    for e in (0, 5):
        n = C.c_int64()
        r = (C.c_double * 4)(*rect)
        check(load().dsmc_k_inject(C.byref(p), C.byref(d), r, C.c_double(n_gas),
                                   C.c_double(410.0), C.c_double(-120.0), C.c_double(350.0),
                                   move, RNG_USER, 9, e, cap, *[b.data_ptr() for b in bufs],
                                   C.byref(n), None), "dsmc_k_inject")
        torch.cuda.synchronize()
        before = o.np()
        assert o.generate(rect, n_gas, 410.0, -120.0, 350.0, move, RNG_USER, 9, e) == 0
        assert o.np() - before == n.value, "count draw"
        st = o.particles()
        got = [b[: n.value].cpu().numpy() for b in bufs]
        want = [st[k][before:] for k in ("x", "y", "vx", "vy", "vz")]
        # Positions: IEEE on the shared draws, bit-exact; a pre-move adds
        # Dt * v, whose difference of a few ulp is below an ulp of the
        # position or of the cell size (1 m here) for positions near zero.
        if not move:
            assert_ulp(got[0], want[0], 0, "x")
            assert_ulp(got[1], want[1], 0, "y")
        else:
            assert_ulp_of_scale(got[0], want[0], 1.0, 1, "x")
            assert_ulp_of_scale(got[1], want[1], 1.0, 1, "y")
        for k in range(2, 5):
            assert_ulp_of_scale(got[k], want[k], thermal_speed(350.0, p), TRANSCENDENTAL_ULP,
                                "v")
        total += n.value
    assert total > 0


def test_k_inject_capacity(cuda, engine_lib):
    p = small_case(WALL_DIFFUSE)
    d = setup(p)
    n = C.c_int64()
    r = (C.c_double * 4)(-20.0, -20.0, 20.0, 20.0)
    s = load().dsmc_k_inject(C.byref(p), C.byref(d), r, C.c_double(1e17), C.c_double(0.0),
                             C.c_double(0.0), C.c_double(200.0), 0, RNG_USER, 0, 0, 10, None, None,
                             None, None, None, C.byref(n), None)
    assert s == 31 and n.value > 10  # DSMC_ERR_CAPACITY, and the count


def _collide_setup(torch, seed=3):
    rng = np.random.default_rng(seed)
    n = 3000
    v = rng.normal(0, 450, (3, n))
    n_lists = 60
    sizes = rng.integers(0, 80, n_lists)
    perm = rng.permutation(n)[: sizes.sum()].astype(np.int32)
    start = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    return v, start, perm


@pytest.mark.parametrize("with_ipc", [True, False])
def test_k_collide_matches_oracle(cuda, engine_lib, with_ipc):
    torch = cuda
    p = small_case(WALL_SPECULAR, seed=13)
    d = setup(p)
    v, start, perm = _collide_setup(torch)
    vol = 3e-6  # small cells: many candidate pairs per list
    n_lists = len(start) - 1
    tv = [_dev(torch, v[k]) for k in range(3)]
    ts = _dev(torch, start, torch.int32)
    ti = _dev(torch, perm, torch.int32) if with_ipc else None
    ent = np.arange(n_lists, dtype=np.int64) * 3 + 1
    te = _dev(torch, ent, torch.int64).to(torch.int32)
    nc = torch.zeros(n_lists, dtype=torch.int32, device="cuda")
    check(load().dsmc_k_collide(C.byref(p), C.byref(d), C.c_double(vol), n_lists, ts.data_ptr(),
                                ti.data_ptr() if ti is not None else None,
                                *[t.data_ptr() for t in tv], RNG_USER, 4, te.data_ptr(),
                                nc.data_ptr(), None), "dsmc_k_collide")
    torch.cuda.synchronize()
    o = OracleEngine(p, d)
    o.set_particles({"x": np.zeros(v.shape[1]), "y": np.zeros(v.shape[1]), "vx": v[0],
                     "vy": v[1], "vz": v[2]}, raw=True)
    want_nc = []
    for l in range(n_lists):
        ids = perm[start[l]:start[l + 1]] if with_ipc else np.arange(start[l], start[l + 1])
        want_nc.append(o.collide_list(vol, ids, RNG_USER, 4, int(ent[l])))
    assert nc.cpu().numpy().tolist() == want_nc
    assert sum(want_nc) > 100
    st = o.particles()
    for k, key in enumerate(("vx", "vy", "vz")):
        assert_ulp_of_scale(tv[k].cpu().numpy(), st[key], 450.0, CHAINED_ULP, key)


def test_k_elastic_matches_oracle(cuda, engine_lib):
    torch = cuda
    rng = np.random.default_rng(4)
    n = 2000
    v1, v2 = rng.normal(0, 500, (n, 3)), rng.normal(0, 500, (n, 3))
    cr = np.linalg.norm(v2 - v1, axis=1)
    p = default_params()
    t1, t2, tc = _dev(torch, v1.ravel()), _dev(torch, v2.ravel()), _dev(torch, cr)
    check(load().dsmc_k_elastic(C.byref(p), n, t1.data_ptr(), t2.data_ptr(), tc.data_ptr(),
                                RNG_USER, 7, None, None), "dsmc_k_elastic")
    torch.cuda.synchronize()
    g1, g2 = t1.cpu().numpy().reshape(n, 3), t2.cpu().numpy().reshape(n, 3)
    o = OracleEngine(p)
    w1, w2 = np.empty_like(g1), np.empty_like(g2)
    for i in range(n):
        w1[i], w2[i] = o.elastic(v1[i], v2[i], cr[i], RNG_USER, 7, i)
    assert_ulp_of_scale(g1, w1, 500.0, TRANSCENDENTAL_ULP, "V1")
    assert_ulp_of_scale(g2, w2, 500.0, TRANSCENDENTAL_ULP, "V2")
    # Momentum and energy are conserved (to rounding).
    assert np.allclose(g1 + g2, v1 + v2, rtol=0, atol=1e-9)
    assert np.allclose((g1 ** 2 + g2 ** 2).sum(1), (v1 ** 2 + v2 ** 2).sum(1), rtol=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_append_particles_matches_oracle(cuda, engine_lib, precision):
    """Particles appended between steps: the ones outside the domain are
    removed in swap-with-last order and the population is re-sorted, exactly
    as the oracle's GenerateNewParticles + removal + Indexing order them."""
    from dsmc_erlend_b200.abi import FP32, FP64

    torch = cuda
    p = small_case(WALL_DIFFUSE, seed=91, precision=FP32 if precision == "fp32" else FP64)
    g = Engine(p)
    g.InitialConditions()
    g.step(3)
    g.synchronize()
    before = g.particles()
    rng = np.random.default_rng(1)
    m = 5000
    add = {"x": rng.uniform(-22, 22, m), "y": rng.uniform(-22, 22, m),
           "vx": rng.normal(0, 300, m), "vy": rng.normal(0, 300, m), "vz": rng.normal(0, 300, m)}
    if precision == "fp32":  # values the FP32 state holds exactly
        add = {k: v.astype(np.float32).astype(np.float64) for k, v in add.items()}
    t = {k: _dev(torch, v) for k, v in add.items()}
    check(load().dsmc_append_particles_device(g._h, 0, *[t[k].data_ptr() for k in
                                                         ("x", "y", "vx", "vy", "vz")], m),
          "dsmc_append_particles_device")
    o = OracleEngine(p)
    o.set_particles({k: np.concatenate([before[k], add[k]]) for k in add}, raw=True)
    o.remove_outside_domain()
    assert o.stage("index") == 0
    after, want = g.particles(), o.particles()
    assert len(after["x"]) == len(want["x"]) < len(before["x"]) + m
    for k in after:
        assert np.array_equal(after[k], want[k]), k
    np.testing.assert_array_equal(g.cell_starts(), o.cell_starts())
    # The run continues from the edited population.
    g.step(2)
    g.synchronize()
    assert g.counters()["step"] == 5
    g.close()


def test_remove_inside_box_matches_oracle(cuda, engine_lib):
    torch = cuda
    rng = np.random.default_rng(2)
    p = small_case(WALL_SPECULAR, seed=5, npc_free=40.0)  # slots for 20000 particles
    g = Engine(p)
    n = 20000
    st = {"x": rng.uniform(-8, 10, n), "y": rng.uniform(-6, 5, n), "vx": rng.normal(0, 300, n),
          "vy": rng.normal(0, 300, n), "vz": rng.normal(0, 300, n)}
    g.set_particles(st)
    o = OracleEngine(p)
    assert o.set_particles(st) == 0
    check(load().dsmc_remove_inside_box(g._h, 0), "dsmc_remove_inside_box")
    o.remove_inside_box()
    assert o.stage("index") == 0
    a, b = g.particles(), o.particles()
    assert 0 < len(a["x"]) < n and len(a["x"]) == len(b["x"])
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_collide_list_on_context_matches_oracle(cuda, engine_lib):
    p = small_case(WALL_SPECULAR, seed=8)
    g = Engine(p)
    g.InitialConditions()
    g.synchronize()
    st = g.particles()
    starts = g.cell_starts()
    o = OracleEngine(p)
    o.set_particles(st, raw=True)
    busiest = np.argsort(np.diff(starts))[-5:]
    for j, cell in enumerate(busiest):
        ipc = np.arange(starts[cell], starts[cell + 1], dtype=np.int32)[::-1].copy()
        nc = C.c_int32()
        check(load().dsmc_collide_list(g._h, 0, C.c_double(2e-6), len(ipc),
                                       ipc.ctypes.data_as(C.POINTER(C.c_int32)), RNG_USER, 11, j,
                                       C.byref(nc)), "dsmc_collide_list")
        assert nc.value == o.collide_list(2e-6, ipc, RNG_USER, 11, j)
    a, b = g.particles(), o.particles()
    for k in ("vx", "vy", "vz"):
        assert_ulp_of_scale(a[k], b[k], thermal_speed(p.t_free, p), CHAINED_ULP, k)
    for k in ("x", "y"):
        assert np.array_equal(a[k], b[k])
    bad = np.array([0, len(st["x"])], dtype=np.int32)
    assert load().dsmc_collide_list(g._h, 0, C.c_double(1.0), 2,
                                    bad.ctypes.data_as(C.POINTER(C.c_int32)), RNG_USER, 0, 0,
                                    C.byref(C.c_int32())) == 2  # DSMC_ERR_ARGUMENT: index out of range
    g.close()
