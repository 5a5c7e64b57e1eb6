"""Pins the CPU oracle (oracle/dsmc_oracle.c) to the reference solver:

  * the known answers of the reference's own tests (tests/GeometryTests.cpp,
    tests/CLLTests.cpp), restated;
  * golden digests of full seeded steps produced by the reference's routines
    (tests/golden/reference_steps.json, made by make_golden.py);
  * the reference's routines themselves when oracle/_ref is built.
"""
from __future__ import annotations

import hashlib
import json
import math
from pathlib import Path

import numpy as np
import pytest

from dsmc_erlend_b200.abi import (RNG_MOVE, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, Derived,
                                  Params, default_params)
from oracle.cpu import OracleEngine, RefEngine, ref_available
from tests.helpers import small_case

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_steps.json"
K_B = 1.380662e-23


def _params(d: dict) -> Params:
    p = Params()
    for k, v in d.items():
        setattr(p, k, v)
    return p


def _derived(d: dict) -> Derived:
    x = Derived()
    for k, v in d.items():
        setattr(x, k, v)
    return x


# -- known answers of tests/GeometryTests.cpp ----------------------------------

def test_inside_box():
    o = OracleEngine(default_params().copy(box_width=6.0, box_height=6.0))
    assert o.inside_box(0.0, 0.0)
    assert o.inside_box(2.9, -2.9)
    assert not o.inside_box(3.0, 0.0)  # the surface is not interior
    assert not o.inside_box(0.0, 3.1)


@pytest.mark.parametrize("row", [
    (-4, 0, 2, 0, 0.5, -1, 0), (4, 0, -2, 0, 0.5, 1, 0), (0, -4, 0, 2, 0.5, 0, -1),
    (0, 4, 0, -2, 0.5, 0, 1), (-10, 0, 20, 0, 0.35, -1, 0), (-4, 0, 1, 0, 1.0, -1, 0),
    (-3, 0, 1, 0, 0.0, -1, 0), (-4, -4, 2, 2, 0.5, -1, 0), (-4, 2, 4, -1, 0.25, -1, 0),
    (-4, 0, -1, 0, None), (-3, 0, -1, 0, None), (-4, 3, 8, 0, None), (-4, 2, 2, 2, None),
    (4, 4, 0, 0, None), (-4, 0, 0.5, 0, None),
])
def test_intersect_known_answers(row):
    o = OracleEngine(default_params().copy(box_width=6.0, box_height=6.0))
    hit, t, nx, ny = o.intersect(*row[:4])
    if row[4] is None:
        assert not hit
    else:
        assert hit and abs(t - row[4]) < 1e-12 and nx == row[5] and ny == row[6]


def test_intersect_translated_rectangle():
    o = OracleEngine(default_params().copy(box_x=2.0, box_y=-1.0, box_width=4.0,
                                           box_height=2.0))
    assert o.intersect(-1, -1, 2, 0)[:4] == (True, 0.5, -1.0, 0.0)
    assert o.intersect(2, 1, 0, -2)[:4] == (True, 0.5, 0.0, 1.0)
    assert o.inside_box(3.9, -1.9)


def test_flow_angle_convention():
    s, d = OracleEngine.setup(default_params().copy(attack_angle=90.0))
    assert s == 0 and abs(d.ux_free) < 1e-10 and abs(d.uy_free + d.u_free) < 1e-10
    s, d = OracleEngine.setup(default_params().copy(attack_angle=-45.0))
    assert d.ux_free > 0 and d.uy_free > 0


def test_remove_particles_inside_box_order():
    # GeometryTests.cpp:82-87: of (0,0), (4,0), (2,2) only (4,0) survives.
    p = default_params().copy(box_width=6.0, box_height=6.0, nx=10, ny=10)
    o = OracleEngine(p)
    st = {"x": np.array([0.0, 4.0, 2.0]), "y": np.array([0.0, 0.0, 2.0]),
          "vx": np.zeros(3), "vy": np.zeros(3), "vz": np.zeros(3)}
    o.set_particles(st, raw=True)
    assert o._status("remove_inside_box") == 0
    out = o.particles()
    assert len(out["x"]) == 1 and out["x"][0] == 4.0


def test_specular_invariants():
    o = OracleEngine(default_params().copy(wall_model=WALL_SPECULAR))
    dg = math.sqrt(0.5)
    v = np.array([-3.0, -4.0, 5.0])
    vn, vt = (v[0] + v[1]) * dg, (-v[0] + v[1]) * dg
    s, w = o.scatter(v, dg, dg, RNG_MOVE, 0, 0)
    assert s == 0
    assert abs((w[0] + w[1]) * dg + vn) < 1e-12
    assert abs((-w[0] + w[1]) * dg - vt) < 1e-12
    assert w[2] == 5 and abs(w @ w - 50) < 1e-12


def test_specular_move_known_answer():
    # GeometryTests.cpp:104-117
    p = default_params().copy(wall_model=WALL_SPECULAR, box_width=6.0, box_height=6.0,
                              dt=0.002, nx=10, ny=10)
    o = OracleEngine(p)
    o.set_particles({"x": [-4.0], "y": [0.0], "vx": [1000.0], "vy": [100.0], "vz": [50.0]},
                    raw=True)
    assert o.stage("move") == 0
    st, c = o.particles(), o.counters()
    assert (st["vx"][0], st["vy"][0], st["vz"][0]) == (-1000.0, 100.0, 50.0)
    assert abs(st["x"][0] + 4) < 2e-12 and abs(st["y"][0] - 0.2) < 1e-12
    assert c["drag_collision_count"] == 1
    _, d = OracleEngine.setup(p)
    assert abs(c["drag_impulse_total"] / (d.weight * d.molecule_mass) - 2000) < 1e-10


def test_free_flight_known_answer():
    # GeometryTests.cpp:144-150
    p = default_params().copy(wall_model=WALL_DIFFUSE, box_width=6.0, box_height=6.0,
                              dt=0.002, nx=10, ny=10)
    o = OracleEngine(p)
    o.set_particles({"x": [-10.0], "y": [10.0], "vx": [1000.0], "vy": [0.0], "vz": [0.0]},
                    raw=True)
    o.stage("move")
    st = o.particles()
    assert st["x"][0] == -8 and st["y"][0] == 10 and st["vx"][0] == 1000
    assert o.counters()["drag_collision_count"] == 0


@pytest.mark.parametrize("wall", [WALL_DIFFUSE, WALL_CLL])
def test_reflections_leave_the_box(wall):
    # GeometryTests.cpp:119-143 and CLLTests.cpp:256-285
    p = default_params().copy(wall_model=wall, box_width=6.0, box_height=6.0, dt=0.002,
                              cll_normal=0.3, cll_tangential=0.7, nx=10, ny=10)
    o = OracleEngine(p)
    approaches = [((-4, 0), (1000, 100, 50)), ((4, 0), (-1000, 100, 50)),
                  ((0, -4), (100, 1000, 50)), ((0, 4), (100, -1000, 50)),
                  ((-4, -4), (1000, 1000, 50))]
    for (x, y), v in approaches:
        for sample in range(100):
            o.set_step(sample)
            o.set_particles({"x": [x], "y": [y], "vx": [v[0]], "vy": [v[1]], "vz": [v[2]]},
                            raw=True)
            hit, t, nx, ny = o.intersect(x, y, 0.002 * v[0], 0.002 * v[1])
            assert hit
            before = o.counters()["drag_collision_count"]
            assert o.stage("move") == 0
            st = o.particles()
            assert o.counters()["drag_collision_count"] == before + 1
            assert not o.inside_box(st["x"][0], st["y"][0])
            assert st["vx"][0] * nx + st["vy"][0] * ny > 0
            assert math.isfinite(st["x"][0]) and math.isfinite(st["y"][0])


# -- known answers of tests/CLLTests.cpp -----------------------------------------

def test_cll_zero_accommodation_is_specular():
    dg = math.sqrt(0.5)
    pspec = default_params().copy(wall_model=WALL_SPECULAR)
    pcll = default_params().copy(wall_model=WALL_CLL, cll_normal=0.0, cll_tangential=0.0)
    _, want = OracleEngine(pspec).scatter([-3, -4, 5], dg, dg, RNG_MOVE, 0, 0)
    _, got = OracleEngine(pcll).scatter([-3, -4, 5], dg, dg, RNG_MOVE, 0, 0)
    assert np.array_equal(got, want)


def _cll_moments(an, at, samples=100000):
    # Incident (-2, 3, 1.5) in a frame rotated by 45 degrees, kT/m = 1.
    n = math.sqrt(0.5)
    mass = K_B * 300.0
    p = default_params().copy(wall_model=WALL_CLL, cll_normal=an, cll_tangential=at,
                              molar_mass=mass * 6.022045e23, t_wall=300.0)
    o = OracleEngine(p)
    normal2 = np.empty(samples)
    tangent = np.empty(samples)
    z = np.empty(samples)
    for i in range(samples):
        s, v = o.scatter([-5 * n, n, 1.5], n, n, RNG_MOVE, 0, i)
        assert s == 0
        nn = (v[0] + v[1]) * n
        assert nn > 0 and math.isfinite(nn)
        normal2[i] = nn * nn
        tangent[i] = (-v[0] + v[1]) * n
        z[i] = v[2]
    return normal2, tangent, z


@pytest.mark.parametrize("an,at", [(1, 1), (0.3, 0.7), (0, 0.6), (0.6, 0)])
def test_cll_conditional_moments(an, at):
    samples = 20000
    normal2, tangent, z = _cll_moments(an, at, samples)
    mean2 = (1 - an) * 4 + 2 * an
    var2 = 4 * an * (1 - an) * 4 + 4 * an * an
    tmean = math.sqrt(1 - at) * 3
    zmean = math.sqrt(1 - at) * 1.5
    tol = 6 * math.sqrt(at / samples) + 1e-10
    assert abs(normal2.mean() - mean2) < 6 * math.sqrt(var2 / samples) + 1e-10
    assert abs(tangent.mean() - tmean) < tol
    assert abs(z.mean() - zmean) < tol
    t2tol = 6 * math.sqrt((2 * at * at + 4 * tmean * tmean * at) / samples) + 1e-10
    z2tol = 6 * math.sqrt((2 * at * at + 4 * zmean * zmean * at) / samples) + 1e-10
    assert abs((tangent ** 2).mean() - tmean * tmean - at) < t2tol
    assert abs((z ** 2).mean() - zmean * zmean - at) < z2tol


@pytest.mark.parametrize("bad", [-0.1, 1.1, float("nan")])
@pytest.mark.parametrize("which", ["normal", "tangential"])
def test_cll_rejects_bad_coefficients(bad, which):
    kw = {"cll_normal": 0.8, "cll_tangential": 0.8, f"cll_{which}": bad}
    s, _ = OracleEngine.setup(default_params().copy(wall_model=WALL_CLL, **kw))
    assert s == 40


# -- golden digests of the reference's own steps ----------------------------------

def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


@pytest.mark.parametrize("wall", ["specular", "diffuse", "cll"])
def test_oracle_reproduces_reference_steps(wall):
    g = json.loads(GOLDEN.read_text())
    case = g["cases"][wall]
    p, d = _params(case["params"]), _derived(case["derived"])
    o = OracleEngine(p, d)
    assert o.init_cold() == 0
    step = 0
    for snap in g["snapshots"]:
        while step < snap:
            assert o.step() == 0
            step += 1
        want = case["snapshots"][str(snap)]
        c = o.counters()
        for k, v in want["counters"].items():
            assert c[k] == v, f"{wall} step {snap}: {k}"
        assert hashlib.sha256(o.cell_starts().astype(np.int32).tobytes()).hexdigest() == \
            want["cell_starts_digest"]
        st = o.particles()
        for k, dg in want["state_digest"].items():
            assert _digest(st[k]) == dg, f"{wall} step {snap}: {k} differs from the reference"
        assert _digest(o.fields()) == want["fields_digest"]


# -- the reference's routines, live --------------------------------------------------

@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("wall", [WALL_SPECULAR, WALL_DIFFUSE, WALL_CLL])
def test_oracle_matches_reference_routines(wall):
    p = small_case(wall, seed=300 + wall, attack_angle=-7.0)
    ref = RefEngine(p)
    d = ref.derived()
    o = OracleEngine(p, d)
    assert ref.init_cold() == 0 and o.init_cold() == 0
    for s in range(15):
        assert ref.step() == 0 and o.step() == 0
        pr, po = ref.particles(), o.particles()
        for k in pr:
            assert np.array_equal(pr[k], po[k]), f"step {s}: {k}"
    assert np.array_equal(ref.fields(), o.fields())
    cr, co = ref.counters(), o.counters()
    for k in ("drag_collision_count_window", "drag_impulse_window"):  # not in the reference
        cr.pop(k), co.pop(k)
    assert cr == co


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")
def test_gaussian_draw_order_of_reference_compiler():
    """frand_Gaussian (src/Boundary.cpp:49-50) has two unsequenced draws; the
    reference build takes the logarithm's draw first, as the oracle does."""
    import ctypes as C

    L = RefEngine.lib()
    L.dsmc_ref_configure(C.byref(default_params()))
    L.dsmc_ref_select_stream(7, 1, 2)
    g = L.dsmc_ref_gaussian(0.0, 1.0)
    L.dsmc_ref_select_stream(7, 1, 2)
    u1, u2 = L.dsmc_ref_brng(), L.dsmc_ref_brng()
    assert g == math.sqrt(-2.0 * 1.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


# -- single routines of the reference headers, live ----------------------------

@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("n_gas,move", [(1e17, 1), (3e15, 0), (2e18, 1)])
def test_generate_matches_reference(n_gas, move):
    """GenerateNewParticles(X1, Y1, X2, Y2, Ngas, Ugasx, Ugasy, Tgas, MoveFlag)
    (src/Boundary.cpp:60-92) with non-freestream gas: same count, same bits."""
    p = small_case(WALL_DIFFUSE, seed=41)
    ref = RefEngine(p)
    o = OracleEngine(p, ref.derived())
    ref.set_particles({k: np.zeros(0) for k in ("x", "y", "vx", "vy", "vz")}, raw=True)
    o.set_particles({k: np.zeros(0) for k in ("x", "y", "vx", "vy", "vz")}, raw=True)
    rect = (-3.0, 1.0, 2.5, 4.0)
    for e in range(3):
        assert ref.generate(rect, n_gas, 410.0, -120.0, 350.0, move, 2, 9, e) == 0
        assert o.generate(rect, n_gas, 410.0, -120.0, 350.0, move, 2, 9, e) == 0
    pr, po = ref.particles(), o.particles()
    assert len(pr["x"]) == len(po["x"]) > 0
    for k in pr:
        assert np.array_equal(pr[k], po[k]), k


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")
def test_collide_list_and_elastic_match_reference():
    """BinaryCollisionsInCell(CellVolume, NPC, IPC) and ElasticCollision
    (src/Collision.cpp:7-44) over arbitrary index lists: same pairs, bits."""
    rng = np.random.default_rng(5)
    p = small_case(WALL_SPECULAR, seed=2)
    ref = RefEngine(p)
    o = OracleEngine(p, ref.derived())
    n = 400
    st = {"x": rng.uniform(-10, 10, n), "y": rng.uniform(-10, 10, n),
          "vx": rng.normal(0, 400, n), "vy": rng.normal(0, 400, n), "vz": rng.normal(0, 400, n)}
    ref.set_particles(st, raw=True)
    o.set_particles(st, raw=True)
    total = 0
    for e in range(40):
        ipc = rng.permutation(n)[: rng.integers(2, 60)]
        vol = 10 ** rng.uniform(-7, -3)  # small volumes: many candidate pairs
        a = ref.collide_list(vol, ipc, 3, 17, e)
        b = o.collide_list(vol, ipc, 3, 17, e)
        assert a == b
        total += a
    assert total > 50
    pr, po = ref.particles(), o.particles()
    for k in pr:
        assert np.array_equal(pr[k], po[k]), k
    v1, v2 = rng.normal(0, 500, 3), rng.normal(0, 500, 3)
    for e in range(20):
        ra = ref.elastic(v1, v2, 731.5 + e, 5, 1, e)
        oa = o.elastic(v1, v2, 731.5 + e, 5, 1, e)
        assert np.array_equal(ra[0], oa[0]) and np.array_equal(ra[1], oa[1])


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")
def test_remove_inside_box_matches_reference():
    """RemoveParticlesInsideBox (src/Geometry.cpp:231-247): swap-with-last order."""
    rng = np.random.default_rng(9)
    p = small_case(WALL_SPECULAR, seed=2)
    ref = RefEngine(p)
    o = OracleEngine(p, ref.derived())
    n = 3000
    st = {"x": rng.uniform(-6, 8, n), "y": rng.uniform(-4, 3, n),
          "vx": rng.normal(0, 400, n), "vy": rng.normal(0, 400, n), "vz": rng.normal(0, 400, n)}
    ref.set_particles(st, raw=True)
    o.set_particles(st, raw=True)
    ref.remove_inside_box()
    o.remove_inside_box()
    pr, po = ref.particles(), o.particles()
    assert 0 < len(pr["x"]) < n
    for k in pr:
        assert np.array_equal(pr[k], po[k]), k
