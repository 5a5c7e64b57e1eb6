"""Parity with the oracle at the last-place level, on the benchmark's own
configurations: the plain reference case (100 x 100, NPCFree 10, box 4 x 4,
FP64) and the large single instance's grid (1000 x 1000) in FP64.

What is bit-exact and what is not:
  * integer results - particle counts, cell starts (hence every cell list),
    collision counts, impact counts, sample counts - are identical;
  * free flight, the box intersection, specular reflection, cold-start and
    inflow positions use IEEE arithmetic on the same draws: 0 ulp;
  * a value that passes through log, cos, sin, pow or hypot (diffuse and CLL
    velocities, Maxwellian and isotropic draws, post-collision velocities)
    can differ in its last bits: CUDA's double functions and the host libm
    are each within 1-2 ulp of the exact value.  Velocity components are
    held to VEL_ULP units in the last place of the particle's speed (a
    component near zero after a cancellation is compared on the scale of the
    speed it came from); positions, which add Dt * v to a coordinate, to
    POS_ULP units in the last place of the coordinate.
Each test prints its measured maxima and the histogram of the velocity
differences.
"""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import (FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, default_params,
                                  large_case)
from oracle.cpu import OracleEngine
from tests.helpers import ulp_distance

pytestmark = pytest.mark.gpu

VEL_ULP = 16
POS_ULP = 2
WALLS = {"specular": WALL_SPECULAR, "diffuse": WALL_DIFFUSE, "cll": WALL_CLL}


def speed_scaled_ulps(g: dict, o: dict) -> np.ndarray:
    """|v_gpu - v_oracle| per component in units of the last place of the
    oracle particle's largest velocity component."""
    s = np.maximum.reduce([np.abs(o["vx"]), np.abs(o["vy"]), np.abs(o["vz"])])
    sp = np.spacing(np.maximum(s, 1e-300))
    return np.stack([np.abs(g[k] - o[k]) / sp for k in ("vx", "vy", "vz")])


def compare_state(g: dict, o: dict, what: str) -> dict:
    assert len(g["x"]) == len(o["x"]), f"{what}: particle count"
    pos = {k: ulp_distance(g[k], o[k]) for k in ("x", "y")}
    vel_raw = {k: ulp_distance(g[k], o[k]) for k in ("vx", "vy", "vz")}
    vel = speed_scaled_ulps(g, o)
    rep = {"particles": len(g["x"]),
           "pos_ulp_max": int(max(v.max(initial=0) for v in pos.values())),
           "pos_differ": int(sum((v > 0).sum() for v in pos.values())),
           "vel_ulp_of_speed_max": float(vel.max(initial=0.0)),
           "vel_raw_ulp_max": int(max(v.max(initial=0) for v in vel_raw.values())),
           "vel_differ": int(sum((v > 0).sum() for v in vel_raw.values())),
           "vel_hist": {str(b): int(c) for b, c in zip(*np.unique(
               np.minimum(np.ceil(vel[vel > 0]), 64).astype(int), return_counts=True))}}
    print(what, rep)
    assert rep["pos_ulp_max"] <= POS_ULP, (what, rep)
    assert rep["vel_ulp_of_speed_max"] <= VEL_ULP, (what, rep)
    return rep


def compare_integers(ge: Engine, oe: OracleEngine, what: str):
    cg, co = ge.counters(), oe.counters()
    for k in ("np", "step", "sample_step", "collisions_last_step", "collisions_total",
              "drag_collision_count", "drag_collision_count_window", "particle_steps"):
        assert cg[k] == co[k], f"{what}: {k} {cg[k]} != {co[k]}"
    np.testing.assert_array_equal(ge.cell_starts(), oe.cell_starts(), err_msg=what)


@pytest.mark.parametrize("wall", ["specular", "diffuse", "cll"])
def test_move_stage_last_place(cuda, engine_lib, wall):
    """MoveParticles alone, from one shared FP64 state with an established
    flow around the box: every slot that does not hit the box is bit-exact
    (free flight), specular impacts are bit-exact, diffuse and CLL impacts
    are within the bounds."""
    p = default_params().copy(wall_model=WALLS[wall], seed=31, first_sampling_step=10**6)
    o = OracleEngine(p)
    assert o.init_cold() == 0
    assert o.step(150) == 0  # reflected particles around the box
    st = o.particles()
    g = Engine(p)
    g.set_particles(st)
    o2 = OracleEngine(p)
    assert o2.set_particles(st) == 0
    g.MoveParticles()
    assert o2.stage("move") == 0
    a, b = g.particles(), o2.particles()
    hit = (b["vx"] != st["vx"]) | (b["vy"] != st["vy"]) | (b["vz"] != st["vz"])
    assert hit.sum() > 20, "the state has impacts to check"
    free = ~hit
    for k in a:
        assert np.array_equal(a[k][free], b[k][free]), f"free flight {k} not bit-exact"
    if wall == "specular":
        for k in a:
            assert np.array_equal(a[k], b[k]), f"specular impact {k} not bit-exact"
    else:
        compare_state({k: v[hit] for k, v in a.items()}, {k: v[hit] for k, v in b.items()},
                      f"{wall} impacts")
    g.close()


def test_plain_reference_case_200_steps(cuda, engine_lib):
    """The plain reference case (100 x 100, NPCFree 10, box 4 x 4, Ma 4,
    specular, FP64), 200 steps with sampling from step 100: every integer
    result identical at every check, the state within the bounds, the
    sampled counts identical and the moment sums to the last bits."""
    p = default_params().copy(wall_model=WALL_SPECULAR, seed=2024, first_sampling_step=100,
                              n_step=4000)
    g = Engine(p)
    o = OracleEngine(p)
    g.InitialConditions()
    assert o.init_cold() == 0
    for s in range(4):
        g.step(50)
        assert o.step(50) == 0
        g.synchronize()
        what = f"plain case step {50 * (s + 1)}"
        compare_integers(g, o, what)
        compare_state(g.particles(), o.particles(), what)
    fg, fo = g.fields(), o.fields()
    np.testing.assert_array_equal(fg[:, 0], fo[:, 0])    # CountNP
    np.testing.assert_array_equal(fg[:, 16], fo[:, 16])  # CountNC
    scale = np.abs(fo).max(axis=0, keepdims=True) + 1e-300
    assert (np.abs(fg - fo) / scale).max() <= 1e-12
    g.close()


@pytest.mark.parametrize("wall", ["diffuse", "cll"])
def test_large_grid_fp64_steps(cuda, engine_lib, wall):
    """The large single instance's 1000 x 1000 grid in FP64 at NPCFree 1.5
    (about 1.5e6 particles, cell ids up to 1e6, hundreds of look-back tiles
    per scan), angle 10, its walls: 6 steps, integers identical and the state
    within the bounds after each."""
    p = large_case(wall_model=WALLS[wall], precision=FP64, seed=77).copy(
        npc_free=1.5, first_sampling_step=2)
    g = Engine(p)
    o = OracleEngine(p)
    g.InitialConditions()
    assert o.init_cold() == 0
    g.synchronize()
    compare_integers(g, o, f"{wall} 1000^2 cold start")
    st_g, st_o = g.particles(), o.particles()
    for k in ("x", "y"):
        assert np.array_equal(st_g[k], st_o[k]), "cold-start positions bit-exact"
    for s in range(6):
        g.step(1)
        assert o.step() == 0
        g.synchronize()
        what = f"{wall} 1000^2 step {s + 1}"
        compare_integers(g, o, what)
        compare_state(g.particles(), o.particles(), what)
    g.close()
