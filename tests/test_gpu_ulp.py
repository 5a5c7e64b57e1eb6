"""Parity with the oracle at the last-place level, on the benchmark's own
configurations: the plain reference case (100 x 100, NPCFree 10, box 4 x 4,
FP64) and the large single instance's grid (1000 x 1000) in FP64.

What is bit-exact and what is not:
  * integer results - particle counts, cell starts (hence every cell list),
    collision counts, impact counts, sample counts - are identical;
  * free flight, the box intersection, specular reflection and cold-start
    positions use IEEE arithmetic on the same draws: 0 ulp;
  * a value that passes through log, cos, sin, pow or hypot (diffuse and CLL
    velocities, Maxwellian and isotropic draws, post-collision velocities)
    can differ in its last bits: CUDA's double functions and the host libm
    are each within 1-2 ulp of the exact value.  Such a difference is
    measured in units in the last place of the magnitude it was computed
    from (tests/helpers.ulp_of_scale): for a velocity component the larger
    of the component and the case's thermal speed sqrt(k T / m) (a component
    near zero is a sum that cancelled).  A particle whose velocity differs in
    its last bits rounds x + Dt v differently by up to one ulp of x in each
    step, so its position drifts by at most one ulp of the domain's extent
    (max |X1|, |X2|, |Y1|, |Y2|) per step: positions are held to POS_ULP
    ulp of the extent per step run.  Bounds: VEL_ULP, POS_ULP.
Each test prints its measured maxima, how many values differ at all, and
the histogram of the velocity differences.
"""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import (FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, default_params,
                                  large_case)
from oracle.cpu import OracleEngine
from tests.helpers import ulp_distance, ulp_of_scale

pytestmark = pytest.mark.gpu

VEL_ULP = 8
POS_ULP = 1  # per step
WALLS = {"specular": WALL_SPECULAR, "diffuse": WALL_DIFFUSE, "cll": WALL_CLL}
K_B = 1.380662e-23


def thermal_speed(p) -> float:
    return float(np.sqrt(K_B * p.t_free / (p.molar_mass / 6.022045e23)))


def compare_state(g: dict, o: dict, p, what: str, steps: int = 1) -> dict:
    assert len(g["x"]) == len(o["x"]), f"{what}: particle count"
    c = thermal_speed(p)
    extent = max(abs(p.x1), abs(p.x2), abs(p.y1), abs(p.y2))
    pos = np.stack([ulp_of_scale(g[k], o[k], extent) for k in ("x", "y")])
    vel = np.stack([ulp_of_scale(g[k], o[k], c) for k in ("vx", "vy", "vz")])
    raw = np.stack([ulp_distance(g[k], o[k]) for k in ("x", "y", "vx", "vy", "vz")])
    rep = {"particles": len(g["x"]),
           "pos_ulp_max": float(pos.max(initial=0.0)),
           "vel_ulp_max": float(vel.max(initial=0.0)),
           "values_differing": int((raw > 0).sum()), "values": int(raw.size),
           "raw_ulp_max": int(raw.max(initial=0)),
           "vel_hist": {str(b): int(n) for b, n in zip(*np.unique(
               np.minimum(np.ceil(vel[vel > 0]), 64).astype(int), return_counts=True))}}
    print(what, rep)
    assert rep["pos_ulp_max"] <= POS_ULP * max(steps, 1), (what, rep)
    assert rep["vel_ulp_max"] <= VEL_ULP, (what, rep)
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
    # Ten times the reference's Dt and four times its particles: about a
    # hundred impacts in one move.
    p = default_params().copy(wall_model=WALLS[wall], seed=31, first_sampling_step=10**6,
                              dt=1e-4, npc_free=40.0)
    o = OracleEngine(p)
    assert o.init_cold() == 0
    assert o.step(60) == 0  # reflected particles around the box
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
        compare_state({k: v[hit] for k, v in a.items()}, {k: v[hit] for k, v in b.items()}, p,
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
        compare_state(g.particles(), o.particles(), p, what, steps=50 * (s + 1))
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
        compare_state(g.particles(), o.particles(), p, what, steps=s + 1)
    g.close()
