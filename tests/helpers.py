"""Shared case definitions and comparison helpers of the tests."""
from __future__ import annotations

import numpy as np

from dsmc_erlend_b200.abi import (WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, Params, default_params)

WALLS = {"specular": WALL_SPECULAR, "diffuse": WALL_DIFFUSE, "cll": WALL_CLL}


def small_case(wall: int = WALL_CLL, seed: int = 7, **kw) -> Params:
    """A 40x30 grid with an off-centre 6x3 m box, 8 particles per cell,
    a 12 degree flow and sampling from step 2: every stage is exercised
    (impacts, inflow, removal, cell changes, collisions, sampling) in a few
    thousand particles."""
    base = dict(nx=40, ny=30, npc_free=8.0, wall_model=wall, attack_angle=12.0,
                first_sampling_step=2, box_width=6.0, box_height=3.0, box_x=1.0, box_y=-0.5,
                seed=seed, dt=4e-5, n_step=1000)
    base.update(kw)
    return default_params().copy(**base)


def assert_close(a: np.ndarray, b: np.ndarray, rtol: float, atol: float, what: str):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    if a.size == 0:
        return
    bad = ~np.isclose(a, b, rtol=rtol, atol=atol, equal_nan=True)
    if bad.any():
        i = np.flatnonzero(bad)[:5]
        raise AssertionError(
            f"{what}: {bad.sum()} of {a.size} differ; first {i.tolist()}: "
            f"{a.ravel()[i].tolist()} vs {b.ravel()[i].tolist()}")


# Scales of the state: positions ~20 m, velocities ~1e3 m/s.  FP64 kernels
# differ from the host's libm only in the last bits of log/cos/sin/pow/hypot,
# so states agree to ~1e-13 relative over a few steps.
def assert_state_close(gpu: dict, ref: dict, what: str, rtol: float = 1e-11):
    for k, atol in (("x", 1e-9), ("y", 1e-9), ("vx", 1e-7), ("vy", 1e-7), ("vz", 1e-7)):
        assert_close(gpu[k], ref[k], rtol, atol, f"{what} {k}")


def ulp_distance(a, b) -> np.ndarray:
    """Distance in units in the last place between FP64 arrays: the number
    of representable doubles between a and b (0 when bit-identical; +0 and
    -0 are 0 apart)."""
    def ordered(x):
        i = np.ascontiguousarray(x, dtype=np.float64).view(np.int64)
        return np.where(i < 0, np.int64(-0x8000000000000000) - i, i)
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, f"shape {a.shape} != {b.shape}"
    return np.abs(ordered(a) - ordered(b))


def assert_ulp(gpu, ref, max_ulp: int, what: str):
    """Every element within max_ulp units in the last place (0: bit-exact)."""
    u = ulp_distance(gpu, ref)
    if u.size and u.max() > max_ulp:
        i = int(np.argmax(u))
        raise AssertionError(f"{what}: {int((u > max_ulp).sum())} of {u.size} beyond {max_ulp} ulp;"
                             f" worst {int(u.max())} ulp at {i}: {np.ravel(gpu)[i]!r} vs "
                             f"{np.ravel(ref)[i]!r}")
    return int(u.max()) if u.size else 0


def ulp_of_scale(gpu, ref, scale) -> np.ndarray:
    """|gpu - ref| in units in the last place of max(|ref|, scale): the
    distance measured on the magnitude of the operands a value came from.
    A sum that cancels (a Maxwellian draw around a drift, a centre-of-mass
    velocity plus half the relative one) keeps the absolute error of its
    operands, which in its own last place can be many units."""
    ref = np.asarray(ref, dtype=np.float64)
    mag = np.maximum(np.abs(ref), np.broadcast_to(np.asarray(scale, dtype=np.float64), ref.shape))
    return np.abs(np.asarray(gpu, dtype=np.float64) - ref) / np.spacing(np.maximum(mag, 1e-300))


def assert_ulp_of_scale(gpu, ref, scale, max_ulp: float, what: str) -> float:
    u = ulp_of_scale(gpu, ref, scale)
    worst = float(u.max()) if u.size else 0.0
    if worst > max_ulp:
        i = int(np.argmax(u))
        raise AssertionError(f"{what}: {int((u > max_ulp).sum())} of {u.size} beyond {max_ulp} "
                             f"ulp of the scale; worst {worst:.2f} at {i}: "
                             f"{np.ravel(gpu)[i]!r} vs {np.ravel(ref)[i]!r}")
    return worst
