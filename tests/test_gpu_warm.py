"""Warm start (dsmc_init_warm; no counterpart in the reference): particles
drawn from the local Maxwellian of a given field.

  * a uniform freestream field gives the cold start's particle count (within
    Poisson noise), the freestream's mean velocity and temperature, no
    particle inside the box, and a cell-sorted state;
  * a field varying from cell to cell is reproduced cell by cell;
  * the fill is deterministic for a seed and differs between seeds;
  * the residual check of warm.warm_start keeps a good prediction and falls
    back to the cold start for a wrong one;
  * the two-population fill (dsmc_init_warm_mixture) draws the freestream
    fraction and the second population with the mixture's moments.
"""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine, setup
from dsmc_erlend_b200.abi import FP32, FP64, WALL_DIFFUSE
from dsmc_erlend_b200.fields import K_BOLTZMANN
from dsmc_erlend_b200.timetofield import reference_field
from dsmc_erlend_b200.warm import warm_start
from helpers import small_case

pytestmark = pytest.mark.gpu


def _uniform(p, d, n=None, t=None):
    f = np.empty((p.nx * p.ny, 4))
    f[:, 0] = p.n_free if n is None else n
    f[:, 1] = d.ux_free
    f[:, 2] = d.uy_free
    f[:, 3] = p.t_free if t is None else t
    return f


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_uniform_field_matches_freestream(cuda, engine_lib, precision):
    p = small_case(WALL_DIFFUSE, seed=12, precision=precision, npc_free=20.0)
    d = setup(p)
    cold = Engine(p)
    cold.InitialConditions()
    n_cold = cold.counters()["np"]
    cold.close()
    e = Engine(p)
    e.init_warm(_uniform(p, d))
    st = e.particles()
    n = len(st["x"])
    assert abs(n - n_cold) < 5 * np.sqrt(n_cold), (n, n_cold)
    inside = (np.abs(st["x"] - p.box_x) < p.box_width / 2) & \
             (np.abs(st["y"] - p.box_y) < p.box_height / 2)
    assert not inside.any()
    assert (st["x"] >= p.x1).all() and (st["x"] < p.x2).all()
    sig = np.sqrt(K_BOLTZMANN * p.t_free / d.molecule_mass)
    for k, mean in (("vx", d.ux_free), ("vy", d.uy_free), ("vz", 0.0)):
        assert abs(st[k].mean() - mean) < 5 * sig / np.sqrt(n), k
        assert abs(st[k].std() / sig - 1) < 0.02, k
    # Cell-sorted: the cell of every slot is non-decreasing, and the starts agree.
    k = np.floor((st["x"] - p.x1) / d.dx).astype(int)
    l = np.floor((st["y"] - p.y1) / d.dy).astype(int)
    cell = k * p.ny + l
    assert (np.diff(cell) >= 0).all()
    starts = e.cell_starts()
    assert np.array_equal(np.bincount(cell, minlength=p.nx * p.ny), np.diff(starts))
    c = e.counters()
    assert c["step"] == 0 and c["sample_step"] == 0
    e.step(3)  # and it runs
    e.close()


def test_varying_field_is_reproduced(cuda, engine_lib):
    p = small_case(WALL_DIFFUSE, seed=14, npc_free=40.0, first_sampling_step=0)
    d = setup(p)
    k = np.repeat(np.arange(p.nx), p.ny)
    f = _uniform(p, d, n=p.n_free * (1.0 + 0.8 * np.sin(2 * np.pi * k / p.nx)),
                 t=p.t_free * (1.0 + k / p.nx))
    e = Engine(p)
    e.init_warm(f)
    counts = np.diff(e.cell_starts()).astype(float)
    lam = f[:, 0] * d.dv / d.weight
    # Column sums (away from the box) against the expected counts.
    box_cols = np.abs(p.x1 + (np.arange(p.nx) + 0.5) * d.dx - p.box_x) < p.box_width / 2 + d.dx
    got = counts.reshape(p.nx, p.ny).sum(1)[~box_cols]
    want = lam.reshape(p.nx, p.ny).sum(1)[~box_cols]
    assert np.all(np.abs(got - want) < 5 * np.sqrt(want) + 1)
    st = e.particles()
    kk = np.floor((st["x"] - p.x1) / d.dx).astype(int)
    for col in (3, p.nx // 2 + 7, p.nx - 4):
        v = st["vz"][kk == col]
        sig = np.sqrt(K_BOLTZMANN * p.t_free * (1.0 + col / p.nx) / d.molecule_mass)
        assert abs(v.std() / sig - 1) < 0.1, col
    e.close()


def test_fill_is_deterministic(cuda, engine_lib):
    p = small_case(seed=5)
    d = setup(p)
    a, b = Engine(p), Engine(p)
    a.init_warm(_uniform(p, d))
    b.init_warm(_uniform(p, d))
    pa, pb = a.particles(), b.particles()
    for k in pa:
        assert np.array_equal(pa[k], pb[k])
    c = Engine(small_case(seed=6))
    c.init_warm(_uniform(p, d))
    assert not np.array_equal(c.particles()["x"][:100], pa["x"][:100])
    for e in (a, b, c):
        e.close()


def test_residual_check_keeps_good_and_rejects_bad_prediction(cuda, engine_lib):
    # A dense case (mean free path ~0.1 m, well below the 1 m cells): there
    # the local Maxwellian is the state itself.  (In the rarefied cases the
    # gas upstream of the box mixes the freestream with particles the box
    # reflected, far from a Maxwellian, and the early window relaxes.)
    kw = dict(npc_free=30.0, n_free=1e19)
    p = small_case(WALL_DIFFUSE, seed=40, **kw)
    # The prediction: this case's own field, 4 replicas sampled after two
    # flow-through times of a cold start.
    want = reference_field(p, 4, transient=2000, steps=2000)
    e = Engine(small_case(WALL_DIFFUSE, seed=41, first_sampling_step=0, **kw))
    mode, res = warm_start(e, [want], check_steps=300, tol=0.05, block=2)
    assert mode == "warm", res
    assert e.counters()["step"] == 300
    for kind in ("mixture", "mixture_tensor"):  # the two-population seeds pass too
        mode, res = warm_start(e, [want], check_steps=300, tol=0.05, block=2, kind=kind)
        assert mode == "warm", (kind, res)
    bad = dict(want)
    bad["t"] = want["t"] * 1.5
    mode, res = warm_start(e, [bad], check_steps=300, tol=0.05, block=2)
    assert mode == "cold" and res[0]["t"] > 0.05
    assert e.counters()["step"] == 0
    huge = dict(want)
    huge["n"] = want["n"] * 20.0  # more particles than the case holds
    mode, res = warm_start(e, [huge], check_steps=300, tol=0.05, block=2)
    assert mode == "cold" and e.counters()["step"] == 0
    e.close()


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_mixture_fill_has_the_mixture_moments(cuda, engine_lib, precision):
    p = small_case(WALL_DIFFUSE, seed=21, precision=precision, npc_free=40.0)
    d = setup(p)
    alpha, ur = 0.4, (-150.0, 60.0)
    rxx, ryy, rzz, rxy = 900.0, 500.0, 700.0, 150.0  # the second population's tensor [K]
    f = np.zeros((p.nx * p.ny, 8))
    f[:, 0] = p.n_free
    f[:, 1] = alpha
    f[:, 2], f[:, 3] = ur
    f[:, 4:8] = (rxx, ryy, rzz, rxy)
    e = Engine(p)
    e.init_warm(f)
    st = e.particles()
    n = len(st["x"])
    c = K_BOLTZMANN / d.molecule_mass
    s_free = c * p.t_free
    mean = {"vx": alpha * d.ux_free + (1 - alpha) * ur[0],
            "vy": alpha * d.uy_free + (1 - alpha) * ur[1], "vz": 0.0}
    dx, dy = d.ux_free - ur[0], d.uy_free - ur[1]
    w = alpha * (1 - alpha)
    cov = {("vx", "vx"): alpha * s_free + (1 - alpha) * c * rxx + w * dx * dx,
           ("vy", "vy"): alpha * s_free + (1 - alpha) * c * ryy + w * dy * dy,
           ("vz", "vz"): alpha * s_free + (1 - alpha) * c * rzz,
           ("vx", "vy"): (1 - alpha) * c * rxy + w * dx * dy}
    for k, m in mean.items():
        assert abs(st[k].mean() - m) < 5 * np.sqrt(cov[(k, k)] / n), k
    for (a, b), v in cov.items():
        got = np.mean((st[a] - st[a].mean()) * (st[b] - st[b].mean()))
        scale = np.sqrt(cov[(a, a)] * cov[(b, b)])
        assert abs(got - v) < 0.03 * scale, (a, b, got, v)
    # The two populations: the share of particles within one freestream
    # thermal speed of the freestream velocity (in the x-y plane) is alpha
    # times 1 - exp(-1/2) = 0.39, plus the second population's small overlap.
    near = np.hypot(st["vx"] - d.ux_free, st["vy"] - d.uy_free) < np.sqrt(s_free)
    share = near.mean()
    assert alpha * 0.39 - 0.02 < share < alpha * 0.39 + 0.05, share
    again = Engine(p)
    again.init_warm(f)
    st2 = again.particles()
    assert all(np.array_equal(st[k], st2[k]) for k in st)
    e.step(3)
    e.synchronize()
    e.close()
    again.close()
