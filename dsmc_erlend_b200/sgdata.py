"""Training data of the field surrogate: DSMC ensembles run on the GPU, their
sampled fields resampled to the surrogate's canvas, and the case inputs.

The canvas is the domain on RES x RES cells, x-major like the solver's fields
(index kx * RES + ly), i.e. an NHWC image whose H axis is x and W axis is y.
"""
from __future__ import annotations

import math

import numpy as np

from . import Engine, setup
from .ensemble import WALL_CHOICES, case_key
from .fields import macroscopic
from .abi import FP32, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, default_params
from .surrogate import CH, IN_CH, OUT_CH, OUT_NAMES, RES


def surrogate_cases(n: int, seed: int, steps: int = 5000, precision: int = FP32,
                    grid_range=(64, 400)) -> list:
    """Cases for the surrogate's data: the ensemble generator's ranges (grid
    side U[64, 400], angle U[-30, 30] deg, Ma U[2, 8], n log-U[1e16, 1e18],
    box U[2, 6] m, wall uniform over specular, diffuse, CLL with U[0, 1]
    coefficients, NPCFree U[5, 20]) with the box width and height drawn
    independently, so that rectangular boxes are covered."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        side = int(rng.integers(grid_range[0], grid_range[1] + 1))
        out.append(default_params().copy(
            nx=side, ny=side,
            attack_angle=float(rng.uniform(-30.0, 30.0)),
            ma_free=float(rng.uniform(2.0, 8.0)),
            n_free=float(10.0 ** rng.uniform(16.0, 18.0)),
            t_free=200.0,
            box_width=float(rng.uniform(2.0, 6.0)),
            box_height=float(rng.uniform(2.0, 6.0)),
            wall_model=WALL_CHOICES[int(rng.integers(0, 3))],
            cll_normal=float(rng.uniform(0.0, 1.0)),
            cll_tangential=float(rng.uniform(0.0, 1.0)),
            npc_free=float(rng.uniform(5.0, 20.0)),
            n_step=steps, first_sampling_step=steps // 2,
            precision=precision, seed=case_key(seed, i)))
    return out


def canvas_centres(p, res: int = RES):
    xs = p.x1 + (np.arange(res) + 0.5) * (p.x2 - p.x1) / res
    ys = p.y1 + (np.arange(res) + 0.5) * (p.y2 - p.y1) / res
    return np.meshgrid(xs, ys, indexing="ij")


def box_mask(p, res: int = RES) -> np.ndarray:
    x, y = canvas_centres(p, res)
    return ((np.abs(x - p.box_x) < p.box_width / 2) &
            (np.abs(y - p.box_y) < p.box_height / 2)).astype(np.float32)


def case_input(p, res: int = RES) -> np.ndarray:
    """(res, res, CH) float32: the channels listed in the surrogate module."""
    x, y = canvas_centres(p, res)
    a = math.radians(p.attack_angle)
    wall = [1.0 if p.wall_model == w else 0.0 for w in (WALL_SPECULAR, WALL_DIFFUSE, WALL_CLL)]
    cll = (p.cll_normal, p.cll_tangential) if p.wall_model == WALL_CLL else (0.0, 0.0)
    consts = [p.ma_free / 8.0, math.cos(a), math.sin(a), math.log10(p.n_free) - 17.0, *wall,
              *cll, p.box_width / 6.0, p.box_height / 6.0]
    out = np.zeros((res, res, CH), dtype=np.float32)
    out[..., 0] = box_mask(p, res)
    out[..., 1] = x / 20.0
    out[..., 2] = y / 20.0
    for i, v in enumerate(consts):
        out[..., 3 + i] = v
    assert 3 + len(consts) == IN_CH
    return out


def _bilinear(src: np.ndarray, p, tx: int, ty: int) -> np.ndarray:
    """Resamples a cell field src (sx, sy) on the domain to tx x ty cells:
    bilinear between cell centres, clamped at the edges."""
    sx, sy = src.shape
    xs = (np.arange(tx) + 0.5) / tx * sx - 0.5
    ys = (np.arange(ty) + 0.5) / ty * sy - 0.5
    fx, fy = np.meshgrid(np.clip(xs, 0, sx - 1), np.clip(ys, 0, sy - 1), indexing="ij")
    i0 = np.minimum(np.floor(fx).astype(int), max(sx - 2, 0))
    j0 = np.minimum(np.floor(fy).astype(int), max(sy - 2, 0))
    wx, wy = fx - i0, fy - j0
    i1, j1 = np.minimum(i0 + 1, sx - 1), np.minimum(j0 + 1, sy - 1)
    return ((1 - wx) * (1 - wy) * src[i0, j0] + wx * (1 - wy) * src[i1, j0] +
            (1 - wx) * wy * src[i0, j1] + wx * wy * src[i1, j1])


def t_scale(p) -> float:
    """The temperature unit of the surrogate: the freestream's stagnation
    temperature TFree (1 + (gamma - 1) / 2 Ma^2), gamma = 5/3, so that the
    targets of every Mach number are of order one."""
    return p.t_free * (1.0 + p.ma_free ** 2 / 3.0)


def _free_and_scale(p, d):
    ts = t_scale(p)
    free = {"n": p.n_free, "ux": d.ux_free, "uy": d.uy_free, "t": p.t_free, "txx": p.t_free,
            "tyy": p.t_free, "tzz": p.t_free, "txy": 0.0}
    scale = {"n": p.n_free, "ux": d.u_free, "uy": d.u_free, "t": ts, "txx": ts, "tyy": ts,
             "tzz": ts, "txy": ts}
    return free, scale


def field_target(p, d, f: dict, res: int = RES):
    """A sampled field on the canvas, normalised: (res, res, OUT_CH) targets
    n / NFree, ux / UFree, uy / UFree, T / t_scale and Txx, Tyy, Tzz, Txy /
    t_scale, and the (res, res) mask of canvas cells that are outside the
    box and whose neighbourhood was sampled."""
    nx, ny = p.nx, p.ny
    valid = (f["count"] > 0) & np.isfinite(f["ux"]) & np.isfinite(f["t"])
    for k in OUT_NAMES[4:]:
        valid &= np.isfinite(f[k])
    free, scale = _free_and_scale(p, d)
    out = np.zeros((res, res, OUT_CH), dtype=np.float32)
    for i, k in enumerate(OUT_NAMES):
        v = np.where(valid, f[k], free[k] if k != "n" else 0.0).reshape(nx, ny)
        out[..., i] = _bilinear(v, p, res, res) / scale[k]
    ok = _bilinear(valid.reshape(nx, ny).astype(np.float64), p, res, res) > 0.99
    mask = (ok & (box_mask(p, res) == 0)).astype(np.float32)
    return out, mask


def prediction_field(p, d, pred: np.ndarray) -> dict:
    """A canvas prediction (res, res, >= 4) back on the case's grid, as the
    field dict dsmc_init_warm's input is made from (count 1 outside the
    box, n = 0 inside it); with 8 channels also the temperature tensor that
    dsmc_init_warm_tensor takes."""
    back = {}
    _, scale = _free_and_scale(p, d)
    for i, k in enumerate(OUT_NAMES[:pred.shape[-1]]):
        back[k] = (_bilinear(pred[..., i].astype(np.float64), p, p.nx, p.ny) * scale[k]).ravel()
    back["n"] = np.maximum(back["n"], 0.0)
    for k in ("t", "txx", "tyy", "tzz"):
        if k in back:
            back[k] = np.maximum(back[k], 1.0)
    xs = p.x1 + (np.arange(p.nx) + 0.5) * (p.x2 - p.x1) / p.nx
    ys = p.y1 + (np.arange(p.ny) + 0.5) * (p.y2 - p.y1) / p.ny
    x, y = np.meshgrid(xs, ys, indexing="ij")
    inside = ((np.abs(x - p.box_x) < p.box_width / 2) &
              (np.abs(y - p.box_y) < p.box_height / 2)).ravel()
    back["n"][inside] = 0.0
    back["count"] = np.where(inside, 0.0, 1.0)
    return back


def generate(cases, chunk: int = 128, verbose: bool = False):
    """Runs the cases as ensembles of `chunk` (each case to its own n_step,
    the ensemble to the longest) and returns inputs (N, RES, RES, IN_CH) float16 (the network pads them to CH),
    targets (N, RES, RES, OUT_CH), masks (N, RES, RES) and the particle-steps
    run."""
    xs, ts, ms = [], [], []
    ps_total = 0
    for c0 in range(0, len(cases), chunk):
        part = cases[c0:c0 + chunk]
        eng = Engine(part)
        eng.InitialConditions()
        eng.step(max(p.n_step for p in part))
        eng.synchronize()
        for i, p in enumerate(part):
            d = eng.derived[i]
            c = eng.counters(i)
            ps_total += c["particle_steps"]
            f = macroscopic(eng.GatherGlobalField(i), d.weight, d.dv, d.molecule_mass,
                            c["sample_step"])
            t, m = field_target(p, d, f)
            xs.append(case_input(p)[..., :IN_CH].astype(np.float16))  # compact; padded on use
            ts.append(t)
            ms.append(m)
        eng.close()
        if verbose:
            print(f"generated {c0 + len(part)}/{len(cases)}", flush=True)
    return np.stack(xs), np.stack(ts), np.stack(ms), ps_total
