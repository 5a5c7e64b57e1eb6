"""Macroscopic fields from the sampled moments, and field distances.

The moments are the reference's CELL layout (include/Cell.h:4-10, 17 doubles
per cell).  The conversion follows Printing (src/Sampling.cpp:36-268):
n = W CountNP / SampleStep / DV, u = CountV / CountNP, T = m (<vv> - u u) / k
with T the mean of its three diagonal components.
"""
from __future__ import annotations

import numpy as np

K_BOLTZMANN = 1.380662e-23


def macroscopic(cells: np.ndarray, weight: float, dv: float, molecule_mass: float,
                sample_step: int) -> dict:
    """n, ux, uy, T and the sample count of every cell from summed moments."""
    cells = np.asarray(cells, dtype=np.float64)
    npc = cells[:, 0]
    n = weight * npc / max(sample_step, 1) / dv
    with np.errstate(invalid="ignore", divide="ignore"):
        u = cells[:, 1:4] / npc[:, None]
        vv = cells[:, [4, 8, 12]] / npc[:, None]
        t = molecule_mass * (vv - u * u) / K_BOLTZMANN
        txy = molecule_mass * (cells[:, 5] / npc - u[:, 0] * u[:, 1]) / K_BOLTZMANN
    return {"n": n, "ux": u[:, 0], "uy": u[:, 1], "t": t.mean(axis=1), "count": npc,
            "txx": t[:, 0], "tyy": t[:, 1], "tzz": t[:, 2], "txy": txy}


def wall_cells(p) -> np.ndarray:
    """Cells whose centre lies within one cell of the box (x-major)."""
    dx = (p.x2 - p.x1) / p.nx
    dy = (p.y2 - p.y1) / p.ny
    k, l = np.meshgrid(np.arange(p.nx), np.arange(p.ny), indexing="ij")
    xc = p.x1 + (k.ravel() + 0.5) * dx
    yc = p.y1 + (l.ravel() + 0.5) * dy
    return (np.abs(xc - p.box_x) < p.box_width / 2 + dx) & \
           (np.abs(yc - p.box_y) < p.box_height / 2 + dy)


def weighted_errors(a: dict, b: dict, p, u_free: float) -> dict:
    """Relative L2 errors of field a against field b outside the wall cells,
    each cell weighted by b's sample count: the statistically natural norm
    for a short sampling window, where a cell's noise falls as one over the
    root of its samples.  Velocities are normalised by the freestream speed,
    n and T by their own weighted norms."""
    ok = ~wall_cells(p) & (a["count"] > 0) & (b["count"] > 0)
    for k in ("ux", "uy", "t"):
        ok &= np.isfinite(a[k]) & np.isfinite(b[k])
    w = np.where(ok, b["count"], 0.0)
    out = {}
    for k in ("n", "t"):
        d = np.nan_to_num(a[k] - b[k])
        out[k] = np.sqrt((w * d * d).sum() / max((w * np.nan_to_num(b[k]) ** 2).sum(), 1e-300))
    for k in ("ux", "uy"):
        d = np.nan_to_num(a[k] - b[k])
        out[k] = np.sqrt((w * d * d).sum() / max(w.sum(), 1e-300)) / u_free
    return out


def field_errors(a: dict, b: dict, p, u_free: float) -> dict:
    """Relative L2 errors of field a against field b outside the wall cells.

    n is compared over every such cell both fields sampled.  Velocity and
    temperature are moments per sampled particle, undefined where almost
    nothing is sampled (the near-vacuum wake behind the box, where even
    independent runs of the reference differ by O(100%)); ux, uy and T leave
    out cells whose sample count in b is below 5% of b's median.  Velocities
    are normalised by the freestream speed, n by ||n_b||, T by ||T_b||."""
    sampled = ~wall_cells(p) & (a["count"] > 0) & (b["count"] > 0)
    dense = sampled & (b["count"] >= 0.05 * np.median(b["count"][b["count"] > 0]))
    out = {"n": np.linalg.norm(a["n"][sampled] - b["n"][sampled]) /
                np.linalg.norm(b["n"][sampled]),
           "t": np.linalg.norm(a["t"][dense] - b["t"][dense]) / np.linalg.norm(b["t"][dense])}
    for key in ("ux", "uy"):
        out[key] = np.linalg.norm(a[key][dense] - b[key][dense]) / \
            (u_free * np.sqrt(max(int(dense.sum()), 1)))
    return out


def warm_input(f: dict, tensor: bool = False) -> np.ndarray:
    """The (n, ux, uy, T) array per cell that dsmc_init_warm takes, or with
    tensor the (n, ux, uy, Txx, Tyy, Tzz, Txy) one of dsmc_init_warm_tensor;
    cells without samples are left empty (n = 0)."""
    ok = np.isfinite(f["ux"]) & np.isfinite(f["uy"]) & np.isfinite(f["t"]) & (f["count"] > 0)
    keys = ("txx", "tyy", "tzz", "txy") if tensor else ("t",)
    for k in keys:
        ok &= np.isfinite(f[k])
    out = np.zeros((len(f["n"]), 3 + len(keys)), dtype=np.float64)
    out[ok, 0] = f["n"][ok]
    out[ok, 1] = f["ux"][ok]
    out[ok, 2] = f["uy"][ok]
    for i, k in enumerate(keys):
        out[ok, 3 + i] = f[k][ok] if k == "txy" else np.maximum(f[k][ok], 0.0)
    return out


def mixture_input(f: dict, ux_free: float, uy_free: float, t_free: float,
                  molecule_mass: float, tensor: bool = False, alpha_max: float = 0.9,
                  t_floor: float = 0.05, reg: float = 0.05) -> np.ndarray:
    """dsmc_init_warm_mixture's (n, alpha, ux_r, uy_r, Txx_r, Tyy_r, Tzz_r,
    Txy_r) per cell from a field with the temperature tensor (n, ux, uy, txx,
    tyy, tzz, txy): each cell's gas as a fraction alpha of freestream
    molecules (the case's freestream Maxwellian, U = (ux_free, uy_free),
    T = t_free) and 1 - alpha of a second population (u_r and its tensor).

    For such a mixture, with c = k / m and an isotropic second population T_r:
        u   = alpha U + (1 - alpha) u_r
        Tzz = alpha T_free + (1 - alpha) T_r
        c (Txx + Tyy - 2 Tzz) = alpha (1 - alpha) |U - u_r|^2
                              = alpha / (1 - alpha) |U - u|^2,
    so R = c (Txx + Tyy - 2 Tzz) / |U - u|^2 gives alpha = R / (1 + R), then
    u_r = (u - alpha U) / (1 - alpha) and T_r = (Tzz - alpha T_free) /
    (1 - alpha).  |U - u|^2 is regularised by (reg |U|)^2 so that a cell
    at freestream conditions (both terms near zero) takes alpha near 0 (one
    Maxwellian of its own moments); alpha is capped at alpha_max (u_r
    amplifies errors in u by 1 / (1 - alpha)) and lowered where T_r would
    fall below t_floor T_free.  That matches n, u and Tzz exactly, and
    Txx + Tyy when alpha is not capped.  With `tensor` the second
    population keeps that alpha but takes the whole remaining tensor,
        T_r,ij = (T_ij - alpha T_free d_ij - alpha (1 - alpha) dU_i dU_j / c)
                 / (1 - alpha),   dU = U - u_r,
    so that the mixture matches Txx, Tyy, Tzz and Txy one by one (its
    diagonal kept at t_floor T_free or more, its xy entry within 0.95 of
    the geometric mean of the diagonal)."""
    c = K_BOLTZMANN / molecule_mass
    n = np.asarray(f["n"], dtype=np.float64)
    ux, uy = np.asarray(f["ux"], np.float64), np.asarray(f["uy"], np.float64)
    txx, tyy, tzz = (np.asarray(f[k], np.float64) for k in ("txx", "tyy", "tzz"))
    txy = np.asarray(f.get("txy", np.zeros_like(n)), np.float64)
    ok = np.isfinite(ux) & np.isfinite(uy) & np.isfinite(txx) & np.isfinite(tyy) & \
        np.isfinite(tzz) & (n > 0) & (np.asarray(f.get("count", np.ones_like(n))) > 0)
    if tensor:
        ok &= np.isfinite(txy)
    u2 = ux_free * ux_free + uy_free * uy_free
    e = (ux_free - ux) ** 2 + (uy_free - uy) ** 2 + reg * reg * u2
    tfl = t_floor * t_free
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.maximum(c * (txx + tyy - 2.0 * tzz), 0.0) / e
        alpha = np.minimum(r / (1.0 + r), alpha_max)
        # T_r >= tfl  <=>  alpha <= (Tzz - tfl) / (T_free - tfl)
        cap = np.where(t_free > tfl, (tzz - tfl) / (t_free - tfl), 0.0)
        alpha = np.clip(np.minimum(alpha, cap), 0.0, alpha_max)
        alpha = np.where(ok, alpha, 0.0)
        uxr = (ux - alpha * ux_free) / (1.0 - alpha)
        uyr = (uy - alpha * uy_free) / (1.0 - alpha)
        tr = np.maximum((tzz - alpha * t_free) / (1.0 - alpha), 0.0)
        if tensor:
            dx, dy = ux_free - uxr, uy_free - uyr
            w = alpha * (1.0 - alpha) / c
            rxx = np.maximum((txx - alpha * t_free - w * dx * dx) / (1.0 - alpha), tfl)
            ryy = np.maximum((tyy - alpha * t_free - w * dy * dy) / (1.0 - alpha), tfl)
            rzz = np.maximum(tr, tfl)
            rxy = (txy - w * dx * dy) / (1.0 - alpha)
            lim = 0.95 * np.sqrt(rxx * ryy)
            rxy = np.clip(rxy, -lim, lim)
        else:
            rxx = ryy = rzz = tr
            rxy = np.zeros_like(tr)
    out = np.zeros((len(n), 8), dtype=np.float64)
    for i, v in enumerate((n, alpha, uxr, uyr, rxx, ryy, rzz, rxy)):
        out[ok, i] = np.broadcast_to(v, n.shape)[ok]
    return out


def coarsen(f: dict, nx: int, ny: int, b: int) -> dict:
    """Field on blocks of b x b cells (nx, ny multiples of b): n averaged,
    velocity and temperature weighted by the sample counts."""
    def blocks(a):
        return a.reshape(nx // b, b, ny // b, b)

    cnt = blocks(np.nan_to_num(f["count"])).sum(axis=(1, 3))
    out = {"n": blocks(f["n"]).mean(axis=(1, 3)).ravel(), "count": cnt.ravel()}
    w = blocks(np.nan_to_num(f["count"]))
    with np.errstate(invalid="ignore", divide="ignore"):
        for k in ("ux", "uy", "t"):
            out[k] = ((blocks(np.nan_to_num(f[k])) * w).sum(axis=(1, 3)) / cnt).ravel()
    return out
