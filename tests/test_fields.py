"""The two-population decomposition of a field for the mixture warm start
(fields.mixture_input), on CPU: exact moments of a known mixture give back
its parameters, freestream cells give one Maxwellian of their own moments,
and the caps hold."""
from __future__ import annotations

import numpy as np

from dsmc_erlend_b200.fields import K_BOLTZMANN, mixture_input

M = 6.63e-26
C = K_BOLTZMANN / M
U = (1500.0, 400.0)
TF = 200.0


def mixture_moments(alpha, ur, tr, n=1e17):
    """n, u and the temperature tensor of alpha freestream + (1 - alpha)
    Maxwellian(ur, tr) molecules."""
    alpha = np.asarray(alpha, float)
    ux = alpha * U[0] + (1 - alpha) * ur[0]
    uy = alpha * U[1] + (1 - alpha) * ur[1]
    s = alpha * TF + (1 - alpha) * tr  # the isotropic part, in K

    def extra(a, b):  # alpha (1 - alpha) dU_a dU_b, in K
        return alpha * (1 - alpha) * a * b / C

    dx, dy = U[0] - ur[0], U[1] - ur[1]
    return {"n": np.full(alpha.shape, n), "ux": ux, "uy": uy,
            "txx": s + extra(dx, dx), "tyy": s + extra(dy, dy), "tzz": s,
            "txy": extra(dx, dy), "count": np.ones(alpha.shape)}


def test_recovers_a_known_mixture():
    alpha = np.array([0.1, 0.3, 0.5, 0.8])
    ur = (-200.0, 150.0)
    tr = 900.0
    out = mixture_input(mixture_moments(alpha, ur, tr), U[0], U[1], TF, M, reg=0.0)
    np.testing.assert_allclose(out[:, 1], alpha, rtol=1e-10)
    np.testing.assert_allclose(out[:, 2], ur[0], rtol=1e-9)
    np.testing.assert_allclose(out[:, 3], ur[1], rtol=1e-9)
    for col in (4, 5, 6):  # Txx_r = Tyy_r = Tzz_r = T_r, Txy_r = 0
        np.testing.assert_allclose(out[:, col], tr, rtol=1e-9)
    assert np.all(out[:, 7] == 0.0)
    np.testing.assert_allclose(out[:, 0], 1e17)


def test_freestream_cells_take_one_maxwellian():
    f = mixture_moments(np.array([1.0, 1.0]), (0.0, 0.0), 0.0)
    f["tzz"] = np.array([TF, 1.02 * TF])
    f["txx"], f["tyy"] = f["tzz"].copy(), f["tzz"].copy()
    out = mixture_input(f, U[0], U[1], TF, M)
    np.testing.assert_allclose(out[:, 1], 0.0, atol=1e-12)
    np.testing.assert_allclose(out[:, 2], U[0])
    np.testing.assert_allclose(out[:, 3], U[1])
    np.testing.assert_allclose(out[:, 6], f["tzz"])


def mixture_tensor(out):
    """n, u and the temperature tensor of dsmc_init_warm_mixture's input."""
    a, uxr, uyr, rxx, ryy, rzz, rxy = (out[:, k] for k in range(1, 8))
    dx, dy = U[0] - uxr, U[1] - uyr
    w = a * (1 - a) / C
    return {"ux": a * U[0] + (1 - a) * uxr, "uy": a * U[1] + (1 - a) * uyr,
            "txx": a * TF + (1 - a) * rxx + w * dx * dx,
            "tyy": a * TF + (1 - a) * ryy + w * dy * dy,
            "tzz": a * TF + (1 - a) * rzz, "txy": (1 - a) * rxy + w * dx * dy}


def test_tensor_second_population_matches_every_moment():
    # An anisotropic cell: the isotropic form matches n, u, Tzz and the
    # trace Txx + Tyy only; the tensor form matches each entry.
    f = mixture_moments(np.array([0.2, 0.5, 0.7]), (-250.0, 100.0), 800.0)
    f["txx"] = f["txx"] + np.array([120.0, -60.0, 40.0])
    f["tyy"] = f["tyy"] - np.array([120.0, -60.0, 40.0])
    f["txy"] = f["txy"] + np.array([30.0, -20.0, 10.0])
    iso = mixture_tensor(mixture_input(f, U[0], U[1], TF, M, reg=0.0))
    full = mixture_tensor(mixture_input(f, U[0], U[1], TF, M, tensor=True, reg=0.0))
    for k in ("ux", "uy", "tzz"):
        np.testing.assert_allclose(iso[k], f[k], rtol=1e-9)
    np.testing.assert_allclose(iso["txx"] + iso["tyy"], f["txx"] + f["tyy"], rtol=1e-9)
    assert np.abs(iso["txx"] - f["txx"]).max() > 10.0
    for k in ("ux", "uy", "txx", "tyy", "tzz", "txy"):
        np.testing.assert_allclose(full[k], f[k], rtol=1e-9, atol=1e-6)


def test_caps_keep_a_valid_second_population():
    # A strongly anisotropic cell asks for alpha near 1; a cold one for a
    # negative T_r.  Both are capped and still match n, u and Tzz.
    f = mixture_moments(np.array([0.97, 0.6]), (-300.0, 0.0), 50.0)
    f["tzz"] = np.array([f["tzz"][0], 0.5 * TF])
    out = mixture_input(f, U[0], U[1], TF, M, alpha_max=0.9, t_floor=0.05)
    a = out[:, 1]
    assert np.all(a <= 0.9 + 1e-12) and np.all(a >= 0.0)
    assert np.all(out[:, 6] >= 0.05 * TF - 1e-9)
    np.testing.assert_allclose(a * U[0] + (1 - a) * out[:, 2], f["ux"], rtol=1e-12)
    np.testing.assert_allclose(a * TF + (1 - a) * out[:, 6], f["tzz"], rtol=1e-12)


def test_empty_and_invalid_cells_stay_empty():
    f = mixture_moments(np.array([0.5, 0.5, 0.5]), (0.0, 0.0), 300.0)
    f["n"] = np.array([0.0, 1e17, 1e17])
    f["ux"] = np.array([1.0, np.nan, 1.0])
    out = mixture_input(f, U[0], U[1], TF, M)
    assert np.all(out[:2] == 0.0) and out[2, 0] > 0
