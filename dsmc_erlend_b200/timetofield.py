"""Time to a converged field: wall time until the field a run has sampled is
within a relative L2 tolerance (fields.field_errors: n, ux, uy, T outside
the wall cells) of a reference field, for a cold start (the reference's
InitialConditions) and for a warm start from a predicted field.

    ref = reference_field(p, replicas=8, transient=..., steps=...)
    cold = time_to_field(p, ref, start="cold", first_sampling_step=...)
    warm = time_to_field(p, ref, start="warm", predicted=field)

The reference field is the merged moments of independent replicas (distinct
Philox keys) of the same case, run far past the transient.
"""
from __future__ import annotations

import time

import numpy as np

from . import Engine, setup
from .ensemble import replicas
from .fields import field_errors, macroscopic, mixture_input, warm_input


def warm_array(p, d, predicted: dict, kind: str = "moments") -> np.ndarray:
    """The warm-start input of a predicted field: "moments" (n, u, T: one
    local Maxwellian), "tensor" (n, u and the temperature tensor: one
    anisotropic Maxwellian), "mixture" (freestream plus an isotropic second
    population, fields.mixture_input) or "mixture_tensor" (the second
    population with the remaining temperature tensor)."""
    if kind in ("mixture", "mixture_tensor"):
        return mixture_input(predicted, d.ux_free, d.uy_free, p.t_free, d.molecule_mass,
                             tensor=kind == "mixture_tensor")
    if kind not in ("moments", "tensor"):
        raise ValueError(kind)
    return warm_input(predicted, tensor=kind == "tensor")


def merged_field(eng: Engine, n_cases: int) -> dict:
    p, d = eng.params[0], eng.derived[0]
    m = sum(eng.GatherGlobalField(i) for i in range(n_cases))
    ss = sum(eng.counters(i)["sample_step"] for i in range(n_cases))
    return macroscopic(m, d.weight, d.dv, d.molecule_mass, ss)


def reference_field(p, replicas_n: int, transient: int, steps: int, seed: int = 9000) -> dict:
    """Merged field of `replicas_n` replicas sampled for `steps` steps after
    `transient` steps."""
    base = p.copy(first_sampling_step=transient)
    cases = replicas(base, replicas_n, seed=seed)
    eng = Engine(cases)
    eng.InitialConditions()
    eng.step(transient + steps)
    eng.synchronize()
    out = merged_field(eng, len(cases))
    eng.close()
    return out


def time_to_field(p, ref: dict, start: str, predicted: dict | None = None,
                  first_sampling_step: int = 0, tol: float = 0.02, check_every: int = 250,
                  max_steps: int = 200000, kind: str = "moments") -> dict:
    """Runs one case from `start` ("cold" or "warm") with sampling after
    `first_sampling_step`, checking the sampled field every `check_every`
    steps (a warm start seeds `predicted` as warm_array's `kind`); returns the steps and the wall time of the run itself (start and
    steps, device synchronised; the field checks are measurement and their
    time is left out) at the first check within `tol`."""
    q = p.copy(first_sampling_step=first_sampling_step)
    d = setup(q)
    eng = Engine(q)
    t0 = time.perf_counter()
    if start == "warm":
        eng.init_warm(warm_array(q, d, predicted, kind))
    else:
        eng.InitialConditions()
    eng.synchronize()
    seconds = time.perf_counter() - t0
    steps, err = 0, None
    while steps < max_steps:
        t0 = time.perf_counter()
        eng.step(check_every)
        eng.synchronize()
        seconds += time.perf_counter() - t0
        steps += check_every
        if steps <= first_sampling_step:
            continue
        got = merged_field(eng, 1)
        err = field_errors(got, ref, q, d.u_free)
        if max(err.values()) <= tol:
            break
    converged = err is not None and max(err.values()) <= tol
    eng.close()
    return {"start": start, "seconds": seconds, "steps": steps, "errors": err,
            "converged": converged, "first_sampling_step": first_sampling_step}


def best_cold(p, ref: dict, candidates, **kw) -> dict:
    """The fastest cold run over several sampling start steps (the cold
    start's best case: its sampling start tuned with hindsight)."""
    runs = [time_to_field(p, ref, "cold", first_sampling_step=f, **kw) for f in candidates]
    ok = [r for r in runs if r["converged"]]
    best = min(ok, key=lambda r: r["seconds"]) if ok else None
    return {"best": best, "runs": runs}


def coarse_prediction(p, factor: int = 2, npc_scale: float = 0.25, transient: int = 6000,
                      steps: int = 4000) -> tuple[dict, float]:
    """A prediction of case p from the same case on a grid `factor` times
    coarser per side with `npc_scale` of its particles per cell (so about
    npc_scale / factor^2 of the particles), run cold through its transient
    and sampled; returns the field on p's grid and the wall time it took."""
    from .sgdata import _bilinear

    q = p.copy(nx=p.nx // factor, ny=p.ny // factor, npc_free=p.npc_free * npc_scale,
               first_sampling_step=transient)
    t0 = time.perf_counter()
    eng = Engine(q)
    eng.InitialConditions()
    eng.step(transient + steps)
    eng.synchronize()
    f = merged_field(eng, 1)
    eng.close()
    seconds = time.perf_counter() - t0
    ok = (f["count"] > 0) & np.isfinite(f["ux"]) & np.isfinite(f["t"])
    d = setup(p)
    free = {"n": 0.0, "ux": d.ux_free, "uy": d.uy_free, "t": p.t_free}
    out = {}
    for k in ("n", "ux", "uy", "t"):
        v = np.where(ok, f[k], free[k]).reshape(q.nx, q.ny)
        out[k] = _bilinear(v, p, p.nx, p.ny).ravel()
    out["count"] = np.ones(p.nx * p.ny)
    return out, seconds
