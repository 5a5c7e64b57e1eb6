"""Warm start with a residual check (no counterpart in the reference).

A run starts from the local Maxwellian of a predicted field (dsmc_init_warm)
instead of the uniform freestream.  After `check_steps` steps the field the
run itself sampled is compared with the prediction; when any relative L2
residual (n, ux, uy, T; fields.weighted_errors on blocks of cells) exceeds
`tol` the prediction is taken to be wrong and the run falls back to the cold
start of the reference (InitialConditions).  Sampling should begin at once (FirstSamplingStep 0 or
small): the warm field needs no flow-through transient.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from ._lib import DsmcError
from .fields import coarsen, macroscopic, mixture_input, warm_input, weighted_errors


def predicted_input(fields: Sequence[dict], kind: str = "moments",
                    engine=None) -> np.ndarray:
    """The warm-start array for the cases of a context, from one predicted
    field dict per case: "moments" (n, ux, uy, t, count: dsmc_init_warm),
    "tensor" (with txx, tyy, tzz, txy: dsmc_init_warm_tensor), or "mixture"
    / "mixture_tensor" (freestream plus a second population,
    dsmc_init_warm_mixture; needs the engine for each case's freestream)."""
    if kind in ("mixture", "mixture_tensor"):
        parts = []
        for i, f in enumerate(fields):
            p, d = engine.params[i], engine.derived[i]
            parts.append(mixture_input(f, d.ux_free, d.uy_free, p.t_free, d.molecule_mass,
                                       tensor=kind == "mixture_tensor"))
        return np.concatenate(parts, axis=0)
    return np.concatenate([warm_input(f, tensor=kind == "tensor") for f in fields], axis=0)


def sampled_field(engine, case: int = 0) -> dict:
    d = engine.derived[case]
    return macroscopic(engine.GatherGlobalField(case), d.weight, d.dv, d.molecule_mass,
                       engine.counters(case)["sample_step"])


def residual(engine, case: int, predicted: dict, block: int = 4) -> dict:
    """Relative L2 residuals of the field sampled so far against the
    prediction (fields.weighted_errors: cells weighted by their samples),
    both on blocks of `block` x `block` cells (grids that are not multiples
    of the block use single cells), so that the check measures the
    prediction rather than the sampling noise of a short window."""
    p = engine.params[case]
    got = sampled_field(engine, case)
    b = block if p.nx % block == 0 and p.ny % block == 0 else 1
    if b > 1:
        got = coarsen(got, p.nx, p.ny, b)
        predicted = coarsen(predicted, p.nx, p.ny, b)
        p = p.copy(nx=p.nx // b, ny=p.ny // b)
    return weighted_errors(got, predicted, p, engine.derived[case].u_free)


def warm_start(engine, predicted: Sequence[dict], check_steps: int = 200, tol: float = 0.05,
               block: int = 4, kind: str = "moments"):
    """Warm-starts every case of `engine` from `predicted` (one field per case,
    seeded as predicted_input's `kind`) and checks the early residual.
    Returns ("warm" | "cold", residuals per case).  On fallback the engine
    is cold-started (InitialConditions) and has run no steps; a prediction
    with more particles than a case's capacity falls back at once."""
    try:
        engine.init_warm(predicted_input(predicted, kind, engine))
    except DsmcError as e:
        if e.status != 31:  # DSMC_ERR_CAPACITY: more particles than the case holds
            raise
        engine.InitialConditions()
        return "cold", [{"n": float("inf")} for _ in predicted]
    engine.step(check_steps)
    res = [residual(engine, i, f, block) for i, f in enumerate(predicted)]
    if max(max(r.values()) for r in res) > tol:
        engine.InitialConditions()
        return "cold", res
    return "warm", res
