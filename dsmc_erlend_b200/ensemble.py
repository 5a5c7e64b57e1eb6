"""The batched ensemble: many independent cases of uneven grid and particle
count advanced together in one context (one CUDA graph per step).

ensemble_cases() draws the case parameters from one seed:
  square grid side U[64, 400]; angle U[-30, 30] deg; Ma U[2, 8];
  n log-uniform in [1e16, 1e18] m^-3; T 200 K; square box side U[2, 6] m;
  wall model uniform over specular, diffuse, CLL with acc_n, acc_t U[0, 1];
  NPCFree U[5, 20]; domain [-20, 20]^2 m and Dt 1e-5 s as the reference's.
Each case gets its own Philox key, so a case run inside the ensemble and the
same case run alone produce identical results.
"""
from __future__ import annotations

import numpy as np

from .abi import FP32, FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, Params, default_params

WALL_CHOICES = (WALL_SPECULAR, WALL_DIFFUSE, WALL_CLL)


def case_key(seed: int, i: int) -> int:
    """64-bit Philox key of case i of an ensemble drawn from `seed`."""
    x = (seed * 0x9E3779B97F4A7C15 + (i + 1) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x ^= x >> 31
    x = (x * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 29)


def ensemble_cases(n: int = 256, seed: int = 2024, steps: int = 5000,
                   precision: int = FP32, grid_range=(64, 400)) -> list[Params]:
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(n):
        side = int(rng.integers(grid_range[0], grid_range[1] + 1))
        wall = WALL_CHOICES[int(rng.integers(0, 3))]
        box = float(rng.uniform(2.0, 6.0))
        p = default_params().copy(
            nx=side, ny=side,
            attack_angle=float(rng.uniform(-30.0, 30.0)),
            ma_free=float(rng.uniform(2.0, 8.0)),
            n_free=float(10.0 ** rng.uniform(16.0, 18.0)),
            t_free=200.0,
            box_width=box, box_height=box,
            wall_model=wall,
            cll_normal=float(rng.uniform(0.0, 1.0)),
            cll_tangential=float(rng.uniform(0.0, 1.0)),
            npc_free=float(rng.uniform(5.0, 20.0)),
            n_step=steps, first_sampling_step=steps // 2,
            precision=precision,
            seed=case_key(seed, i))
        cases.append(p)
    return cases


def shard(cases: list[Params], rank: int, world: int) -> list[tuple[int, Params]]:
    """The cases rank `rank` of `world` runs: case i goes to rank i mod world,
    so uneven cases spread evenly on average and every rank's share is known
    without communication.  Returns (case index, parameters) pairs in case
    order.  Cases are independent: the ranks exchange nothing while they run
    (each case keeps its own Philox key, so its results do not depend on
    which rank runs it or with which other cases)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return [(i, p) for i, p in enumerate(cases) if i % world == rank]


def gather_by_case(local: dict, group=None) -> dict:
    """Merges {case index: result} dicts of every rank into one on every rank
    (torch.distributed all_gather_object; for per-case summaries such as
    counters or small fields, not for bulk data)."""
    import torch.distributed as dist

    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for part in parts:
        merged.update(part)
    return dict(sorted(merged.items()))


def replicas(p: Params, n: int, seed: int = 1) -> list[Params]:
    """n copies of one case with distinct Philox keys (replica statistics)."""
    return [p.copy(seed=case_key(seed, i)) for i in range(n)]


__all__ = ["ensemble_cases", "replicas", "case_key", "shard", "gather_by_case", "FP32", "FP64"]
