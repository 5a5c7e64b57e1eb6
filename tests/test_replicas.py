"""Replica reduction on two ranks over gloo (CPU).  Each rank runs the CPU
oracle of the same case with its own Philox key; the merged moments must be
the sum of both replicas' moments and the merged SampleStep their total."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(rank: int):
    from tests.helpers import small_case

    return small_case(seed=500 + rank, nx=20, ny=16, npc_free=5.0, first_sampling_step=0)


def _run(rank: int):
    from oracle.cpu import OracleEngine

    o = OracleEngine(_case(rank))
    o.init_cold()
    o.step(6)
    return o.fields(), o.counters()["sample_step"]


def _worker(rank, world, port, out):
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import torch.distributed as dist

    from dsmc_erlend_b200.replicas import reduce_replica_fields

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        f, ss = _run(rank)
        t = torch.from_numpy(f.copy())
        merged, total = reduce_replica_fields(t, ss)
        if rank == 0:
            np.save(out, merged.numpy())
            with open(out + ".ss", "w") as fh:
                fh.write(str(total))
    finally:
        dist.destroy_process_group()


def test_two_replicas_sum_over_gloo(tmp_path):
    out = str(tmp_path / "merged.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    merged = np.load(out)
    total = int(open(out + ".ss").read())
    f0, s0 = _run(0)
    f1, s1 = _run(1)
    assert total == s0 + s1
    np.testing.assert_array_equal(merged, f0 + f1)
    assert not np.array_equal(f0, f1)  # distinct keys, distinct replicas


# -- ensemble sharding: case i on rank i mod N, no exchange while running --------

def _ensemble():
    from dsmc_erlend_b200.ensemble import FP64, ensemble_cases

    cases = ensemble_cases(5, seed=77, steps=8, grid_range=(16, 28), precision=FP64)
    for p in cases:
        p.npc_free = min(p.npc_free, 6.0)
        p.first_sampling_step = 2
    return cases


def _run_case(p):
    from oracle.cpu import OracleEngine

    o = OracleEngine(p)
    assert o.init_cold() == 0
    assert o.step(int(p.n_step)) == 0
    return o.fields(), o.counters()


def _shard_worker(rank, world, port, out):
    import pickle
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import torch.distributed as dist

    from dsmc_erlend_b200.ensemble import gather_by_case, shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = {i: _run_case(p) for i, p in shard(_ensemble(), rank, world)}
        assert all(i % world == rank for i in mine)
        merged = gather_by_case(mine)
        if rank == 0:
            with open(out, "wb") as fh:
                pickle.dump(merged, fh)
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_equals_single_process(tmp_path):
    """Two gloo ranks each run their share of an ensemble (the CPU oracle);
    gathered, every case's moments and counters equal a single process's."""
    import pickle

    out = str(tmp_path / "merged.pkl")
    mp.start_processes(_shard_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    with open(out, "rb") as fh:
        merged = pickle.load(fh)
    cases = _ensemble()
    assert sorted(merged) == list(range(len(cases)))
    for i, p in enumerate(cases):
        f, c = _run_case(p)
        np.testing.assert_array_equal(merged[i][0], f)
        assert merged[i][1] == c


def test_shard_assignment():
    from dsmc_erlend_b200.ensemble import shard

    cases = list(range(10))
    parts = [shard(cases, r, 3) for r in range(3)]
    assert [i for i, _ in parts[0]] == [0, 3, 6, 9]
    assert sorted(i for part in parts for i, _ in part) == cases
    with pytest.raises(ValueError):
        shard(cases, 3, 3)
