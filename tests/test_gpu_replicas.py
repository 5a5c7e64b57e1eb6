"""The device side of the replica reduction (dsmc_erlend_b200/replicas.py) on
one GPU: engine_replica_reduce reads a case's moments into device memory,
reduces them and stores the merged moments and SampleStep back into the
context.  A second replica's moments stand in for the other rank (the
reducer adds them), so the read-out and store-back are checked against the
sum taken on the host; the NCCL path itself runs with a world of one."""
from __future__ import annotations

import numpy as np
import pytest

from dsmc_erlend_b200 import Engine
from dsmc_erlend_b200.abi import WALL_DIFFUSE
from dsmc_erlend_b200.engine import write_field
from dsmc_erlend_b200.replicas import engine_replica_reduce
from tests.helpers import small_case

pytestmark = pytest.mark.gpu


def _replica(seed):
    g = Engine(small_case(WALL_DIFFUSE, seed=seed, first_sampling_step=2))
    g.InitialConditions()
    g.step(20)
    g.synchronize()
    return g


def test_replica_reduce_reads_out_and_stores_back(cuda, engine_lib, tmp_path):
    torch = cuda
    a, b = _replica(610), _replica(611)
    fa, fb = a.fields(), b.fields()
    sa, sb = a.counters()["sample_step"], b.counters()["sample_step"]
    assert sa > 0 and not np.array_equal(fa, fb)

    def add_other(fields, sample_step):  # the other rank's all-reduce share
        fields += torch.from_numpy(fb.reshape(-1, 17)).cuda()
        return fields, sample_step + sb

    total = engine_replica_reduce(a, reduce=add_other)
    assert total == sa + sb == a.counters()["sample_step"]
    np.testing.assert_array_equal(a.fields(), fa + fb)
    # Printing() of the merged context equals Printing() of the host sum.
    a.Printing(str(tmp_path / "dev"))
    write_field(a.params[0], a.derived[0], sa + sb, fa + fb, str(tmp_path / "host"))
    for name in ("DSMC2D_Field.plt", "DSMC2D_Field.json"):
        assert (tmp_path / "dev" / "diffuse" / name).read_bytes() == \
            (tmp_path / "host" / "diffuse" / name).read_bytes()
    # The run continues from the merged moments.
    a.step(2)
    a.synchronize()
    assert a.counters()["sample_step"] == sa + sb + 2
    a.close()
    b.close()


def test_replica_reduce_over_nccl_world_of_one(cuda, engine_lib, tmp_path):
    import datetime
    import os

    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29561")
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60),
                            device_id=cuda.device("cuda", 0))
    try:
        a = _replica(612)
        f, s = a.fields(), a.counters()["sample_step"]
        assert engine_replica_reduce(a) == s
        np.testing.assert_array_equal(a.fields(), f)
        a.close()
    finally:
        dist.destroy_process_group()
