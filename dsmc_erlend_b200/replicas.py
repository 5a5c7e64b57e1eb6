"""Replica statistics across ranks.

DSMC fields are time averages of sampled moments, so independent replicas of
one case (same parameters, different Philox keys) combine by summing: every
moment of CELL (include/Cell.h:4-10) is a sum over samples, and the merged
SampleStep is the total number of sampling steps.  Printing() of the merged
field then yields the mean over all replicas' samples (Sampling.cpp:114-133
divides by SampleStep).  One all-reduce per output, no per-step exchange:
the replica path shards with no data-path collective.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def reduce_replica_fields(fields: torch.Tensor, sample_step: int, group=None):
    """Sums a (ncell, 17) FP64 moment tensor and the sample counts over the
    ranks of `group`, in place; returns (fields, total sample steps).
    Works with NCCL (device tensors) and gloo (host tensors)."""
    if fields.dtype != torch.float64:
        raise TypeError("moments are FP64")
    dist.all_reduce(fields, op=dist.ReduceOp.SUM, group=group)
    ss = torch.tensor([float(sample_step)], dtype=torch.float64, device=fields.device)
    dist.all_reduce(ss, op=dist.ReduceOp.SUM, group=group)
    return fields, int(ss.item())


def engine_replica_reduce(engine, case: int = 0, group=None, reduce=None) -> int:
    """All-reduces the moments of one case of a device Engine over NCCL and
    stores the merged moments back in the context.  Returns the merged
    SampleStep.  `reduce(fields, sample_step) -> (fields, total)` replaces
    the all-reduce (default reduce_replica_fields over `group`)."""
    p = engine.params[case]
    buf = torch.empty(p.nx * p.ny * 17, dtype=torch.float64, device="cuda")
    engine.fields_to_device(case, buf.data_ptr())
    torch.cuda.synchronize()
    ss = engine.counters(case)["sample_step"]
    if reduce is None:
        _, total = reduce_replica_fields(buf.view(-1, 17), ss, group)
    else:
        _, total = reduce(buf.view(-1, 17), ss)
    engine.fields_from_device(case, buf.data_ptr(), total)
    torch.cuda.synchronize()
    return total
