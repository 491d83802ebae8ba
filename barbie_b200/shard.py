"""One bispectrum split over several GPUs, one process per GPU.

The reference's MPI estimator splits the triangle loop over ranks and sums
the bins with MPI_Reduce (zBS_fast_mpi.c:149,294-296). Here each rank builds a
plan with ``shard=(rank, world)``: the library gives every rank the same
longest-processing-time assignment of ring triplets (beam_shard_assign) and
the rank's plan sums only its own triplets, so its bs/norm/count are partial
sums. The one exchange is a sum-reduce of those partial bins (FP64 bs and
norm, int64 counts) over torch.distributed -- NCCL between GPUs, gloo on the
host -- after which every rank normalises as the reference does
(barbie.c:390: out = bs / (vol * norm)).

Counts are integers and add exactly; bs and norm differ from the one-GPU
result only by the order of the final additions.
"""
from __future__ import annotations

import numpy as np


def finalize(bs: np.ndarray, norm: np.ndarray, count: np.ndarray, vol: float, ana_sum=None) -> dict:
    """Bins from summed partials: out = bs / (vol * norm), as the epilogue
    kernel and barbie.c:390 compute it, and ana = ana_sum / norm (barbie.c:391);
    0/0 gives NaN for empty bins."""
    if ana_sum is None:
        ana_sum = np.zeros_like(bs)
    with np.errstate(divide="ignore", invalid="ignore"):
        out = bs / (vol * norm)
        ana = ana_sum / norm
    return dict(bs=bs, norm=norm, out=out, count=count, ana_sum=ana_sum, ana=ana)


def sum_partials(parts: list[dict], vol: float) -> dict:
    """Add the partial bins of all shards in shard order (one process)."""
    bs = np.zeros_like(parts[0]["bs"])
    norm = np.zeros_like(parts[0]["norm"])
    ana_sum = np.zeros_like(parts[0]["bs"])
    count = np.zeros_like(parts[0]["count"])
    for p in parts:
        bs += p["bs"]
        norm += p["norm"]
        ana_sum += p.get("ana_sum", 0.0)
        count += p["count"]
    return finalize(bs, norm, count, vol, ana_sum)


def allreduce_partials(part: dict, vol: float, group=None, device=None) -> dict:
    """Sum-reduce this rank's partial bins over the process group and
    normalise. `device` is where the reduction buffers live: a CUDA device for
    NCCL, None (host) for gloo. Every rank makes the same two collectives."""
    import torch
    import torch.distributed as dist

    shape, cshape = part["bs"].shape, part["count"].shape
    ana_sum = part.get("ana_sum", np.zeros(shape))
    vals = torch.from_numpy(np.concatenate([part["bs"].ravel(), part["norm"].ravel(), ana_sum.ravel()]))
    cnt = torch.from_numpy(np.ascontiguousarray(part["count"], dtype=np.int64).ravel().copy())
    if device is not None:
        vals, cnt = vals.to(device), cnt.to(device)
    dist.all_reduce(vals, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(cnt, op=dist.ReduceOp.SUM, group=group)
    vals, cnt = vals.cpu().numpy(), cnt.cpu().numpy()
    n = int(np.prod(shape))
    return finalize(vals[:n].reshape(shape), vals[n:2 * n].reshape(shape), cnt.reshape(cshape), vol,
                    vals[2 * n:].reshape(shape))


def run_sharded(ctx, r2c, rank: int, world: int, NN: int, UL_k1: int, LL_k1: int, BW_k1: int, *, group=None,
                device=None, **plan_kw) -> dict:
    """This rank's share of one bispectrum, reduced over the group: a plan
    with shard=(rank, world), one run, then allreduce_partials."""
    from barbie_b200 import beam

    plan = beam.Plan(ctx, NN, UL_k1, LL_k1, BW_k1, shard=(rank, world), **plan_kw)
    try:
        part = plan.run(r2c)
        vol = plan.info["vol"]
    finally:
        plan.close()
    return allreduce_partials(part, vol, group=group, device=device)
