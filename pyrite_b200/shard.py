"""History sharding across ranks, one process per GPU.

The reference shards a run into independent history blocks
(``montecarlo/runner/history_shards.py:1-23``, ``runner/block_transport.py``):
block k transports histories ``[start_k, start_k + n_k)`` with its own
counter-RNG keys, and the blocks' spectra and tallies add exactly. Here each
rank takes one contiguous range; with the Philox stream keyed by (seed,
history, draw) a history's result does not depend on which rank ran it, so
the partition changes nothing but the order of the final FP64 sums. The data
path has no collective: each rank scores its own batches into device-resident
spectra, and one all-reduce at the end sums spectra (FP64) and tallies
(int64), as ``ncclAllReduce`` over NVLink when the group is NCCL.
"""

from __future__ import annotations

from typing import Iterator


def history_range(n_histories: int, rank: int, world: int) -> tuple[int, int]:
    """``(start, count)`` of rank ``rank``'s block of ``n_histories`` over ``world`` ranks.

    Blocks are contiguous, cover ``[0, n_histories)`` exactly once and differ
    in size by at most one history.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n_histories < 0:
        raise ValueError("n_histories must be >= 0")
    lo = n_histories * rank // world
    hi = n_histories * (rank + 1) // world
    return lo, hi - lo


def batches(start: int, count: int, batch: int) -> Iterator[tuple[int, int]]:
    """Split ``[start, start + count)`` into ``(e_start, n)`` batches of at most ``batch``."""
    if batch < 1:
        raise ValueError("batch must be >= 1")
    e = start
    end = start + count
    while e < end:
        n = min(batch, end - e)
        yield e, n
        e += n


def reduce_results(results: dict, group=None) -> dict:
    """Sum every tensor of ``results`` over the process group, in place.

    Floating tensors reduce in FP64 and integer tallies in int64 (unsigned
    64-bit histograms are carried as int64 bit patterns, exact for counts
    below 2**63). Tensors are reduced in sorted key order so every rank issues
    the same collectives in the same order. Returns ``results``.
    """
    import torch
    import torch.distributed as dist

    for key in sorted(results):
        t = results[key]
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{key}: expected a tensor, got {type(t).__name__}")
        if t.dtype.is_floating_point:
            buf = t if t.dtype == torch.float64 else t.to(torch.float64)
        else:
            buf = t if t.dtype == torch.int64 else t.to(torch.int64)
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        if buf is not t:
            t.copy_(buf)
    return results


def average_gradients(grad, group=None):
    """Data-parallel training step: replace ``grad`` (one flat tensor of every
    parameter's gradient) by its mean over the process group, in place, so
    every rank applies the same optimizer step to the same parameters. One
    all-reduce of the ~330 k surrogate parameters per step."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if world > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
        grad.div_(world)
    return grad
