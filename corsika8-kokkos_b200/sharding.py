"""Sharding one shower's radio projection over ranks (one process per GPU).

Pairs (track, antenna) are independent and a trace is a sum, so the path
shards without a collective on the data path:

* antenna shards: each rank owns a contiguous run of antennas (balanced by
  trace bins) and projects every track at them; the disjoint traces are
  gathered once at the end;
* track shards: each rank projects a contiguous range of the tracks at every
  antenna (the reference's spool partition, StaticFrontierIO.cpp:307-351);
  the int64 fixed-point snapshots are summed once at the end, which is exact
  and independent of the order (the reference's CooperativeRadioMerge,
  CooperativeRadioMerge.inl:180-202).

The helpers take a torch.distributed process group (NCCL on GPUs, gloo on
CPU); `max_over_ranks` is the device-time reduction of the benchmark.
"""
from __future__ import annotations

import numpy as np


def track_shard(count: int, rank: int, world: int) -> tuple:
    """[begin, end) of rank's contiguous share of `count` tracks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def antenna_shard(observers: np.ndarray, rank: int, world: int) -> tuple:
    """[begin, end) of rank's contiguous run of antennas, balanced by bins:
    the cut after antenna i goes where the running bin total first reaches
    rank/world of the whole."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    bins = np.asarray(observers["number_of_bins"], dtype=np.float64)
    cumulative = np.concatenate([[0.0], np.cumsum(bins)])
    total = cumulative[-1]
    cuts = [int(np.searchsorted(cumulative, total * r / world, side="left")) for r in range(world)]
    cuts.append(len(bins))
    return cuts[rank], max(cuts[rank], cuts[rank + 1])


def merge_track_shards(coreas: np.ndarray, zhs: np.ndarray, group=None) -> tuple:
    """Exact sum over ranks of int64 fixed-point traces (every rank gets it).

    Each value is split into a signed high and an unsigned low 32-bit half,
    and the halves are summed over the ranks as int64 (no half sum can leave
    the int64 range below 2^31 ranks), so the reduction cannot wrap.  The
    total is then rebuilt and checked: if any bin's exact sum lies outside the
    int64 range, OverflowError is raised on every rank and nothing is
    returned, as CooperativeRadioMerge::commit rejects an overflowing merge
    before writing a bin (CooperativeRadioMerge.inl:180-202,
    FixedAccumulatorMerge.inl:12-29)."""
    import torch
    import torch.distributed as dist

    halves = []
    shapes = []
    for traces in (coreas, zhs):
        values = np.ascontiguousarray(traces, dtype=np.int64)
        shapes.append(values.shape)
        flat = values.reshape(-1)
        halves.append(flat >> 32)                   # signed high half
        halves.append(flat & np.int64(0xFFFFFFFF))  # unsigned low half
    t = torch.from_numpy(np.concatenate(halves)).clone()
    if _device_backend(group):
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    summed = t.cpu().numpy()
    out, offset, bad = [], 0, False
    for shape in shapes:
        n = int(np.prod(shape))
        high = summed[offset: offset + n]
        low = summed[offset + n: offset + 2 * n]
        offset += 2 * n
        high = high + (low >> 32)                   # carry of the low sums
        low = low & np.int64(0xFFFFFFFF)
        bad = bad or bool(np.any((high < -(1 << 31)) | (high >= (1 << 31))))
        out.append(((high << 32) | low).reshape(shape))
    if bad:
        raise OverflowError("cooperative fixed-point accumulation overflow")
    return tuple(out)


def gather_antenna_shards(traces: np.ndarray, observers: np.ndarray, group=None) -> np.ndarray:
    """Reassembles (3, total bins) traces from each rank's (3, its bins) shard
    (rank order = antenna order); every rank gets the whole."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    bins = np.asarray(observers["number_of_bins"], dtype=np.int64)
    widths = []
    for r in range(world):
        b, e = antenna_shard(observers, r, world)
        widths.append(int(bins[b:e].sum()))
    local = torch.from_numpy(np.ascontiguousarray(traces)).reshape(3, -1)
    if local.shape[1] != widths[dist.get_rank(group)]:
        raise ValueError("local shard width does not match the antenna shard")
    widest = max(widths) if widths else 0
    padded = torch.zeros((3, widest), dtype=local.dtype)
    padded[:, : local.shape[1]] = local
    if _device_backend(group):
        padded = padded.cuda()
    parts = [torch.zeros_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return np.concatenate([p.cpu().numpy()[:, :w] for p, w in zip(parts, widths)], axis=1)


def max_over_ranks(value: float, group=None) -> float:
    """Largest value over ranks (device times: the job is as slow as its slowest rank)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64)
    if _device_backend(group):
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def _device_backend(group) -> bool:
    import torch.distributed as dist

    return dist.get_backend(group) == "nccl"
