"""Channel sharding across GPUs (one process per GPU).

Channels of DSPLIB_fir and DSPLIB_cascadeBiquad never interact
(src/DSPLIB_fir/DSPLIB_fir_cn.cpp:54, src/DSPLIB_cascadeBiquad/
DSPLIB_cascadeBiquad_cn.cpp:46), so a multi-GPU run gives each rank its own
block of channels and needs no collective on the data path.  Ranks only meet
to agree on timing (max over ranks) and, when a caller wants the full result on
one rank, to gather outputs.
"""
from __future__ import annotations

import heapq


def channel_block(rank: int, world: int, channels: int) -> tuple[int, int]:
    """Contiguous block [c0, c1) of ``channels`` owned by ``rank`` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(channels, world)
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


def balance_ragged(lengths, world: int) -> list[list[int]]:
    """Greedy longest-first assignment of ragged channels to ranks, minimising
    the largest per-rank total length.  Returns the channel indices per rank
    (each list in ascending order)."""
    order = sorted(range(len(lengths)), key=lambda i: -int(lengths[i]))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(lengths[i]), r))
    return [sorted(v) for v in out]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar (elapsed time) over all ranks; identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
