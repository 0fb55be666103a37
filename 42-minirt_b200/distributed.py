"""Multi-GPU plumbing for the path tracer: one process per GPU.

The reference's only parallelism beyond one device is its TCP sample farm
(src/network: clients render the full frame at their own sample counts and
the server sums their float frames, handle_client.c:67-75). Here the same
sample-parallel decomposition runs as one process per GPU with
torch.distributed (NCCL on GPUs, gloo on CPU for tests):

  * shard_samples: every rank renders a contiguous range of sample indices.
    Paths draw from counter-based streams keyed by (seed, pixel, sample), so
    the union over ranks is exactly the single-GPU render, up to the order of
    the final floating-point sum.
  * reduce_frame: one sum-reduce of the W*H*3 accumulators to rank 0 — the
    only collective of a render.
  * partition_scenes: for multi-scene batches, scenes are owned by ranks
    (longest-processing-time bin packing on predicted cost); no collective.
  * allgather_photons: the kNN caustic estimate is not linear in the photon
    set, so each rank gathers every rank's photons into its own memory
    before building its grid (fixed-radius mode needs no gather: per-rank
    partial radiances add up).
Scenes are replicated: each rank uploads the host scene to its own GPU.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_samples(total_spp: int, world: int, rank: int, sample_base: int = 0) -> tuple[int, int]:
    """(first sample index, sample count) of `rank`: contiguous, balanced
    to within one sample, covering [sample_base, sample_base + total_spp)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if total_spp < 0:
        raise ValueError("negative sample count")
    q, r = divmod(total_spp, world)
    count = q + (1 if rank < r else 0)
    first = sample_base + rank * q + min(rank, r)
    return first, count


def partition_scenes(costs: list[float], world: int) -> list[list[int]]:
    """LPT bin packing: scene indices per rank, largest predicted cost first
    onto the least-loaded rank."""
    if world <= 0:
        raise ValueError("world must be positive")
    bins = [(0.0, r) for r in range(world)]
    heapq.heapify(bins)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        load, r = heapq.heappop(bins)
        out[r].append(i)
        heapq.heappush(bins, (load + float(costs[i]), r))
    return out


def scene_cost(width: int, height: int, spp: int, depth: int, n_prims: int) -> float:
    """Predicted cost of a render: paths x depth x BVH depth."""
    return float(width) * height * spp * depth * np.log2(2.0 + n_prims)


def reduce_frame(frame, dist, dst: int = 0):
    """Sum a float accumulator tensor (any device) onto rank `dst`."""
    dist.reduce(frame, dst=dst, op=dist.ReduceOp.SUM)
    return frame


def allgather_photons(pos: np.ndarray, power: np.ndarray, dist, device="cpu"):
    """All ranks' photons (rank order), as numpy float64 (n, 3) arrays."""
    import torch
    world = dist.get_world_size()
    n = torch.tensor([len(pos)], dtype=torch.int64, device=device)
    sizes = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    cap = max(sizes) if sizes else 0
    buf = torch.zeros((cap, 6), dtype=torch.float64, device=device)
    if len(pos):
        buf[: len(pos)] = torch.from_numpy(np.concatenate([pos, power], 1)).to(device)
    outs = [torch.zeros((cap, 6), dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(outs, buf)
    allp = np.concatenate([o[:k].cpu().numpy() for o, k in zip(outs, sizes)], 0)
    return allp[:, :3], allp[:, 3:]
