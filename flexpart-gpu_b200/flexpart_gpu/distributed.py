"""Multi-GPU plumbing: one process per GPU over torch.distributed.

Particles are independent within a step and release scenarios are
independent entirely, so the path shards with no collective in the data
path: each rank steps its own particles (or scenarios) against a replicated
met bracket.  The one exchange is the sum of the concentration grids at
output times.  The grids are u32 counts and u32 fixed-point masses summed
with wrapping u32 atomics (concentration_gridding.wgsl:323-345), so the sum
over ranks taken modulo 2^32 is bit-identical to the grid one GPU computes
over the whole population, in any order.

Philox streams of different ranks must not overlap: rank r uses the
counter's top word r (the step advance only carries into it after 2^96
blocks).

An inversion whose instances are sharded across ranks exchanges one thing:
the wind-bias gradient, shared by every instance, summed once per backward
in fixed point (int64 at a common power-of-two scale) so that the sum does
not depend on the reduction order.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, world: int, rank: int):
    """Contiguous slot range [lo, hi) of rank `rank` out of `world` (sizes
    differ by at most one)."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_scenarios(counts, world: int):
    """Scenario indices per rank, balancing particle counts: largest first
    onto the least loaded rank (ties to the lower rank), each rank's list in
    ascending order.  Deterministic, so every rank computes the same
    assignment without communicating."""
    order = sorted(range(len(counts)), key=lambda s: (-int(counts[s]), s))
    load = [0] * world
    out = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(s)
        load[r] += int(counts[s])
    return [sorted(x) for x in out]


def rank_counter(counter, rank: int):
    """Initial Philox counter of rank `rank`: the caller's counter with the
    rank in the top word."""
    c = [int(x) & 0xFFFFFFFF for x in counter]
    c[3] = (c[3] + rank) & 0xFFFFFFFF
    return c


def allreduce_grids(counts: np.ndarray, mass_scaled: np.ndarray, group=None):
    """Sum of every rank's u32 grids, modulo 2^32 (host arrays; any backend)."""
    import torch
    import torch.distributed as dist

    out = []
    for a in (counts, mass_scaled):
        t = torch.from_numpy(np.ascontiguousarray(a, np.uint32).astype(np.int64))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out.append((t.numpy() & 0xFFFFFFFF).astype(np.uint32))
    return out[0], out[1]


class _CudaArray:
    """A device buffer owned by libfpg seen as a torch tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (int(ptr), False), "version": 3}


def allreduce_grids_device(counts_ptr: int, mass_ptr: int, n: int, group=None):
    """In-place sum over ranks of two u32 device grids of n cells (NCCL).
    They are summed as int32: two's-complement addition wraps exactly as the
    u32 sum does, so the bits are those of the u32 sum modulo 2^32."""
    import torch
    import torch.distributed as dist

    for ptr in (counts_ptr, mass_ptr):
        t = torch.as_tensor(_CudaArray(ptr, n), device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def _fixed_point_exponent(max_abs: float, world: int, bits: int = 62) -> int:
    """Power-of-two scale 2^e for the fixed-point sum: the largest e with
    world * max_abs * 2^e <= 2^bits, so no partial sum overflows int64."""
    if not (max_abs > 0.0) or not np.isfinite(max_abs):
        return 0
    return int(np.floor(np.log2(2.0 ** bits / (world * max_abs))))


def fixed_point_sum(arrays, bits: int = 62) -> np.ndarray:
    """The sum allreduce_gradient_fixed_point computes, in one process: each
    array rounded to int64 at the common power-of-two scale, the integers
    summed exactly, the total scaled back."""
    arrays = [np.asarray(a, np.float64) for a in arrays]
    e = _fixed_point_exponent(max(float(np.max(np.abs(a))) if a.size else 0.0 for a in arrays), len(arrays), bits)
    q = sum(np.rint(np.ldexp(a, e)).astype(np.int64) for a in arrays)
    return np.ldexp(q.astype(np.float64), -e)


def allreduce_gradient_fixed_point(grad: np.ndarray, group=None, bits: int = 62) -> np.ndarray:
    """Sum over ranks of a float gradient (the wind-bias gradient of an
    inversion whose instances are sharded across ranks) in fixed point:
    one MAX all-reduce fixes a common power-of-two scale, the rounded int64
    values are summed exactly, so the result does not depend on the ranks'
    reduction order and is bit-identical to fixed_point_sum of the ranks'
    gradients.  Host arrays; CUDA tensors when the group's backend is NCCL."""
    import torch
    import torch.distributed as dist

    g = np.asarray(grad, np.float64)
    world = dist.get_world_size(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    m = torch.tensor([float(np.max(np.abs(g))) if g.size else 0.0], dtype=torch.float64, device=dev)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    e = _fixed_point_exponent(float(m.item()), world, bits)
    q = torch.from_numpy(np.rint(np.ldexp(g, e)).astype(np.int64)).to(dev)
    dist.all_reduce(q, op=dist.ReduceOp.SUM, group=group)
    return np.ldexp(q.cpu().numpy().astype(np.float64), -e).reshape(np.shape(grad))


__all__ = ["shard_range", "shard_scenarios", "rank_counter", "allreduce_grids", "allreduce_grids_device",
           "fixed_point_sum", "allreduce_gradient_fixed_point"]
