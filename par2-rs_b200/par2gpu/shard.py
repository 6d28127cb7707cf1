"""Multi-GPU sharding of the erasure-coding path: one process per GPU, no
collective on the data path.

Encode and repair are column-separable: the recovery (or rebuilt) bytes in
[a, b) depend only on the source bytes in [a, b) (par2-rs computes them chunk
by chunk for the same reason, par2_rs.rs:442-675).  So one set is split into
contiguous byte slabs, one per rank, aligned to the kernels' 2048-byte column
tile; independent sets are dealt to ranks whole.  The only collectives are
host-side bookkeeping: the max of the ranks' timings and, optionally, a gather
of the output slabs onto one rank.
"""
import numpy as np

TILE = 2048  # bytes per column tile of the multiply-accumulate kernels


def column_slabs(slice_bytes, world):
    """Contiguous [begin, end) byte ranges covering a slice, one per rank;
    every begin is a multiple of TILE, sizes differ by at most one tile.
    Ranks beyond the tile count get an empty range."""
    tiles = (slice_bytes + TILE - 1) // TILE
    out = []
    for r in range(world):
        t0 = tiles * r // world
        t1 = tiles * (r + 1) // world
        out.append((min(slice_bytes, t0 * TILE), min(slice_bytes, t1 * TILE)))
    return out


def rank_sets(nsets, rank, world):
    """Indices of the independent sets rank `rank` processes (round robin)."""
    return list(range(rank, nsets, world))


def max_over_ranks(value, device=None):
    """Max of a per-rank float over the default process group (the timing
    rule for multi-GPU numbers); the value itself without a group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_slabs(local, slab, slice_bytes, dst=0):
    """Assembles the ranks' output slabs on rank `dst`.  local: uint8 array
    [n, end - begin] of this rank's slab of n output slices; returns the
    [n, slice_bytes] array on dst and None elsewhere.  CPU tensors: gloo."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(), dist.get_rank()
    n = local.shape[0]
    slabs = column_slabs(slice_bytes, world)
    assert tuple(slab) == slabs[rank]
    width = max(b - a for a, b in slabs)
    buf = torch.zeros((n, width), dtype=torch.uint8)
    buf[:, : local.shape[1]] = torch.from_numpy(np.ascontiguousarray(local))
    parts = [torch.zeros_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, parts, dst=dst)
    if rank != dst:
        return None
    out = np.zeros((n, slice_bytes), np.uint8)
    for (a, b), p in zip(slabs, parts):
        out[:, a:b] = p[:, : b - a].numpy()
    return out
