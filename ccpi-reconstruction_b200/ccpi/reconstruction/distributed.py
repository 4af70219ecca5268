"""One process per GPU: z-slab sharding of parallel-beam problems.

Parallel-beam detector rows map to their own voxel slices (gen_mapping,
Core/src/p2D.cpp:22-61), which is how the reference splits a volume over
MPI ranks (Core/src/voxels.cpp:27-45).  SIRT and MLEM on a slab are
therefore exactly the slab of the whole solve: ranks exchange nothing on
the data path, and only timing uses a collective (the maximum over ranks).
Cone beam does not shard this way (rays cross every slab): N ranks run N
independent problems.

torch.distributed is plumbing here (process group, barrier, the timing
reduction); the work itself is the library's CUDA solver on each rank's
GPU.
"""
from __future__ import annotations


def slab_bounds(n_slices: int, world: int, rank: int, align: int = 1):
    """Slices [z0, z1) of `rank` when `n_slices` are split over `world`
    ranks in contiguous slabs whose sizes are multiples of `align` (the
    last slab takes the remainder); earlier ranks get the larger share."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    if align < 1 or n_slices < 0:
        raise ValueError("bad slab request")
    units = n_slices // align
    base, extra = divmod(units, world)
    z0 = align * (rank * base + min(rank, extra))
    z1 = align * ((rank + 1) * base + min(rank + 1, extra))
    if rank == world - 1:
        z1 = n_slices
    return z0, z1


def slab_rows(n_rows: int, rows_per_slice: int, z0: int, z1: int):
    """Detector rows [v0, v1) that map to slices [z0, z1) when every slice
    takes `rows_per_slice` consecutive rows (map types 1, 2 and 4)."""
    return z0 * rows_per_slice, min(z1 * rows_per_slice, n_rows)


def max_over_ranks(value: float, group=None, device=None) -> float:
    """Maximum of a per-rank float over the process group (the bench's
    timing rule); identity when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def barrier(group=None):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier(group=group)
