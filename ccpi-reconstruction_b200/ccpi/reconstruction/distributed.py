"""One process per GPU: z-slab sharding of parallel-beam problems.

Parallel-beam detector rows map to their own voxel slices (gen_mapping,
Core/src/p2D.cpp:22-61), which is how the reference splits a volume over
MPI ranks (Core/src/voxels.cpp:27-45).  SIRT and MLEM on a slab are
therefore exactly the slab of the whole solve: ranks exchange nothing on
the data path, and only timing uses a collective (the maximum over ranks).
The CGLS family needs two FP64 sums over the whole volume per iteration
and, for TV, one z plane across each cut: run_slabs drives the library's
staged solver (ccpi_shard_*) with those exchanges (SlabComm: one slab per
rank over torch.distributed; LocalComm: several slabs in one process).
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


# ---------------------------------------------------------------------------
# z-sharded CGLS, CGLS-Tikhonov and CGLS-TV
#
# CGLS needs two sums over the whole volume per iteration (|A d|^2, plus
# |Ad_vox|^2 for the regularised forms, and |A^T r|^2: cgls.cpp:87-157,
# :343-423); TV's stencil reads one z plane beyond each cut (total_v.cpp:
# 95-101).  The library runs the iteration in stages (ccpi_shard_stage); this
# driver makes the exchange between stages: an all-reduce of one FP64 value
# and, for TV, a swap of edge planes into the neighbours' halo buffers.

SETUP, FORWARD, UPDATE, BACKWARD, NEXT = 0, 1, 2, 3, 4
_AFTER = {SETUP: ("reduce", "swap"), FORWARD: ("reduce",), UPDATE: ("swap",),
          BACKWARD: ("reduce",), NEXT: ("swap",)}


class SlabComm:
    """Exchanges between the slabs of one process group, one slab per rank
    (rank r holds slabs in z order).  `sum` is a 1-element float64 tensor,
    `edges` (2, nx, ny) and `halos` (2, nx, ny) float32 tensors on the
    rank's device (NCCL) or on the host (gloo)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def reduce(self, slabs):
        (s,) = slabs
        self.dist.all_reduce(s.sum, op=self.dist.ReduceOp.SUM, group=self.group)

    def swap(self, slabs):
        (s,) = slabs
        d, reqs = self.dist, []
        peer = lambda r: d.get_global_rank(self.group, r) if self.group is not None else r  # noqa
        if self.rank > 0:
            reqs.append(d.isend(s.edges[0].contiguous(), peer(self.rank - 1), group=self.group))
            reqs.append(d.irecv(s.halos[0], peer(self.rank - 1), group=self.group))
        if self.rank < self.world - 1:
            reqs.append(d.isend(s.edges[1].contiguous(), peer(self.rank + 1), group=self.group))
            reqs.append(d.irecv(s.halos[1], peer(self.rank + 1), group=self.group))
        for r in reqs:
            r.wait()


class LocalComm:
    """Exchanges between several slabs driven by one process (in z order):
    the all-reduce is a sum over the slabs, the swap a copy."""

    def reduce(self, slabs):
        total = slabs[0].sum.clone()
        for s in slabs[1:]:
            total += s.sum
        for s in slabs:
            s.sum.copy_(total)

    def swap(self, slabs):
        for i, s in enumerate(slabs):
            if i > 0:
                s.halos[0].copy_(slabs[i - 1].edges[1])
            if i + 1 < len(slabs):
                s.halos[1].copy_(slabs[i + 1].edges[0])


def run_slabs(slabs, comm, niterations, tv):
    """The staged CGLS-family protocol over `slabs` (objects with .stage(k),
    .finish(), and the .sum / .edges / .halos buffers of SlabComm)."""
    def stage(k):
        for s in slabs:
            s.stage(k)
        for what in _AFTER[k]:
            if what == "reduce":
                comm.reduce(slabs)
            elif tv:
                comm.swap(slabs)
    stage(SETUP)
    for _ in range(int(niterations)):
        for k in (FORWARD, UPDATE, BACKWARD, NEXT):
            stage(k)
    return [s.finish() for s in slabs]


class DeviceSlab:
    """One z slab on this process's GPU: the library's staged solver
    (ccpi_shard_*) on a slab plan, with its exchange buffers as torch
    tensors.  has_lower / has_upper: whether slabs exist below / above."""

    def __init__(self, plan, alg, sino, x, niterations, regularize=0.0, has_lower=False,
                 has_upper=False):
        import ctypes

        import torch

        from . import _native as N
        self._N = N
        dev = x.device
        nx, ny, _ = plan.shape
        self.sum = torch.zeros(1, dtype=torch.float64, device=dev)
        self.edges = torch.zeros((2, nx, ny), dtype=torch.float32, device=dev)
        self.halos = torch.zeros((2, nx, ny), dtype=torch.float32, device=dev)
        self.plan, self.sino, self.x = plan, sino, x
        vp = ctypes.c_void_p
        lo = vp(self.halos[0].data_ptr()) if has_lower else None
        hi = vp(self.halos[1].data_ptr()) if has_upper else None
        self._stream = vp(torch.cuda.current_stream(dev).cuda_stream)
        h = vp()
        N.check(N.lib.ccpi_shard_create(plan.handle, int(alg), vp(sino.data_ptr()),
                                        vp(x.data_ptr()), float(regularize), int(niterations),
                                        vp(self.sum.data_ptr()), vp(self.edges.data_ptr()), lo,
                                        hi, self._stream, ctypes.byref(h)),
                "ccpi_shard_create")
        self._h = h
        self.done = 0

    def stage(self, k):
        self._N.check(self._N.lib.ccpi_shard_stage(self._h, int(k)), "ccpi_shard_stage")
        if k == NEXT:
            self.done += 1

    def finish(self):
        import numpy as np
        norms = np.zeros(max(self.done, 1), np.float64)
        self._N.check(self._N.lib.ccpi_shard_finish(self._h, norms.ctypes.data),
                      "ccpi_shard_finish")
        return norms[:self.done]

    def close(self):
        if self._h:
            self._N.lib.ccpi_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
