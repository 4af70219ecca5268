"""Multi-rank host logic on CPU (gloo, world size 2).

The N-GPU bench gives every rank its own z-slab of a parallel-beam problem
and takes the maximum of the per-rank times.  These tests run two gloo
ranks on the host and check:
  * the slab split covers every slice exactly once;
  * the max-over-ranks reduction sees every rank's value;
  * SIRT on each rank's slab (solved here by the CPU oracle standing in for
    the GPU solver) equals that slab of the whole-volume solve, bit for
    bit, i.e. z-sharding needs no exchange step.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    sys.path[:0] = [os.path.join(ROOT, "ccpi-reconstruction_b200"), os.path.join(ROOT, "oracle")]
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from ccpi.reconstruction.distributed import barrier, max_over_ranks, slab_bounds
        import oracle as O
        nz = 6
        z0, z1 = slab_bounds(nz, world, rank)
        t = max_over_ranks(float(rank + 1) * 0.5)
        rng = np.random.default_rng(7)  # same problem on every rank
        g = O.parallel_geometry((20, 20, nz), 24, 30)
        x_true = rng.random(g.shape).astype(np.float32)
        sino = O.forward(g, x_true)
        gs = O.parallel_geometry((20, 20, z1 - z0), 24, 30)
        local = O.solve(gs, 1, np.ascontiguousarray(sino[:, :, z0:z1]), 4)
        barrier()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), z=np.array([z0, z1]), t=t,
                 local=local)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_slab_sirt(tmp_path):
    import oracle as O
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    zs = [tuple(p["z"]) for p in parts]
    assert zs[0][0] == 0 and zs[-1][1] == 6
    assert all(zs[i][1] == zs[i + 1][0] for i in range(world - 1))
    assert all(float(p["t"]) == 1.0 for p in parts)
    rng = np.random.default_rng(7)
    g = O.parallel_geometry((20, 20, 6), 24, 30)
    x_true = rng.random(g.shape).astype(np.float32)
    full = O.solve(g, 1, O.forward(g, x_true), 4)
    for p, (z0, z1) in zip(parts, zs):
        assert np.array_equal(p["local"], full[:, :, z0:z1])


@pytest.mark.parametrize("n,world,align", [(256, 2, 1), (257, 3, 1), (64, 8, 4), (5, 8, 1)])
def test_slab_bounds_partition(n, world, align):
    from ccpi.reconstruction.distributed import slab_bounds
    covered = []
    for r in range(world):
        z0, z1 = slab_bounds(n, world, r, align)
        assert 0 <= z0 <= z1 <= n
        if r < world - 1:
            assert (z1 - z0) % align == 0
        covered.extend(range(z0, z1))
    assert covered == list(range(n))


# ------------------------------------------------- z-sharded CGLS family
class OracleSlab:
    """One z slab of the staged CGLS family (the stages of
    ccpi_shard_stage, see include/ccpi_b200.h) in FP64 numpy with the
    oracle's projectors and regularisers.  Test infrastructure: it stands
    in for the GPU solver on gloo ranks, so that the protocol of
    ccpi.reconstruction.distributed (stage order, all-reduces, halo swaps)
    runs on the host."""

    def __init__(self, O, g, alg, sino, lam, has_lower, has_upper):
        import torch
        self.O, self.g, self.alg, self.lam = O, g, alg, lam
        self.b = np.asarray(sino, np.float64)
        self.x = np.zeros(g.shape)
        nx, ny, _ = g.shape
        self.sum = torch.zeros(1, dtype=torch.float64)
        self.edges = torch.zeros((2, nx, ny), dtype=torch.float64)
        self.halos = torch.zeros((2, nx, ny), dtype=torch.float64)
        self.has = (has_lower, has_upper)
        self.norms = []
        self.first = True

    def _edges(self, a):
        self.edges[0].copy_(torch_from(a[:, :, 0]))
        self.edges[1].copy_(torch_from(a[:, :, -1]))

    def _reg(self, a):
        parts = []
        if self.has[0]:
            parts.append(self.halos[0].numpy()[:, :, None])
        parts.append(a)
        if self.has[1]:
            parts.append(self.halos[1].numpy()[:, :, None])
        L = self.O.regularize(self.alg, np.concatenate(parts, axis=2), fp64=True)
        lo = 1 if self.has[0] else 0
        return L[:, :, lo:lo + a.shape[2]]

    def stage(self, k):
        import ccpi.reconstruction.distributed as D
        O, g, reg = self.O, self.g, self.alg != 0
        if k == D.SETUP:
            self.r = self.b.copy()
            self.d = O.backward(g, self.r, fp64=True)
            self.t = np.zeros(g.shape)
            self.sum[0] = float(np.sum(self.d * self.d))
            self._edges(self.d)
        elif k == D.FORWARD:
            if self.first:
                self.s0, self.first = float(self.sum[0]), False
            self.q = O.forward(g, self.d, fp64=True)
            tot = float(np.sum(self.q * self.q))
            if reg:
                self.t = self.t + self.lam * self._reg(self.d)
                tot += float(np.sum(self.t * self.t))
            self.sum[0] = tot
        elif k == D.UPDATE:
            tot = float(self.sum[0])
            self.alpha = self.s0 / tot if tot > 0 else 0.0
            self.r = self.r - self.alpha * self.q
            if reg:
                self.u = self.x + self.alpha * self.d
                self._edges(self.u)
        elif k == D.BACKWARD:
            if reg:
                self.x = self.u + self.lam * self._reg(self.u)
            self.s = O.backward(g, self.r, fp64=True)
            self.sum[0] = float(np.sum(self.s * self.s))
        elif k == D.NEXT:
            tot = float(self.sum[0])
            beta = tot / self.s0 if self.s0 > 0 else 0.0
            self.s0 = tot
            self.norms.append(np.sqrt(tot))
            if not reg:
                self.x = self.x + self.alpha * self.d
            self.d = self.s + beta * self.d
            if reg:
                self._edges(self.d)

    def finish(self):
        self.x = np.maximum(self.x, 0.0)
        return np.array(self.norms)


def torch_from(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a))


def slab_geometry(O, g, z0, z1):
    """The geometry of slices [z0, z1) of a unit-voxel parallel geometry
    whose rows map one to one onto slices."""
    nx, ny, _ = g.shape
    return O.Geometry(0, g.angles, g.h_pixels, g.v_pixels[z0:z1],
                      (g.origin[0], g.origin[1], g.origin[2] + z0), g.size, (nx, ny, z1 - z0))


SHARD_CASE = dict(shape=(22, 22, 9), na=26, nh=34, niter=5)


def _shard_worker(rank, world, port, out_dir, alg, lam):
    sys.path[:0] = [os.path.join(ROOT, "ccpi-reconstruction_b200"), os.path.join(ROOT, "oracle")]
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import oracle as O
        from ccpi.reconstruction import distributed as D
        c = SHARD_CASE
        g = O.parallel_geometry(c["shape"], c["na"], c["nh"])
        rng = np.random.default_rng(13)  # the same problem on every rank
        sino = O.forward(g, rng.random(g.shape).astype(np.float32)).astype(np.float64)
        sino += rng.normal(0.0, 0.05, sino.shape)
        z0, z1 = D.slab_bounds(c["shape"][2], world, rank)
        slab = OracleSlab(O, slab_geometry(O, g, z0, z1), alg, sino[:, :, z0:z1], lam,
                          rank > 0, rank < world - 1)
        (norms,) = D.run_slabs([slab], D.SlabComm(), c["niter"], tv=(alg == 4))
        np.savez(os.path.join(out_dir, f"shard{rank}.npz"), z=np.array([z0, z1]), x=slab.x,
                 norms=norms)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("alg,lam,world", [(0, 0.0, 2), (3, 0.02, 2), (4, 0.02, 2),
                                           (4, 0.02, 3)])
def test_gloo_ranks_sharded_cgls_family(alg, lam, world, tmp_path):
    """CGLS, CGLS-Tikhonov and CGLS-TV on a volume cut into z slabs over
    gloo ranks (the all-reduce of the step-scalar sums, and for TV the halo
    swap) equal the unsharded FP64 solve of the oracle to FP64 rounding."""
    import oracle as O
    mp.start_processes(_shard_worker, args=(world, _free_port(), str(tmp_path), alg, lam),
                       nprocs=world, join=True, start_method="spawn")
    c = SHARD_CASE
    g = O.parallel_geometry(c["shape"], c["na"], c["nh"])
    rng = np.random.default_rng(13)
    sino = O.forward(g, rng.random(g.shape).astype(np.float32)).astype(np.float64)
    sino += rng.normal(0.0, 0.05, sino.shape)
    full, norms = O.solve(g, alg, sino, c["niter"], lam=lam, fp64=True, want_norms=True)
    got = np.zeros(g.shape)
    for r in range(world):
        p = np.load(tmp_path / f"shard{r}.npz")
        z0, z1 = p["z"]
        got[:, :, z0:z1] = p["x"]
        assert np.allclose(p["norms"], norms, rtol=1e-12, atol=0)
    err = np.linalg.norm(got - full) / np.linalg.norm(full)
    assert err <= 1e-12, err
