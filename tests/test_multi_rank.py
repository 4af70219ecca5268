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
