"""The z-sharded CGLS family on the GPU (ccpi_shard_*, driven by
ccpi.reconstruction.distributed.run_slabs).

Every run here has one GPU, so the slabs of a volume are driven by one
process with LocalComm (the all-reduce a sum over the slabs, the halo swap a
copy); the stages and kernels are those a rank per GPU runs with SlabComm
over NCCL.  One slab without halos must equal ccpi_solve bit for bit; three
slabs must equal the whole-volume solve to the FP64 rounding of the sums'
order (the step scalars' sums are added per slab first).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _slab_plan(p, z0, z1):
    from ccpi.reconstruction.device import Plan
    ang, h, v = p._arrays
    g = p.geometry
    return Plan("parallel", ang, h, v[z0:z1], (g.origin[0], g.origin[1], g.origin[2] + z0),
                tuple(g.voxel_size), (p.shape[0], p.shape[1], z1 - z0))


@pytest.mark.parametrize("alg,lam", [(0, 0.0), (3, 0.02), (4, 0.02)])
def test_device_slabs_equal_whole_volume(alg, lam, cuda):
    import torch
    from ccpi.reconstruction import distributed as D
    from ccpi.reconstruction.device import parallel_plan
    niter = 6
    p = parallel_plan((40, 40, 12), 48, 60)
    rng = np.random.default_rng(5 + alg)
    sino = p.forward(torch.from_numpy(rng.random(p.shape).astype(np.float32)).to(cuda))
    sino += 0.05 * torch.from_numpy(rng.standard_normal(p.sino_shape).astype(np.float32)).to(cuda)
    ref = torch.zeros(p.shape, device=cuda)
    _, ref_norms = p.solve(alg, sino, ref, niter, regularize=lam, want_norms=True)
    # one slab: the whole volume, no exchange partner
    x1 = torch.zeros(p.shape, device=cuda)
    s1 = D.DeviceSlab(p, alg, sino, x1, niter, lam)
    (n1,) = D.run_slabs([s1], D.LocalComm(), niter, tv=(alg == 4))
    s1.close()
    assert torch.equal(x1, ref)
    assert np.array_equal(n1, ref_norms)
    # three slabs of uneven heights
    bounds = [(0, 4), (4, 7), (7, 12)]
    keep, slabs = [], []
    for i, (z0, z1) in enumerate(bounds):
        ps = _slab_plan(p, z0, z1)
        ss = sino[:, :, z0:z1].contiguous()
        xs = torch.zeros(ps.shape, device=cuda)
        keep.append((ps, ss, xs))
        slabs.append(D.DeviceSlab(ps, alg, ss, xs, niter, lam, has_lower=i > 0,
                                  has_upper=i < len(bounds) - 1))
    norms = D.run_slabs(slabs, D.LocalComm(), niter, tv=(alg == 4))
    got = torch.cat([k[2] for k in keep], dim=2)
    for s in slabs:
        s.close()
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-5
    for n in norms:
        assert rel_l2(n, ref_norms) <= 1e-6


def test_shard_stage_order_is_checked(cuda):
    import ctypes

    import torch
    from ccpi.reconstruction import _native as N
    from ccpi.reconstruction import distributed as D
    from ccpi.reconstruction.device import parallel_plan
    p = parallel_plan((16, 16, 4), 12, 24)
    sino = torch.zeros(p.sino_shape, device=cuda)
    x = torch.zeros(p.shape, device=cuda)
    s = D.DeviceSlab(p, 0, sino, x, 2)
    with pytest.raises(RuntimeError, match="out of order"):
        s.stage(D.FORWARD)
    s.stage(D.SETUP)
    with pytest.raises(RuntimeError, match="out of order"):
        s.stage(D.BACKWARD)
    s.close()
    # SIRT and MLEM need no exchange and are refused
    h = ctypes.c_void_p()
    buf = torch.zeros(2 * 16 * 16, device=cuda)
    one = torch.zeros(1, dtype=torch.float64, device=cuda)
    rc = N.lib.ccpi_shard_create(p.handle, 1, ctypes.c_void_p(sino.data_ptr()),
                                 ctypes.c_void_p(x.data_ptr()), 0.0, 2,
                                 ctypes.c_void_p(one.data_ptr()), ctypes.c_void_p(buf.data_ptr()),
                                 None, None, None, ctypes.byref(h))
    assert rc != 0 and b"CGLS family" in N.lib.ccpi_last_error()
