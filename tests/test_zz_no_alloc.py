"""ccpi_solve_noalloc (solver scratch in a static device area) against
ccpi_solve, called through the C ABI.

Two calls in a row on the same problem must each equal ccpi_solve's result
(rel-L2 <= 1e-6; the kernels and their order are the same, so in practice
the results are identical), and a problem whose workspace exceeds the
static scratch must be refused with a message naming the sizes.  This file
runs last so that it also runs after every other GPU test in one process.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _lib():
    from ccpi.reconstruction import _native as N
    f = N.lib.ccpi_solve_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double, vp, vp]
    f.restype = ctypes.c_int
    return N


@pytest.mark.parametrize("alg,lam", [(0, 0.0), (1, 0.0), (2, 0.0), (3, 0.01), (4, 0.005)])
def test_noalloc_matches_solve_twice(alg, lam, cuda):
    import torch
    from ccpi.reconstruction.device import parallel_plan
    N = _lib()
    p = parallel_plan((96, 96, 16), 120, 144)
    rng = np.random.default_rng(20 + alg)
    x_true = torch.from_numpy(rng.random(p.shape).astype(np.float32)).to(cuda)
    sino = p.forward(x_true)
    niter = 6
    ref = torch.zeros(p.shape, device=cuda)
    p.solve(alg, sino, ref, niter, regularize=lam)
    ref_np = ref.cpu().numpy()
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    for _ in range(2):
        x = torch.zeros(p.shape, device=cuda)
        norms = np.zeros(niter, np.float64)
        rc = N.lib.ccpi_solve_noalloc(p.handle, alg, ctypes.c_void_p(sino.data_ptr()),
                                      ctypes.c_void_p(x.data_ptr()), niter, lam,
                                      norms.ctypes.data, stream)
        assert rc == 0, N.lib.ccpi_last_error().decode()
        assert rel_l2(x.cpu().numpy(), ref_np) <= TOL


def test_noalloc_refuses_large_problem(cuda):
    import torch
    from ccpi.reconstruction.device import parallel_plan
    N = _lib()
    p = parallel_plan((256, 256, 64), 180, 384)
    need = p.workspace_bytes(0, 5)
    assert need > (16 << 20)
    sino = torch.zeros(p.sino_shape, device=cuda)
    x = torch.zeros(p.shape, device=cuda)
    rc = N.lib.ccpi_solve_noalloc(p.handle, 0, ctypes.c_void_p(sino.data_ptr()),
                                  ctypes.c_void_p(x.data_ptr()), 5, 0.0, None, None)
    assert rc != 0
    msg = N.lib.ccpi_last_error().decode()
    assert str(need) in msg and str(16 << 20) in msg
