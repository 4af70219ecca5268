"""ccpi_solve_noalloc (solver scratch in a static device area) against
ccpi_solve, called through the C ABI.

Some callers cannot allocate device memory while they solve: a host that has
handed the whole device to its own memory pool, or a loop whose other
streams must not be stalled by the device-wide synchronisation of a
cudaMalloc/cudaFree pair.  For them the library has one entry point whose
solver workspace is a 16 MiB area compiled into the library.

Checks:
* two calls in a row on the same problem each equal ccpi_solve's result
  (rel-L2 <= 1e-6; the kernels and their order are the same, so in practice
  the results are identical), for a parallel-beam and a cone-beam plan and
  every algorithm;
* a call takes no device memory: the free device memory is the same before
  and after it, and with all but a few MiB of the device held by another
  allocation, ccpi_solve (which allocates its workspace) fails while
  ccpi_solve_noalloc still gives the same result;
* a problem whose workspace exceeds the static scratch is refused with a
  message naming both sizes.

This file runs last, so that it also runs after every other GPU test in one
process; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-6
SCRATCH = 16 << 20


def _lib():
    from ccpi.reconstruction import _native as N
    f = N.lib.ccpi_solve_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double, vp, vp]
    f.restype = ctypes.c_int
    return N


def _plan(kind, large=False):
    from ccpi.reconstruction.device import cone_plan, parallel_plan
    if kind == "parallel":
        return parallel_plan((128, 128, 32), 120, 192) if large else \
            parallel_plan((96, 96, 16), 120, 144)
    return cone_plan(64, 1.0, 90, 80, 1.0, 100.0, 100.0)


def _noalloc(N, p, alg, sino, x, niter, lam, norms, stream):
    return N.lib.ccpi_solve_noalloc(p.handle, alg, ctypes.c_void_p(sino.data_ptr()),
                                    ctypes.c_void_p(x.data_ptr()), niter, lam,
                                    None if norms is None else norms.ctypes.data, stream)


def _problem(kind, alg, cuda, large=False):
    import torch
    p = _plan(kind, large)
    rng = np.random.default_rng(20 + alg)
    x_true = torch.from_numpy(rng.random(p.shape).astype(np.float32)).to(cuda)
    return p, p.forward(x_true)


@pytest.mark.parametrize("kind", ["parallel", "cone"])
@pytest.mark.parametrize("alg,lam", [(0, 0.0), (1, 0.0), (2, 0.0), (3, 0.01), (4, 0.005)])
def test_noalloc_matches_solve_twice(kind, alg, lam, cuda):
    import torch
    N = _lib()
    p, sino = _problem(kind, alg, cuda)
    niter = 6
    assert p.workspace_bytes(alg, niter) <= SCRATCH
    ref = torch.zeros(p.shape, device=cuda)
    _, ref_norms = p.solve(alg, sino, ref, niter, regularize=lam, want_norms=True)
    ref_np = ref.cpu().numpy()
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    for _ in range(2):
        x = torch.zeros(p.shape, device=cuda)
        norms = np.zeros(niter, np.float64)
        rc = _noalloc(N, p, alg, sino, x, niter, lam, norms, stream)
        assert rc == 0, N.lib.ccpi_last_error().decode()
        assert rel_l2(x.cpu().numpy(), ref_np) <= TOL
        if alg in (0, 3, 4):
            assert rel_l2(norms, ref_norms) <= TOL


@pytest.mark.parametrize("kind", ["parallel", "cone"])
def test_noalloc_takes_no_device_memory(kind, cuda):
    import torch
    N = _lib()
    alg, niter, lam = 4, 4, 0.01
    p, sino = _problem(kind, alg, cuda, large=True)
    need = p.workspace_bytes(alg, niter)
    assert 8 << 20 <= need <= SCRATCH
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    ref = torch.zeros(p.shape, device=cuda)
    p.solve(alg, sino, ref, niter, regularize=lam)
    ref_np = ref.cpu().numpy()
    x = torch.zeros(p.shape, device=cuda)
    # a first call loads every kernel the solve uses
    assert _noalloc(N, p, alg, sino, x, niter, lam, None, stream) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(cuda)[0]
    x.zero_()
    assert _noalloc(N, p, alg, sino, x, niter, lam, None, stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(cuda)[0] == free0
    assert rel_l2(x.cpu().numpy(), ref_np) <= TOL
    # hold the free device memory but for half a workspace (plus < 2 MiB of
    # allocation granularity)
    hold = None
    try:
        free = torch.cuda.mem_get_info(cuda)[0]
        two_mib = 2 << 20
        hold = torch.empty(max((free - need // 2) // two_mib * two_mib, 0), dtype=torch.uint8,
                           device=cuda)
        assert torch.cuda.mem_get_info(cuda)[0] < need
        x.zero_()
        rc = N.lib.ccpi_solve(p.handle, alg, ctypes.c_void_p(sino.data_ptr()),
                              ctypes.c_void_p(x.data_ptr()), niter, lam, None, 0, None, 0,
                              stream)
        assert rc != 0, "ccpi_solve found room for its workspace"
        x.zero_()
        rc = _noalloc(N, p, alg, sino, x, niter, lam, None, stream)
        assert rc == 0, N.lib.ccpi_last_error().decode()
        assert rel_l2(x.cpu().numpy(), ref_np) <= TOL
    finally:
        del hold
        torch.cuda.empty_cache()


def test_noalloc_refuses_large_problem(cuda):
    import torch
    from ccpi.reconstruction.device import parallel_plan
    N = _lib()
    p = parallel_plan((256, 256, 64), 180, 384)
    need = p.workspace_bytes(0, 5)
    assert need > SCRATCH
    sino = torch.zeros(p.sino_shape, device=cuda)
    x = torch.zeros(p.shape, device=cuda)
    rc = N.lib.ccpi_solve_noalloc(p.handle, 0, ctypes.c_void_p(sino.data_ptr()),
                                  ctypes.c_void_p(x.data_ptr()), 5, 0.0, None, None)
    assert rc != 0
    msg = N.lib.ccpi_last_error().decode()
    assert str(need) in msg and str(SCRATCH) in msg
