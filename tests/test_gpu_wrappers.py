"""The projector-only calls and the real residual norms, through the numpy
API, against the reference.

* parallelbeam.alg.pb_forward_project / pb_backward_project
  (diamond_wrapper.cpp:421-556, :633-757): bit for bit against the
  reference's fixture and against the reference on fresh shapes, pixels per
  voxel 1 and 2.
* conebeam.alg.create_sinogram (conebeam_wrapper.cpp:346-400): bit for bit
  against the reference's cone_beam::f2D on the same float-rounded
  geometry.
* cgls_conv with real_norms=True: the per-iteration |A^T r| (the residual
  norm cgls.cpp:20-24 would report) against the FP64 oracle's, for parallel
  and cone beam; by default norm_r keeps the reference's zero fill.
"""
import numpy as np
import pytest

import configs as C
import oracle as O
from conftest import golden, max_rel, rel_l2

pytestmark = pytest.mark.gpu


def test_pb_projectors_fixture(cuda):
    from ccpi.reconstruction.parallelbeam import alg
    d = golden("pb_wrappers")
    fp = alg.pb_forward_project(d["vol"], d["angles"], 1)
    assert fp.shape == d["fp"].shape and np.array_equal(fp, d["fp"])
    bp = alg.pb_backward_project(d["stack"], d["angles"], 0.0, 1)
    assert bp.shape == d["bp"].shape and np.array_equal(bp, d["bp"])


@pytest.mark.parametrize("shape,na,ppv", [((30, 22, 12), 25, 1), ((18, 26, 10), 19, 2),
                                          ((16, 16, 8), 40, 1)])
def test_pb_forward_project_vs_reference(shape, na, ppv, cuda):
    if not O.reference_available():
        pytest.skip("oracle/_ref/libccpi_ref.so not built")
    from ccpi.reconstruction.parallelbeam import alg
    rng = np.random.default_rng(sum(shape) + na)
    vol = rng.random(shape).astype(np.float32)
    ang = np.sort(rng.uniform(0.0, 180.0, na)).astype(np.float32)
    got = alg.pb_forward_project(vol, ang, ppv)
    ref = O.ref_pb_forward_project(vol, ang, ppv)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), max_rel(got, ref)


def test_pb_forward_project_padded_rows(cuda):
    """A volume whose height is not a multiple of the row alignment: the
    detector gets padding rows (instruments.cpp:35-64) that map to slices
    outside the volume.  The reference then reads outside the voxel column
    (the neighbouring column's voxels, or memory outside the volume at the
    array's ends; p2D.cpp:63-213 has no bound check); this library projects
    nothing there.  Rows that map into the volume equal the reference bit
    for bit, padding rows are zero."""
    if not O.reference_available():
        pytest.skip("oracle/_ref/libccpi_ref.so not built")
    from ccpi.reconstruction.parallelbeam import alg
    rng = np.random.default_rng(61)
    vol = rng.random((16, 16, 5)).astype(np.float32)
    ang = np.sort(rng.uniform(0.0, 180.0, 40)).astype(np.float32)
    got = alg.pb_forward_project(vol, ang, 1)
    ref = O.ref_pb_forward_project(vol, ang, 1)
    assert got.shape == ref.shape == (40, 8, 16)
    nvp, voff = O.v_alignment(5, 1)
    assert (nvp, voff) == (8, 1)
    inside = slice(voff, voff + 5)
    assert np.array_equal(got[:, inside, :], ref[:, inside, :])
    assert not got[:, :voff, :].any() and not got[:, voff + 5:, :].any()


@pytest.mark.parametrize("na,nv,nh,cor,ppv", [(21, 8, 30, 0.0, 1), (17, 6, 27, 14.75, 1),
                                              (24, 12, 32, 0.0, 2)])
def test_pb_backward_project_vs_reference(na, nv, nh, cor, ppv, cuda):
    if not O.reference_available():
        pytest.skip("oracle/_ref/libccpi_ref.so not built")
    from ccpi.reconstruction.parallelbeam import alg
    rng = np.random.default_rng(na * nh + nv)
    stack = rng.random((na, nv, nh)).astype(np.float32)
    ang = np.linspace(0.0, 180.0, na, endpoint=False).astype(np.float32)
    got = alg.pb_backward_project(stack, ang, cor, ppv)
    ref = O.ref_pb_backward_project(stack, ang, cor, ppv)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), max_rel(got, ref)


@pytest.mark.parametrize("name", ["cb0", "cb1"])
def test_create_sinogram_vs_reference(name, cuda):
    """create_sinogram reads every geometry value as float32, as the
    reference's wrapper does; the reference's f2D on those same values is
    the expected result."""
    if not O.reference_available():
        pytest.skip("oracle/_ref/libccpi_ref.so not built")
    from ccpi.reconstruction.conebeam import alg
    d = golden(name)
    f = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    got = alg.create_sinogram(*[np.float32(x) for x in d["source"]], np.float32(d["detector_x"]),
                              d["h"].astype(np.float32), d["v"].astype(np.float32),
                              d["angles"].astype(np.float32), d["vol"],
                              d["origin"].astype(np.float32), d["size"].astype(np.float32))
    g = O.Geometry(1, f(d["angles"]), f(d["h"]), f(d["v"]), tuple(f(d["origin"])),
                   tuple(f(d["size"])), tuple(int(x) for x in d["shape"]),
                   source=tuple(f(d["source"])), detector_x=float(f(d["detector_x"])))
    ref = O.ref_forward(g, d["vol"])
    assert got.shape == ref.shape
    assert np.array_equal(got, ref, equal_nan=True)


def test_parallel_cgls_conv_real_norms(cuda):
    from ccpi.reconstruction.parallelbeam import alg
    d = golden("api_alg0_cor18.25_ppv1")
    niter = 4
    pix, ang, cor = d["pixels"], d["angles"], float(d["cor"])
    nr = np.zeros(niter)
    alg.cgls_conv(pix, ang, cor, 1, niter, 1, nr, bool(d["is_log"]), real_norms=True)
    na, nv, nh = pix.shape
    g, nvp, voff = O.parallel_api_geometry(na, nv, nh, ang, cor, 1)
    sino = O.parallel_api_sinogram(pix, nvp, voff, bool(d["is_log"]))
    _, n64 = O.solve(g, 0, sino.astype(np.float64), niter, fp64=True, want_norms=True)
    assert np.all(nr > 0)
    assert max_rel(nr, n64) <= 1e-5, (nr, n64)
    # the reference's behaviour by default: a non-zero norm_r is zero-filled
    nz = np.ones(niter)
    alg.cgls_conv(pix, ang, cor, 1, niter, 1, nz, bool(d["is_log"]))
    assert np.all(nz == 0)


def test_cone_cgls_norms_vs_fp64(cuda):
    import torch
    from ccpi.reconstruction.conebeam import alg
    from ccpi.reconstruction.device import Plan
    g, s = C.cone_case()
    p = Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
             source=g.source, detector_x=g.detector_x)
    niter = 4
    x = torch.zeros(p.shape, device=cuda)
    _, norms = p.solve(0, torch.from_numpy(s).to(cuda), x, niter, want_norms=True)
    x64, n64 = O.solve(g, 0, s.astype(np.float64), niter, fp64=True, want_norms=True)
    assert max_rel(norms, n64) <= 1e-5, (norms, n64)
    assert rel_l2(x.cpu().numpy(), x64) <= 1e-4
    # the numpy path: real norms on request, zero fill otherwise
    d = golden("cb_centre")
    args = (d["sino"], d["angles"], np.zeros(1), np.zeros(1), 1, float(d["s2s"]), float(d["s2d"]),
            float(d["px"]), float(d["px"]), float(d["mask_radius"]), False,
            np.zeros(3, np.float32), np.zeros(3, np.float32), 3, 1)
    nr = np.zeros(3)
    rec = alg.cgls_conv(*args, nr, True, real_norms=True)
    assert np.all(nr > 0) and np.all(np.isfinite(rec))
    nz = np.ones(3)
    alg.cgls_conv(*args, nz, True)
    assert np.all(nz == 0)


@pytest.mark.parametrize("algorithm", ["cgls", "sirt"])
def test_reconstruct_explicit_scatter_flag(algorithm, cuda):
    """ccpi_reconstruct_flags with CCPI_RECON_CONE_SCATTER: CGLS back-projects
    with the ray-driven scatter and agrees with the default (gather) solve to
    1e-5 rel-L2 after 4 iterations; SIRT always uses the gather and is
    unchanged bit for bit; unknown flag bits are an error."""
    import ctypes

    from ccpi.reconstruction import _native as N
    from ccpi.reconstruction.conebeam import alg as A
    g, s = C.cone_case()
    args = (algorithm, g.source, g.detector_x, g.h_pixels, g.v_pixels, g.angles, s, g.origin,
            g.size, g.shape, 4)
    base = A.reconstruct_explicit(*args)
    fast = A.reconstruct_explicit(*args, backprojector="scatter")
    if algorithm == "sirt":
        assert np.array_equal(fast, base)
    else:
        assert rel_l2(fast, base) <= 1e-5
    with pytest.raises(ValueError):
        A.reconstruct_explicit(*args, backprojector="bogus")
    geo = N.Geometry()
    out = np.zeros(3, np.float32)
    assert N.lib.ccpi_reconstruct_flags(ctypes.byref(geo), 0, out.ctypes.data, 1, 0.0, None,
                                        out.ctypes.data, 2) == 1
    assert b"unknown flag" in N.lib.ccpi_last_error()


@pytest.mark.parametrize("algorithm,alg,lam", [("cgls", 0, 0.0), ("sirt", 1, 0.0),
                                               ("cgls_TVreg", 4, 0.01)])
def test_reconstruct_explicit_equals_device_solve(algorithm, alg, lam, cuda):
    """ccpi_reconstruct (host buffers, explicit geometry) gives the device
    solver's result bit for bit, and SIRT the reference's."""
    import torch
    from ccpi.reconstruction.conebeam import alg as A
    from ccpi.reconstruction.device import Plan
    g, s = C.cone_case()
    niter = 4
    nr = np.zeros(niter)
    got = A.reconstruct_explicit(algorithm, g.source, g.detector_x, g.h_pixels, g.v_pixels,
                                 g.angles, s, g.origin, g.size, g.shape, niter, lam, nr)
    p = Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
             source=g.source, detector_x=g.detector_x)
    x = torch.zeros(p.shape, device=cuda)
    _, norms = p.solve(alg, torch.from_numpy(s).to(cuda), x, niter, regularize=lam,
                       want_norms=True)
    assert np.array_equal(got, x.cpu().numpy())
    if alg != 1:
        assert np.array_equal(nr, norms)
    else:
        assert np.array_equal(got, O.solve(g, 1, s, niter))
