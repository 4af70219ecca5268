"""CUDA projectors against the reference's golden outputs and the oracle.

Parallel- and cone-beam forward and back projection are expected to equal
the reference bit for bit (same walk decisions, same float rounding and
summation order).  The one exception is the cone back projector for columns
taller than 1024 voxels, which accumulates with shared-memory atomics in
unspecified order and must agree to the projector tolerance,
max|new - ref| / max|ref| <= 1e-5.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden, max_rel, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def plan_from(d, kind):
    from ccpi.reconstruction.device import Plan
    shape = tuple(int(s) for s in d["shape"])
    if kind == 0:
        return Plan("parallel", d["angles"], d["h"], d["v"], tuple(d["origin"]),
                    tuple(d["size"]), shape)
    return Plan("cone", d["angles"], d["h"], d["v"], tuple(d["origin"]), tuple(d["size"]),
                shape, source=tuple(d["source"]), detector_x=float(d["detector_x"]))


def run(plan, fn, arr, cuda):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr, np.float32)).to(cuda)
    out = getattr(plan, fn)(t)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["pb0", "pb1", "pb2"])
def test_parallel_bit_exact_vs_reference(name, cuda):
    d = golden(name)
    p = plan_from(d, 0)
    fp = run(p, "forward", d["vol"], cuda)
    bp = run(p, "backward", d["pix"], cuda)
    assert np.array_equal(fp, d["fp"]), max_rel(fp, d["fp"])
    assert np.array_equal(bp, d["bp"]), max_rel(bp, d["bp"])


@pytest.mark.parametrize("name", ["cb0", "cb1"])
def test_cone_vs_reference(name, cuda):
    d = golden(name)
    p = plan_from(d, 1)
    fp = run(p, "forward", d["vol"], cuda)
    bp = run(p, "backward", d["pix"], cuda)
    assert np.array_equal(fp, d["fp"]), max_rel(fp, d["fp"])
    assert np.array_equal(bp, d["bp"]), max_rel(bp, d["bp"])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_parallel_random_geometries_vs_oracle(seed, cuda):
    from ccpi.reconstruction.device import Plan
    rng = np.random.default_rng(seed)
    nx, ny = rng.integers(8, 70, 2)
    nz = int(rng.choice([1, 3, 4, 8, 12, 36]))
    na, nh = int(rng.integers(1, 60)), int(rng.integers(2, 100))
    g = O.parallel_geometry((int(nx), int(ny), nz), na, nh, cor_shift=float(rng.uniform(-1, 1)),
                            span=float(rng.choice([np.pi, 2 * np.pi])))
    p = Plan("parallel", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape)
    vol = rng.random(g.shape).astype(np.float32)
    pix = rng.random(g.sino_shape).astype(np.float32)
    assert np.array_equal(run(p, "forward", vol, cuda), O.forward(g, vol))
    assert np.array_equal(run(p, "backward", pix, cuda), O.backward(g, pix))


def test_parallel_two_rows_per_slice_vs_oracle(cuda):
    from ccpi.reconstruction.device import Plan
    rng = np.random.default_rng(5)
    g = O.parallel_geometry((20, 20, 4), 17, 24, nv=8)
    g.size = (1.0, 1.0, 2.0)
    g.origin = (-10.0, -10.0, -4.0)
    p = Plan("parallel", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape)
    vol = rng.random(g.shape).astype(np.float32)
    pix = rng.random(g.sino_shape).astype(np.float32)
    assert np.array_equal(run(p, "forward", vol, cuda), O.forward(g, vol))
    assert np.array_equal(run(p, "backward", pix, cuda), O.backward(g, pix))


@pytest.mark.parametrize("seed", [0, 1])
def test_cone_random_geometries_vs_oracle(seed, cuda):
    from ccpi.reconstruction.device import Plan
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(8, 24))
    g = O.cone_geometry(n, 1.0, int(rng.integers(4, 40)), int(rng.integers(8, 40)), 0.8,
                        50.0, 50.0)
    p = Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
             source=g.source, detector_x=g.detector_x)
    vol = rng.random(g.shape).astype(np.float32)
    pix = rng.random(g.sino_shape).astype(np.float32)
    # an odd detector puts a row exactly at the source height, where the
    # reference's own arithmetic yields NaN (it reports "Oops"): same NaNs
    assert np.array_equal(run(p, "forward", vol, cuda), O.forward(g, vol), equal_nan=True)
    assert np.array_equal(run(p, "backward", pix, cuda), O.backward(g, pix), equal_nan=True)


def _off_centre_geometry(seed):
    """A half-circle cone scan with the source off the axis in y and z, a
    shifted detector and volume, and a column tall enough for the
    detector's magnified height (taller detectors make the reference read
    outside its arrays, which the tests avoid)."""
    import math
    rng = np.random.default_rng(500 + seed)
    nv = int(rng.integers(10, 40))
    nz = int(math.ceil(nv * 0.9 * 60.0 / 105.0)) + int(rng.integers(4, 10))
    g = O.cone_geometry((int(rng.integers(10, 24)), int(rng.integers(10, 24)), nz), 1.0,
                        int(rng.integers(6, 30)), int(rng.integers(12, 40)), 0.9, 60.0, 45.0,
                        full_circle=False, n_det_v=nv)
    g.source = (g.source[0], float(rng.uniform(-2, 2)), float(rng.uniform(-1.5, 1.5)))
    g.h_pixels = g.h_pixels + float(rng.uniform(-2, 2))
    g.v_pixels = g.v_pixels + float(rng.uniform(-1, 1))
    g.origin = (g.origin[0] + float(rng.uniform(-1, 1)), g.origin[1] + float(rng.uniform(-1, 1)),
                g.origin[2] + float(rng.uniform(-1, 1)))
    return g, rng


@pytest.mark.parametrize("seed", [0, 1, 3])
def test_cone_off_centre_source(seed, cuda):
    """Source off the axis in y and z, shifted detector and volume, a
    half-circle scan: the forward projector and the gather equal the oracle
    (which equals the reference built here on these seeds) bit for bit, and
    the scatter is within the projector tolerance."""
    from ccpi.reconstruction.device import Plan
    g, rng = _off_centre_geometry(seed)
    p = Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
             source=g.source, detector_x=g.detector_x)
    vol = rng.random(g.shape).astype(np.float32)
    pix = rng.random(g.sino_shape).astype(np.float32)
    assert np.array_equal(run(p, "forward", vol, cuda), O.forward(g, vol), equal_nan=True)
    ref = O.backward(g, pix)
    assert np.array_equal(run(p, "backward", pix, cuda), ref, equal_nan=True)
    p.set_cone_backprojector(1)
    assert _finite_max_rel(run(p, "backward", pix, cuda), ref) <= TOL


def test_cone_tall_columns_atomic_path(cuda):
    """Columns of more than 1024 voxels take the shared-atomic back
    projector: equal to the oracle within the projector tolerance."""
    from ccpi.reconstruction.device import Plan
    rng = np.random.default_rng(7)
    g = O.cone_geometry((4, 4, 1100), 1.0, 12, 16, 0.8, 50.0, 50.0, n_det_v=1100)
    p = Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
             source=g.source, detector_x=g.detector_x)
    pix = rng.random(g.sino_shape).astype(np.float32)
    b_gpu, b_ref = run(p, "backward", pix, cuda), O.backward(g, pix)
    ok = np.isfinite(b_ref)
    assert np.array_equal(np.isfinite(b_gpu), ok)
    assert max_rel(b_gpu[ok], b_ref[ok]) <= TOL
    # the ray-driven scatter has no column-height limit
    p.set_cone_backprojector(1)
    b_sc = run(p, "backward", pix, cuda)
    assert np.array_equal(np.isfinite(b_sc), ok)
    assert max_rel(b_sc[ok], b_ref[ok]) <= TOL


@pytest.mark.parametrize("kind", ["parallel", "cone"])
def test_dot_product_adjoint(kind, cuda):
    """<A x, y> = <x, A^T y> in FP64 sums (rel. error <= 1e-5)."""
    import torch
    from ccpi.reconstruction.device import parallel_plan, cone_plan
    if kind == "parallel":
        p = parallel_plan((48, 48, 8), 60, 64, cor_shift=0.25)
    else:
        p = cone_plan(32, 1.0, 48, 48, 1.0, 60.0, 60.0)
    g = torch.Generator(device="cpu").manual_seed(3)
    x = torch.rand(p.shape, generator=g).to(cuda)
    y = torch.rand(p.sino_shape, generator=g).to(cuda)
    ax = p.forward(x)
    aty = p.backward(y)
    lhs = (ax.double() * y.double()).sum().item()
    rhs = (x.double() * aty.double()).sum().item()
    assert abs(lhs - rhs) / abs(lhs) <= 1e-5


def test_linearity_full_size_parallel(cuda):
    """Config-2-sized parallel projector: A(2x) == 2 A(x) exactly and A^T
    likewise (scaling by 2 is exact in float)."""
    import torch
    from ccpi.reconstruction.device import parallel_plan
    p = parallel_plan((768, 768, 256), 720, 768)
    gen = torch.Generator(device="cuda").manual_seed(1)
    x = torch.rand(p.shape, device=cuda, generator=gen)
    a1 = p.forward(x)
    a2 = p.forward(2 * x)
    assert torch.equal(a2, 2 * a1)
    b1 = p.backward(a1)
    b2 = p.backward(a2)
    assert torch.equal(b2, 2 * b1)
    assert torch.isfinite(b1).all()


def test_create_phantom_like_reference_test(cuda):
    """conebeam.create_phantom returns what the reference's own test checks
    (Wrappers/Python/test/test_conebeam.py:17-27), with finite, non-negative
    projections of the three-cube phantom."""
    from ccpi.reconstruction.conebeam import alg
    data = alg.create_phantom()
    assert data[0].shape == (250, 512, 512)
    assert data[1].shape == (250,)
    assert data[2] == 250.0 and data[3] == 987.0
    assert data[4] == 0.390625 and data[5] == 0.390625
    assert data[6] == 25.151547886198443
    assert np.isfinite(data[0]).all() and data[0].min() >= 0.0 and data[0].max() > 0.0


def test_gather_probe_reports_a_bandwidth(cuda):
    """ccpi_measure_gather (the projectors' L2 gather ceiling that bench.py
    reports) runs and returns a plausible figure."""
    import ctypes

    import numpy as np
    import torch
    from ccpi.reconstruction import _native as N
    out = np.zeros(1, np.float64)
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    N.check(N.lib.ccpi_measure_gather(8 << 20, st, out), "ccpi_measure_gather")
    assert 100.0 < out[0] < 1e5
    assert N.lib.ccpi_measure_gather(16, st, out) == 1


def _finite_max_rel(got, ref):
    ok = np.isfinite(ref)
    assert np.array_equal(np.isfinite(got), ok)
    return max_rel(got[ok], ref[ok])


@pytest.mark.parametrize("case", ["cb0", "cb1", 0, 1, 2])
def test_cone_scatter_back_projector(case, cuda):
    """The ray-driven scatter form of the cone back projector (the forward
    walk transposed, warp-aggregated atomics) equals the reference's b2D
    (the fixtures) and the oracle (random geometries, an odd detector
    included) within the projector tolerance."""
    from ccpi.reconstruction.device import Plan
    if isinstance(case, str):
        d = golden(case)
        p = plan_from(d, 1)
        pix, ref = d["pix"], d["bp"]
    else:
        rng = np.random.default_rng(300 + case)
        n = int(rng.integers(8, 28))
        g = O.cone_geometry((n, n + 3, int(rng.integers(6, 40))), 1.0, int(rng.integers(4, 40)),
                            int(rng.integers(8, 41)), 0.8, 50.0, 50.0,
                            n_det_v=int(rng.integers(8, 41)))
        p = Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
                 source=g.source, detector_x=g.detector_x)
        pix = rng.random(g.sino_shape).astype(np.float32)
        ref = O.backward(g, pix)
    p.set_cone_backprojector(1)
    assert _finite_max_rel(run(p, "backward", pix, cuda), ref) <= TOL
    p.set_cone_backprojector(0)
    assert np.array_equal(run(p, "backward", pix, cuda), ref, equal_nan=True)


def test_cone_scatter_in_cgls(cuda):
    """CGLS with the scatter back projector (the pre-scaled residual, the
    FP64 norm of the scattered volume) agrees with the gather's CGLS to
    1e-5.  The TV-regularised CGLS amplifies float rounding: on this case
    the oracle's own FP32 solve is 7.5e-5 from its FP64 solve after 4
    iterations, so both back projectors are held against the FP64 solve and
    the scatter must come as close to it as the gather does."""
    import torch
    from ccpi.reconstruction.device import Plan
    g = O.cone_geometry(24, 1.0, 40, 36, 1.0, 60.0, 60.0, n_det_v=32)

    def mk():
        return Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
                    source=g.source, detector_x=g.detector_x)
    a, b = mk(), mk()
    b.set_cone_backprojector(1)
    rng = np.random.default_rng(8)
    x = torch.from_numpy(rng.random(a.shape).astype(np.float32)).to(cuda)
    s = a.forward(x)
    s64 = s.cpu().numpy().astype(np.float64)
    for alg, lam in ((0, 0.0), (4, 0.01)):
        xa = torch.zeros(a.shape, device=cuda)
        xb = torch.zeros(b.shape, device=cuda)
        _, na = a.solve(alg, s, xa, 4, regularize=lam, want_norms=True)
        _, nb = b.solve(alg, s, xb, 4, regularize=lam, want_norms=True)
        ga, gb = xa.cpu().numpy(), xb.cpu().numpy()
        if alg == 0:
            assert rel_l2(gb, ga) <= 1e-5
            assert max_rel(nb, na) <= 1e-5
        else:
            r64 = O.solve(g, alg, s64, 4, lam, fp64=True)
            r64 = r64[0] if isinstance(r64, tuple) else r64
            e_gather, e_scatter = rel_l2(ga, r64), rel_l2(gb, r64)
            assert e_scatter <= max(1e-4, 2.0 * e_gather), (e_scatter, e_gather)
