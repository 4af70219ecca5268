"""Solvers through the reference-facing API against the reference's golden
reconstructions.

SIRT and MLEM use only bit-exact projectors and float updates in the
reference's order, so they are expected to equal the reference bit for bit.
The CGLS family computes its step scalars from FP64 inner products (the
reference sums them in float), so it is compared by relative L2 error
against the reference and against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden, golden_names, max_rel, rel_l2

pytestmark = pytest.mark.gpu


def api_call(d, x0=None):
    from ccpi.reconstruction.parallelbeam import alg
    fn = {0: "cgls", 1: "sirt", 2: "mlem", 3: "cgls_tikhonov", 4: "cgls_TVreg"}[int(d["alg"])]
    niter = int(d["niter"])
    args = (d["pixels"], d["angles"], float(d.get("cor", 0.0)), int(d.get("ppv", 1)), niter, 1)
    is_log = bool(d.get("is_log", 0))
    if x0 is not None:
        if fn in ("cgls", "sirt", "mlem"):
            return getattr(alg, fn + "_step")(*args, is_log, x0)
    if fn in ("cgls_tikhonov", "cgls_TVreg"):
        return getattr(alg, fn)(*args, float(d["lam"]), np.zeros(niter), is_log)
    return getattr(alg, fn)(*args, is_log)


@pytest.mark.parametrize("name", golden_names("api_"))
def test_parallel_api_vs_reference(name, cuda):
    d = golden(name)
    rec = api_call(d)
    ref = d["out"]
    assert rec.shape == ref.shape and rec.dtype == np.float32
    if int(d["alg"]) in (1, 2):
        assert np.array_equal(rec, ref), max_rel(rec, ref)
    else:
        # FP64 step scalars vs the reference's FP32 ones: compare with the
        # FP64 oracle (the accurate answer) and bound the distance to the
        # reference by the reference's own rounding error
        pix = d["pixels"]
        na, nv, nh = pix.shape
        g, nvp, voff = O.parallel_api_geometry(na, nv, nh, d["angles"], float(d["cor"]),
                                               int(d["ppv"]))
        sino = O.parallel_api_sinogram(pix, nvp, voff, bool(d["is_log"]))
        r64 = O.solve(g, int(d["alg"]), sino.astype(np.float64), int(d["niter"]),
                      lam=float(d["lam"]), fp64=True)
        e_gpu = rel_l2(rec, r64)
        e_ref = rel_l2(ref, r64)
        assert e_gpu <= 1e-4, (e_gpu, e_ref)
        assert rel_l2(rec, ref) <= max(1e-4, 2.0 * e_ref)


@pytest.mark.parametrize("name", golden_names("step_"))
def test_parallel_step_forms(name, cuda):
    d = golden(name)
    rec = api_call(d, x0=d["x0"])
    if int(d["alg"]) in (1, 2):
        assert np.array_equal(rec, d["out"])
    else:
        assert rel_l2(rec, d["out"]) <= 5e-4


@pytest.mark.parametrize("alg", [0, 1, 2, 3, 4])
def test_plain_and_graph_paths_agree(alg, cuda):
    import torch
    from ccpi.reconstruction.device import parallel_plan
    p = parallel_plan((40, 40, 8), 50, 44)
    rng = np.random.default_rng(alg)
    x_true = torch.from_numpy(rng.random(p.shape).astype(np.float32)).to(cuda)
    sino = p.forward(x_true)
    a = torch.zeros(p.shape, device=cuda)
    b = torch.zeros(p.shape, device=cuda)
    p.solve(alg, sino, a, 7, regularize=0.001)
    p.solve(alg, sino, b, 7, regularize=0.001, plain=True)
    assert torch.equal(a, b)


def test_batched_equals_individual(cuda):
    import torch
    from ccpi.reconstruction.device import parallel_plan, solve_batched
    rng = np.random.default_rng(9)
    plans, sinos, singles = [], [], []
    for i in range(5):
        n, nz, na = int(rng.integers(16, 48)), int(rng.choice([4, 8])), int(rng.integers(20, 70))
        p = parallel_plan((n, n, nz), na, int(1.5 * n))
        x = torch.from_numpy(rng.random(p.shape).astype(np.float32)).to(cuda)
        s = p.forward(x)
        y = torch.zeros(p.shape, device=cuda)
        p.solve(3, s, y, 6, regularize=0.002 * (i + 1))
        plans.append(p)
        sinos.append(s)
        singles.append(y)
    xs = [torch.zeros(p.shape, device=cuda) for p in plans]
    solve_batched(plans, 3, sinos, xs, 6, regularize=[0.002 * (i + 1) for i in range(5)])
    for a, b in zip(xs, singles):
        assert torch.equal(a, b)


def test_slices_batched_equal_per_slice(cuda):
    """SIRT on a 3-D parallel problem equals SIRT run slice by slice."""
    import torch
    from ccpi.reconstruction.device import parallel_plan
    rng = np.random.default_rng(11)
    p3 = parallel_plan((32, 32, 8), 40, 40)
    x = torch.from_numpy(rng.random(p3.shape).astype(np.float32)).to(cuda)
    s = p3.forward(x)
    full = torch.zeros(p3.shape, device=cuda)
    p3.solve(1, s, full, 5)
    p1 = parallel_plan((32, 32, 1), 40, 40)
    for k in range(8):
        sk = s[:, :, k:k + 1].contiguous()
        xk = torch.zeros(p1.shape, device=cuda)
        p1.solve(1, sk, xk, 5)
        assert torch.equal(xk[:, :, 0], full[:, :, k])


def test_cone_api_vs_reference(cuda):
    from ccpi.reconstruction.conebeam import alg
    d = golden("cb_centre")
    rec = alg.cgls(d["sino"], d["angles"], np.zeros(1), np.zeros(1), 1, float(d["s2s"]),
                   float(d["s2d"]), float(d["px"]), float(d["px"]), float(d["mask_radius"]),
                   False, np.zeros(3, np.float32), np.zeros(3, np.float32), 3, 1, True)
    assert rec.shape == d["cgls3"].shape
    assert rel_l2(rec, d["cgls3"]) <= 1e-4


def uneven_problems(n, niter_seed=4):
    """Seeded uneven CGLS-Tikhonov / CGLS-TV problems shaped like the
    64-problem batch (volume width w, detector columns round(1.5 w), angle
    counts and lambda log-uniform in [1e-3, 1e-1]), scaled down; sinograms
    are oracle projections of ellipse phantoms with 2% Gaussian noise."""
    seqs = np.random.SeedSequence(niter_seed).spawn(n)
    out = []
    for i, ss in enumerate(seqs):
        rng = np.random.default_rng(ss)
        w = int(rng.integers(16, 49))
        nz = int(rng.integers(4, 13))
        na = int(rng.integers(20, 91))
        nh = int(round(1.5 * w))
        lam = float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-1))))
        vol = np.zeros((w, w, nz), np.float32)
        c = np.arange(w) + 0.5 - w / 2
        X, Y = np.meshgrid(c, c, indexing="ij")
        for k in range(nz):
            for _ in range(4):
                cx, cy = rng.uniform(-0.3, 0.3, 2) * w
                ax, ay = rng.uniform(0.1, 0.3, 2) * w
                vol[:, :, k] += (((X - cx) / ax) ** 2 + ((Y - cy) / ay) ** 2 <= 1) * \
                    rng.uniform(0.1, 1.0)
        ang = np.linspace(0.0, 180.0, na, endpoint=False).astype(np.float32)
        g = O.parallel_geometry((w, w, nz), na, nh, nz)
        g.angles = np.pi * (ang.astype(np.float64) / 180.0)
        s = O.forward(g, vol)  # (na, nh, nv)
        s = s + rng.normal(0.0, 0.02 * np.abs(s).max(), s.shape).astype(np.float32)
        pixels = np.ascontiguousarray(s.transpose(0, 2, 1), np.float32)  # (na, nv, nh)
        out.append(dict(alg=3 + (i % 2), pixels=pixels, angles=ang, lam=lam))
    return out


def test_batched_api_uneven_vs_single_and_reference(cuda):
    """parallelbeam.alg.reconstruct_batched over uneven regularised problems
    equals the per-problem calls bit for bit, and each result is within the
    CGLS tolerance of the FP64 oracle and the reference's own solver.

    Four iterations: on these small noisy problems any FP32 CGLS (the
    reference's included) loses conjugacy after about five iterations and
    drifts 1e-4 to 1e-2 away from the FP64 iterates, so a longer run would
    measure FP32 itself rather than this implementation."""
    from ccpi.reconstruction.parallelbeam import alg
    niter = 4
    probs = uneven_problems(6)
    for algo in (3, 4):
        sel = [p for p in probs if p["alg"] == algo]
        name = "cgls_tikhonov" if algo == 3 else "cgls_TVreg"
        outs = alg.reconstruct_batched(name, [p["pixels"] for p in sel],
                                       [p["angles"] for p in sel], 0.0, 1, niter, 1, True,
                                       regularize=[p["lam"] for p in sel])
        for p, rec in zip(sel, outs):
            single = getattr(alg, name)(p["pixels"], p["angles"], 0.0, 1, niter, 1, p["lam"],
                                        np.zeros(niter), True)
            assert np.array_equal(rec, single)
            na, nv, nh = p["pixels"].shape
            g, nvp, voff = O.parallel_api_geometry(na, nv, nh, p["angles"], 0.0, 1)
            sino = O.parallel_api_sinogram(p["pixels"], nvp, voff, True)
            r64 = O.solve(g, algo, sino.astype(np.float64), niter, lam=p["lam"], fp64=True)
            ref = O.ref_pb_reconstruct(algo, p["pixels"], p["angles"], 0.0, 1, niter, True,
                                       lam=p["lam"])
            e_ref = rel_l2(ref, r64)
            assert rel_l2(rec, r64) <= 1e-4, (rel_l2(rec, r64), e_ref)
            assert rel_l2(rec, ref) <= max(1e-4, 2.0 * e_ref)


@pytest.mark.parametrize("alg", [1, 2, 0])
def test_device_api_plan_equals_host_call(alg, cuda):
    """parallel_api_plan + pack_parallel + Plan.solve on device data gives
    the same volume as parallelbeam.alg on host data (padding rows, centre
    shift)."""
    import torch
    from ccpi.reconstruction.device import pack_parallel, parallel_api_plan
    from ccpi.reconstruction.parallelbeam import alg as A
    rng = np.random.default_rng(30 + alg)
    na, nv, nh, cor = 40, 7, 50, 26.5
    pixels = rng.uniform(0.0, 2.0, (na, nv, nh)).astype(np.float32)
    deg = np.linspace(0, 180, na, endpoint=False).astype(np.float32)
    fn = {0: A.cgls, 1: A.sirt, 2: A.mlem}[alg]
    host = fn(pixels, deg, cor, 1, 5, 1, True)
    plan, nvp, voff = parallel_api_plan(na, nv, nh, deg, cor, 1)
    sino = pack_parallel(torch.from_numpy(pixels).to(cuda), nvp, voff)
    x = torch.zeros(plan.shape, device=cuda)
    plan.solve(alg, sino, x, 5)
    assert np.array_equal(x.cpu().numpy(), host)


def test_cgls_more_rows_than_one_projector_pass(cuda):
    """A parallel-beam problem of more than 256 detector rows (the forward
    projector then runs in several row passes): CGLS against the FP64
    oracle, whose step scalars use every row."""
    import torch
    from ccpi.reconstruction.device import parallel_plan
    rng = np.random.default_rng(41)
    shape, na, nh = (20, 20, 300), 16, 30
    p = parallel_plan(shape, na, nh)
    x_true = rng.random(shape).astype(np.float32)
    sino = p.forward(torch.from_numpy(x_true).to(cuda))
    x = torch.zeros(shape, device=cuda)
    p.solve(0, sino, x, 3)
    g = O.parallel_geometry(shape, na, nh)
    r64 = O.solve(g, 0, sino.cpu().numpy().astype(np.float64), 3, fp64=True)
    assert rel_l2(x.cpu().numpy(), r64) <= 1e-4


@pytest.mark.parametrize("kind", ["parallel", "cone"])
def test_autotuned_plan_gives_the_same_results(kind, cuda):
    """ccpi_plan_autotune changes launch shapes only: projections and SIRT
    are bit-identical to the untuned plan, CGLS agrees to FP64 rounding of
    its step scalars.  When it picks the cone scatter back projector, the
    back projection and CGLS agree to the projector tolerance instead."""
    import torch
    from ccpi.reconstruction.device import cone_plan, parallel_plan
    mk = (lambda: parallel_plan((48, 48, 32), 60, 72)) if kind == "parallel" else \
        (lambda: cone_plan(24, 1.0, 30, 32, 1.0, 60.0, 60.0))
    a, b = mk(), mk()
    chosen = b.autotune()
    assert chosen[0] > 0
    scatter = kind == "cone" and chosen[1] == 1
    rng = np.random.default_rng(17)
    x = torch.from_numpy(rng.random(a.shape).astype(np.float32)).to(cuda)
    sa, sb = a.forward(x), b.forward(x)
    assert torch.equal(sa, sb)
    ba, bb = a.backward(sa), b.backward(sb)
    if scatter:
        assert max_rel(bb.cpu().numpy(), ba.cpu().numpy()) <= 1e-5
    else:
        assert torch.equal(ba, bb)
    for alg, exact in ((1, True), (0, False)):
        xa = torch.zeros(a.shape, device=cuda)
        xb = torch.zeros(b.shape, device=cuda)
        a.solve(alg, sa, xa, 5)
        b.solve(alg, sb, xb, 5)
        if exact:
            assert torch.equal(xa, xb)
        else:
            assert rel_l2(xb.cpu().numpy(), xa.cpu().numpy()) <= (1e-5 if scatter else 1e-6)


def test_sirt_full_size_slices_equal_single_slice_solves(cuda):
    """The bench workload's size (768x768x256 grid, 720 angles, 768
    columns): SIRT on all 256 slices at once (the lane-parallel float4
    kernels) equals, bit for bit, SIRT on one slice at a time (a one-slice
    plan takes the scalar kernels) for slices at both ends and inside.
    Parallel-beam SIRT is separable by slice, so any difference would be a
    kernel error."""
    import torch
    from ccpi.reconstruction.device import parallel_plan
    p = parallel_plan((768, 768, 256), 720, 768)
    g = torch.Generator(device="cuda").manual_seed(21)
    s = torch.rand(p.sino_shape, device=cuda, generator=g) * 4.0
    full = torch.zeros(p.shape, device=cuda)
    p.solve(1, s, full, 2)
    p1 = parallel_plan((768, 768, 1), 720, 768)
    for k in (0, 97, 255):
        xk = torch.zeros(p1.shape, device=cuda)
        p1.solve(1, s[:, :, k:k + 1].contiguous(), xk, 2)
        assert torch.equal(xk[:, :, 0], full[:, :, k]), k


def test_cone_full_size_linearity(cuda):
    """The 512^3 cone workload (720 angles, 768^2 detector): A(2x) == 2 A(x)
    and A^T(2y) == 2 A^T(y) exactly (scaling by 2 is exact in float), and
    every value finite."""
    import torch
    from ccpi.reconstruction.device import cone_plan
    p = cone_plan(512, 1.0, 720, 768, 0.8, 500.0, 500.0)
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.rand(p.shape, device=cuda, generator=g)
    a1 = p.forward(x)
    assert torch.equal(p.forward(2 * x), 2 * a1)
    assert torch.isfinite(a1).all()
    del x
    b1 = p.backward(a1)
    assert torch.equal(p.backward(2 * a1), 2 * b1)
    assert torch.isfinite(b1).all()
