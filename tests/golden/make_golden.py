"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs CCPi-Reconstruction's own iterative core, compiled from its sources
into oracle/_ref/libccpi_ref.so (``make -C oracle``), on small seeded
synthetic inputs, and stores inputs and outputs as compressed .npz files.
The reference has no golden vectors of its own (its Python tests only
smoke-run), so these fixtures pin both the restatement in oracle/ and the
CUDA path.  Regenerate with:

    make -C oracle && python tests/golden/make_golden.py [name-prefix ...]
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def phantom2d(rng, n, nz, n_ell=6):
    """Sum of random ellipses per slice (densities 0.1..1), n x n x nz."""
    y, x = np.mgrid[0:n, 0:n] + 0.5 - n / 2.0
    vol = np.zeros((n, n, nz), np.float32)
    for k in range(nz):
        for _ in range(n_ell):
            cx, cy = rng.uniform(-0.4 * n, 0.4 * n, 2)
            a, b = rng.uniform(0.05 * n, 0.3 * n, 2)
            th = rng.uniform(0, math.pi)
            d = rng.uniform(0.1, 1.0)
            xr = (x - cx) * math.cos(th) + (y - cy) * math.sin(th)
            yr = -(x - cx) * math.sin(th) + (y - cy) * math.cos(th)
            vol[:, :, k] += np.where((xr / a) ** 2 + (yr / b) ** 2 <= 1.0, d, 0.0).astype(np.float32)
    return vol


def main(prefixes=()):
    """Write every fixture, or only those whose names start with one of
    `prefixes`."""
    os.makedirs(HERE, exist_ok=True)
    rng = np.random.default_rng(20240917)
    out = {}

    # ---- parallel projectors on explicit geometries, incl. axis-parallel
    # and 45-degree angles (ties) and a shifted centre
    cases = []
    for idx, (shape, na, nh, shift, extra) in enumerate(
            [((20, 20, 4), 23, 28, 0.25, [0.0, 45.0, 90.0, 135.0, 180.0, 270.0]),
             ((17, 24, 8), 19, 30, 0.0, [0.0, 90.0, 225.0]),
             ((40, 40, 8), 45, 57, -0.3, [])]):
        g = O.parallel_geometry(shape, na, nh, cor_shift=shift)
        if extra:
            g.angles = np.concatenate([g.angles, np.deg2rad(np.array(extra))])
        vol = rng.random(shape).astype(np.float32)
        pix = rng.random(g.sino_shape).astype(np.float32)
        fp = O.ref_forward(g, vol)
        bp = O.ref_backward(g, pix)
        out[f"pb{idx}"] = dict(angles=g.angles, h=g.h_pixels, v=g.v_pixels,
                              origin=np.array(g.origin), size=np.array(g.size),
                              shape=np.array(shape), vol=vol, pix=pix, fp=fp, bp=bp)
        cases.append(idx)

    # ---- cone projectors on explicit geometries.  The second is the 512^3
    # cone benchmark geometry scaled by 1/32 with a taller detector, so that
    # rays leave the volume through its top and bottom (the reference's
    # edge loops).  Geometries where a ray ENTERS through the top or bottom
    # face are avoided: there the reference reads alpha_inv[-1]
    # (Core/src/c2D.cpp:124-126 with ncom == 0) and its output is undefined.
    for idx, (n, na, nd, ndv, pix_size, s2o, o2d) in enumerate(
            [(16, 24, 24, 24, 0.8, 40.0, 40.0), (16, 24, 24, 28, 0.8, 15.625, 15.625)]):
        g = O.cone_geometry(n, 1.0, na, nd, pix_size, s2o, o2d, n_det_v=ndv)
        vol = rng.random(g.shape).astype(np.float32)
        pix = rng.random(g.sino_shape).astype(np.float32)
        with O.quiet():
            fp = O.ref_forward(g, vol)
            bp = O.ref_backward(g, pix)
        out[f"cb{idx}"] = dict(angles=g.angles, h=g.h_pixels, v=g.v_pixels,
                              origin=np.array(g.origin), size=np.array(g.size),
                              shape=np.array(g.shape), source=np.array(g.source),
                              detector_x=np.array(g.detector_x), vol=vol, pix=pix, fp=fp, bp=bp)

    # ---- parallel-beam API reconstructions (reconstruct_iter semantics)
    na, nv, nh = 30, 6, 36
    ph = phantom2d(rng, 32, nv)
    ang_deg = np.linspace(0.0, 180.0, na, endpoint=False).astype(np.float32)
    g, nvp, voff = O.parallel_api_geometry(na, nv, 32, ang_deg, 0.0, 1)
    gph = O.parallel_geometry((32, 32, nv), na, 32)
    gph.angles = g.angles
    sino_log = O.ref_forward(gph, ph)  # (na, 32, nv)
    sino_log = np.ascontiguousarray(np.transpose(sino_log, (0, 2, 1)))
    sino_log = np.pad(sino_log, ((0, 0), (0, 0), (2, 2)))  # nh = 36
    trans = np.exp(-0.05 * sino_log).astype(np.float32)
    for cor, ppv, is_log, data in [(0.0, 1, False, trans), (18.25, 1, True, sino_log * 0.05),
                                   (0.0, 2, True, sino_log * 0.05)]:
        for alg, lam in [(O.CGLS, 0.0), (O.SIRT, 0.0), (O.MLEM, 0.0), (O.TIKHONOV, 0.002),
                         (O.TV, 0.0005)]:
            with O.quiet():
                rec = O.ref_pb_reconstruct(alg, data, ang_deg, cor, ppv, 6, is_log, lam=lam)
            out[f"api_alg{alg}_cor{cor}_ppv{ppv}"] = dict(
                pixels=np.asarray(data, np.float32), angles=ang_deg, cor=np.array(cor),
                ppv=np.array(ppv), is_log=np.array(int(is_log)), alg=np.array(alg),
                lam=np.array(lam), niter=np.array(6), out=rec)
    # warm-start (step) forms
    x0 = rng.random(O.ref_pb_geometry(na, nv, nh, 0.0, 1)[0][:3]).astype(np.float32) * 0.01
    for alg in (O.CGLS, O.SIRT, O.MLEM):
        with O.quiet():
            rec = O.ref_pb_reconstruct(alg, trans, ang_deg, 0.0, 1, 4, False, x0=x0)
        out[f"step_alg{alg}"] = dict(pixels=trans, angles=ang_deg, alg=np.array(alg), x0=x0,
                                     out=rec, niter=np.array(4))

    # ---- parallel-beam grids of the numpy path
    grids = []
    for (na_, nv_, nh_, cor_, ppv_) in [(91, 8, 160, 0.0, 1), (180, 16, 192, 96.25, 1),
                                        (10, 7, 33, 0.0, 2), (5, 13, 50, 20.0, 3),
                                        (720, 256, 768, 0.0, 1), (3, 1, 9, 4.5, 1)]:
        dims, geo = O.ref_pb_geometry(na_, nv_, nh_, cor_, ppv_)
        grids.append([na_, nv_, nh_, cor_, ppv_, *dims, *geo])
    out["pb_grids"] = dict(rows=np.array(grids, np.float64))

    # ---- pb_forward_project / pb_backward_project wrappers
    vol = rng.random((24, 20, 8)).astype(np.float32)
    ang = np.linspace(0, 180, 16, endpoint=False).astype(np.float32)
    fp = O.ref_pb_forward_project(vol, ang, 1)
    stack = rng.random((16, 8, 26)).astype(np.float32)
    bp = O.ref_pb_backward_project(stack, ang, 0.0, 1)
    out["pb_wrappers"] = dict(vol=vol, angles=ang, fp=fp, stack=stack, bp=bp)

    # ---- cone-beam numpy path: grid and centre search
    cgrid = []
    for (na_, nh_, nv_, ppv_, s2s, s2d, px_h, px_v, mr) in [
            (36, 40, 24, 1, 50.0, 100.0, 0.5, 0.5, 8.0),
            (20, 32, 30, 2, 80.0, 200.0, 0.4, 0.4, 6.0),
            (12, 24, 16, 1, 30.0, 45.0, 1.0, 1.0, 12.0)]:
        dims, geo = O.ref_cb_geometry(na_, nh_, nv_, ppv_, s2s, s2d, px_h, px_v, mr)
        cgrid.append([na_, nh_, nv_, ppv_, s2s, s2d, px_h, px_v, mr, *dims, *geo[:5]])
    out["cb_grids"] = dict(rows=np.array(cgrid, np.float64))
    # centre search on data from a source shifted off the axis
    na_, nh_, nv_ = 40, 48, 16
    s2s, s2d, px = 60.0, 120.0, 0.5
    shift = 0.7
    gshift = O.cone_geometry((24, 24, 16), 0.5, na_, nh_, px, s2s, s2d - s2s, n_det_v=nv_)
    gshift.source = (-s2s, shift, 0.0)
    gshift.h_pixels = gshift.h_pixels + shift
    ball = np.zeros(gshift.shape, np.float32)
    zz, yy, xx = np.meshgrid(*(np.arange(n) - n / 2 + 0.5 for n in gshift.shape), indexing="ij")
    ball[(xx / 8) ** 2 + (yy / 6) ** 2 + ((zz - 2) / 5) ** 2 <= 1] = 1.0
    ball[((xx - 4) / 3) ** 2 + ((yy + 3) / 4) ** 2 + (zz / 4) ** 2 <= 1] += 0.5
    with O.quiet():
        csino = O.ref_forward(gshift, ball)
    ang_c = np.rad2deg(gshift.angles).astype(np.float32)
    with O.quiet():
        dims, geo = O.ref_cb_geometry(na_, nh_, nv_, 1, s2s, s2d, px, px, 6.5, pixels=csino,
                                      angles_deg=ang_c, is_log=True)
        crec = O.ref_cb_reconstruct(O.CGLS, csino, ang_c, 1, s2s, s2d, px, px, 6.5, 3, True)
    out["cb_centre"] = dict(sino=csino, angles=ang_c, s2s=np.array(s2s), s2d=np.array(s2d),
                            px=np.array(px), mask_radius=np.array(6.5), dims=dims, geom=geo,
                            cgls3=crec)

    out.update(aml_cases())
    out.update(prefilter_cases())
    if prefixes:
        out = {k: v for k, v in out.items() if k.startswith(tuple(prefixes))}
    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
    total = sum(os.path.getsize(os.path.join(HERE, f"{n}.npz")) for n in out)
    print(f"wrote {len(out)} fixtures, {total / 1e6:.2f} MB")


def aml_cases():
    """parallelbeam.filters.aml_ring_artefacts on transmission stacks with
    ring artefacts: a phantom projected by the reference, then per-column
    gain errors (stripes in the sinogram, rings in the image)."""
    rng = np.random.default_rng(515)
    out = {}
    for idx, (n, na, nh, nv, pn, pr, ns) in enumerate(
            [(24, 60, 32, 3, 0.0, 0.005, 1), (32, 90, 44, 4, 0.2, 0.01, 3),
             (20, 45, 30, 2, 1.0, 0.1, 2)]):
        g = O.parallel_geometry((n, n, nv), na, nh)
        vol = phantom2d(rng, n, nv) * 0.05
        with O.quiet():
            sino = O.ref_forward(g, vol)  # (na, nh, nv)
        gains = 1.0 + 0.02 * rng.standard_normal((1, nh, nv))
        trans = (np.exp(-sino.astype(np.float64)) * gains).astype(np.float32)
        pixels = np.ascontiguousarray(trans.transpose(0, 2, 1))  # (na, nv, nh)
        res = O.ref_aml_ring_artefacts(pixels, pn, pr, ns)
        out[f"aml{idx}"] = dict(pixels=pixels, param_n=np.float32(pn), param_r=np.float32(pr),
                                num_series=np.array(ns), out=res)
    return out


def prefilter_cases():
    """The reference's high-peaks filter (Diamond::high_peaks_before) and
    column ring filter (remove_column_ring_artefacts) on log sinogram
    stacks (na, nh, nv): a projected phantom with bright single-angle spikes
    (the peaks) and per-element offsets (the stripes), including an
    all-zero padding row."""
    rng = np.random.default_rng(613)
    out = {}
    for idx, (n, na, nh, nv, jump, npix) in enumerate(
            [(24, 60, 32, 3, 0.05, 1), (32, 90, 44, 4, 0.02, 3), (16, 12, 20, 2, 0.0, 11)]):
        g = O.parallel_geometry((n, n, nv), na, nh)
        vol = phantom2d(rng, n, nv) * 0.05
        with O.quiet():
            sino = O.ref_forward(g, vol)  # (na, nh, nv)
        sino = sino + (0.03 * rng.standard_normal((1, nh, nv))).astype(np.float32)
        spikes = rng.random(sino.shape) < 0.02
        sino = np.where(spikes, sino + rng.uniform(0.5, 2.0, sino.shape), sino).astype(np.float32)
        sino[:, :, -1] = 0.0
        out[f"hp{idx}"] = dict(logs=sino, jump=np.array(jump), num_pix=np.array(npix),
                               out=O.ref_high_peaks(sino, jump, npix))
        out[f"colring{idx}"] = dict(logs=sino, out=O.ref_column_ring(sino))
    return out


if __name__ == "__main__":
    main(sys.argv[1:])
