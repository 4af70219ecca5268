"""Seeded synthetic inputs of the stated workload configurations, for the
parity tests (numpy; the projections come from the oracle).

Every input is generated here from a seed; no dataset is read.  Random
draws use numpy.random.default_rng(seed), in the order centres, semi-axes,
rotation, density per ellipse, slice by slice, then noise.
"""
from __future__ import annotations

import math

import numpy as np

import oracle as O


def ellipse_slices(rng, n, nz, n_ell, axes, inner=0.8):
    """n x n x nz volume: per slice n_ell ellipses with centres uniform in
    the inner `inner` fraction of the slice, semi-axes U[axes] px, rotation
    U[0, pi), density U[0.1, 1]; overlapping densities add."""
    c = np.arange(n) + 0.5 - n / 2.0
    X, Y = np.meshgrid(c, c, indexing="ij")
    vol = np.zeros((n, n, nz), np.float32)
    for k in range(nz):
        for _ in range(n_ell):
            cx, cy = rng.uniform(-inner / 2, inner / 2, 2) * n
            a, b = rng.uniform(axes[0], axes[1], 2)
            th = rng.uniform(0.0, math.pi)
            d = rng.uniform(0.1, 1.0)
            xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
            yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
            vol[:, :, k] += np.where((xr / a) ** 2 + (yr / b) ** 2 <= 1.0, d, 0.0).astype(np.float32)
    return vol


def poisson_log(sino, i0, rng, max_integral=3.0):
    """Scale the line integrals so the largest is `max_integral`, draw
    counts ~ Poisson(i0 exp(-mu p)) and return -log(max(counts, 1) / i0) as
    float32 (the log data the solvers take with is_pixels_in_log=True)."""
    mu = max_integral / float(np.max(sino))
    counts = rng.poisson(i0 * np.exp(-mu * sino.astype(np.float64)))
    return (-np.log(np.maximum(counts, 1) / i0)).astype(np.float32), mu


def config1():
    """Plain parallel-beam CGLS case: a 128x128x16 phantom of 10 ellipses
    per slice (semi-axes 5-40 px, seed 1) projected by the reference's
    parallel_beam::f2D at 180 angles in [0, pi) onto 192 columns x 16 rows
    with the centre of rotation at the detector midpoint + 0.25 px, Poisson
    noise at 1e4 photons per ray, -log.  Returns the numpy call's inputs:
    pixels (180, 16, 192) float32 log data, angles in degrees (float32), the
    rotation centre 96.25 and the iteration count 20."""
    rng = np.random.default_rng(1)
    na, nv, nh, n, nz = 180, 16, 192, 128, 16
    vol = ellipse_slices(rng, n, nz, 10, (5.0, 40.0))
    deg = np.linspace(0.0, 180.0, na, endpoint=False).astype(np.float32)
    cor = nh / 2.0 + 0.25
    # the detector the numpy call derives for this centre (diamond.cpp:64-70)
    g = O.parallel_geometry((n, n, nz), na, nh, nv=nv, cor_shift=cor - nh / 2.0)
    g.angles = math.pi * (deg.astype(np.float64) / 180.0)
    sino = O.ref_forward(g, vol) if O.reference_available() else O.forward(g, vol)
    y, _ = poisson_log(sino, 1.0e4, rng)
    pixels = np.ascontiguousarray(np.transpose(y, (0, 2, 1)))
    return pixels, deg, cor, 20


def uneven_problem(j, count=64):
    """Problem j of the 64 seeded uneven CGLS-Tikhonov / CGLS-TV problems
    (SeedSequence(4).spawn(64)[j]): width w ~ U{64..384}, rows nz ~
    U{8..64}, angles ~ U{90..900} over [0, pi), round(1.5 w) detector
    columns, lambda log-uniform in [1e-3, 1e-1]; 10 ellipses per slice
    (semi-axes 4-31 % of w) projected on a centred w x w x nz grid, then
    Gaussian noise of 2 % of the largest projection.  Returns (pixels
    (na, nz, ncols) float32, degrees float32, lambda, algorithm 3 or 4)."""
    ss = np.random.SeedSequence(4).spawn(count)[j]
    rng = np.random.default_rng(ss)
    w = int(rng.integers(64, 385))
    nz = int(rng.integers(8, 65))
    na = int(rng.integers(90, 901))
    nh = int(round(1.5 * w))
    lam = float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-1))))
    deg = np.linspace(0.0, 180.0, na, endpoint=False).astype(np.float32)
    c = np.arange(w) + 0.5 - w / 2.0
    X, Y = np.meshgrid(c, c, indexing="ij")
    vol = np.zeros((w, w, nz), np.float32)
    for k in range(nz):
        for _ in range(10):
            cx, cy = rng.uniform(-0.4, 0.4, 2) * w
            a, b = rng.uniform(0.04, 0.31, 2) * w
            th = rng.uniform(0, math.pi)
            d = rng.uniform(0.1, 1.0)
            xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
            yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
            vol[:, :, k] += (((xr / a) ** 2 + (yr / b) ** 2) <= 1.0).astype(np.float32) * np.float32(d)
    g = O.parallel_geometry((w, w, nz), na, nh, nv=nz)
    g.angles = math.pi * (deg.astype(np.float64) / 180.0)
    s = O.forward(g, vol)
    s = s + rng.normal(0.0, 0.02 * np.abs(s).max(), s.shape).astype(np.float32)
    pixels = np.ascontiguousarray(s.transpose(0, 2, 1), np.float32)
    return pixels, deg, lam, 3 + (j % 2)


def uneven_sizes(count=64):
    """(w, nz, na) of every uneven problem, without building them."""
    out = []
    for ss in np.random.SeedSequence(4).spawn(count):
        rng = np.random.default_rng(ss)
        w = int(rng.integers(64, 385))
        nz = int(rng.integers(8, 65))
        na = int(rng.integers(90, 901))
        out.append((w, nz, na))
    return out


def cone_case():
    """A 24^3 grid, 40 angles over 2 pi, 36 x 32 detector, seeded ellipsoid
    data with 1 % noise."""
    g = O.cone_geometry(24, 1.0, 40, 36, 1.0, 60.0, 60.0, n_det_v=32)
    rng = np.random.default_rng(71)
    c = np.arange(24) + 0.5 - 12
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    vol = np.zeros((24, 24, 24), np.float32)
    for _ in range(5):
        cen = rng.uniform(-5, 5, 3)
        ax = rng.uniform(3, 9, 3)
        vol += ((((X - cen[0]) / ax[0]) ** 2 + ((Y - cen[1]) / ax[1]) ** 2 +
                 ((Z - cen[2]) / ax[2]) ** 2) <= 1).astype(np.float32) * np.float32(rng.uniform(0.1, 1))
    s = O.forward(g, vol)
    s = (s + rng.normal(0, 0.01 * s.max(), s.shape)).astype(np.float32)
    return g, s
