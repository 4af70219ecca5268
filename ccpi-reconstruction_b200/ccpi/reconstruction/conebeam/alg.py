"""``ccpi.reconstruction.conebeam.alg`` on a B200.

Same functions, argument order and conventions as the reference module
(Wrappers/Python/src/conebeam_module.cpp:32-41, conebeam_wrapper.cpp):

* ``pixels``: (n_angles, n_h, n_v) projections (no transpose, unlike the
  parallel-beam module); transmission unless ``is_pixels_in_log``;
* ``angles`` in degrees; the source sits at (-source_to_sample, 0, 0) and
  the detector plane at source_to_detector - source_to_sample;
* ``pixels_per_voxel``, ``pixel_h_size``, ``pixel_v_size`` and
  ``mask_radius`` set the voxel grid the reference derives
  (Readers/xtek.cpp:760-798); the centre of rotation is searched on the
  data (xtek.cpp:671-758) before solving;
* ``h_offsets``, ``v_offsets``, ``beam_harden``, ``full_vox_origin`` and
  ``voxel_size`` are accepted and, as in the reference, do not change the
  result (the reference copies the last two into locals it overwrites);
* result: a new float32 volume (nx, ny, nz), clamped at zero.

``create_sinogram`` is the cone forward projection of an explicit geometry
(angles in radians there, as in the reference).  Deviations as in the
parallel-beam module: conversion instead of reinterpretation of other
dtypes, exceptions instead of (1, 1, 1) zero arrays, ``nthreads`` ignored.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _native as N

__all__ = ["cgls", "cgls_conv", "sirt", "mlem", "cgls_tikhonov", "cgls_TVreg",
           "create_sinogram", "create_phantom", "create_phantom_volume", "grid",
           "find_centre"]


def grid(n_angles, n_h, n_v, pixels_per_voxel, source_to_sample, source_to_detector,
         pixel_h_size, pixel_v_size, mask_radius):
    """((nx, ny, nz, n_v_padded, v_offset), (voxel xy, voxel z, origin x, y, z))."""
    dims = np.zeros(5, np.int32)
    geom = np.zeros(5, np.float64)
    N.check(N.lib.ccpi_cb_grid(int(n_angles), int(n_h), int(n_v), int(pixels_per_voxel),
                               float(source_to_sample), float(source_to_detector),
                               float(pixel_h_size), float(pixel_v_size), float(mask_radius),
                               dims, geom), "conebeam grid")
    return tuple(int(d) for d in dims), tuple(float(g) for g in geom)


def find_centre(padded_log_sino, angles, source_to_sample, source_to_detector, pixel_h_size):
    """Source y offset of the reference's centre search on a padded log
    sinogram (n_angles, n_h, n_v_padded)."""
    s = N.f32(padded_log_sino, "sinogram", 3)
    a = N.f32(angles, "angles", 1)
    y = ctypes.c_double(0.0)
    N.check(N.lib.ccpi_cb_find_centre(s, *s.shape, a, float(source_to_sample),
                                      float(source_to_detector), float(pixel_h_size),
                                      ctypes.byref(y)), "conebeam find_centre")
    return y.value


def _reconstruct(alg, pixels, angles, pixels_per_voxel, source_to_sample, source_to_detector,
                 pixel_h_size, pixel_v_size, mask_radius, niterations, nthreads,
                 is_pixels_in_log, regularize=0.0, norm_r=None, real_norms=False):
    pix = N.f32(pixels, "pixels", 3)
    ang = N.f32(angles, "angles", 1)
    na, nh, nv = pix.shape
    if ang.shape[0] != na:
        raise ValueError(f"Number of projections ({na}) doesn't match angle array "
                         f"({ang.shape[0]})")
    niterations = int(niterations)
    if niterations < 0:
        raise ValueError("niterations must be >= 0")
    dims, _ = grid(na, nh, nv, pixels_per_voxel, source_to_sample, source_to_detector,
                   pixel_h_size, pixel_v_size, mask_radius)
    out = np.zeros(dims[:3], np.float32)
    norms = np.zeros(max(niterations, 1), np.float64)
    N.check(N.lib.ccpi_cb_reconstruct(alg, pix, na, nh, nv, ang, int(pixels_per_voxel),
                                      float(source_to_sample), float(source_to_detector),
                                      float(pixel_h_size), float(pixel_v_size),
                                      float(mask_radius), niterations, int(nthreads),
                                      int(bool(is_pixels_in_log)), float(regularize),
                                      norms.ctypes.data, out), "conebeam reconstruction")
    if norm_r is not None:
        nr = np.asarray(norm_r)
        n = min(niterations, nr.shape[0]) if nr.ndim == 1 else 0
        if real_norms:
            nr[:n] = norms[:n]
        elif n:
            # conebeam_wrapper.cpp:84-93 overwrites norm_r with zeros
            nr[:n] = 0
    return out


def cgls(pixels, angles, h_offsets, v_offsets, pixels_per_voxel, source_to_sample,
         source_to_detector, pixel_h_size, pixel_v_size, mask_radius, beam_harden,
         full_vox_origin, voxel_size, niterations, nthreads, is_pixels_in_log=True):
    return _reconstruct(N.CGLS, pixels, angles, pixels_per_voxel, source_to_sample,
                        source_to_detector, pixel_h_size, pixel_v_size, mask_radius,
                        niterations, nthreads, is_pixels_in_log)


def sirt(pixels, angles, h_offsets, v_offsets, pixels_per_voxel, source_to_sample,
         source_to_detector, pixel_h_size, pixel_v_size, mask_radius, beam_harden,
         full_vox_origin, voxel_size, niterations, nthreads, is_pixels_in_log=True):
    return _reconstruct(N.SIRT, pixels, angles, pixels_per_voxel, source_to_sample,
                        source_to_detector, pixel_h_size, pixel_v_size, mask_radius,
                        niterations, nthreads, is_pixels_in_log)


def mlem(pixels, angles, h_offsets, v_offsets, pixels_per_voxel, source_to_sample,
         source_to_detector, pixel_h_size, pixel_v_size, mask_radius, beam_harden,
         full_vox_origin, voxel_size, niterations, nthreads, is_pixels_in_log=True):
    return _reconstruct(N.MLEM, pixels, angles, pixels_per_voxel, source_to_sample,
                        source_to_detector, pixel_h_size, pixel_v_size, mask_radius,
                        niterations, nthreads, is_pixels_in_log)


def cgls_conv(pixels, angles, h_offsets, v_offsets, pixels_per_voxel, source_to_sample,
              source_to_detector, pixel_h_size, pixel_v_size, mask_radius, beam_harden,
              full_vox_origin, voxel_size, niterations, nthreads, norm_r,
              is_pixels_in_log=True, real_norms=False):
    return _reconstruct(N.CGLS, pixels, angles, pixels_per_voxel, source_to_sample,
                        source_to_detector, pixel_h_size, pixel_v_size, mask_radius,
                        niterations, nthreads, is_pixels_in_log, norm_r=norm_r,
                        real_norms=real_norms)


def cgls_tikhonov(pixels, angles, h_offsets, v_offsets, pixels_per_voxel, source_to_sample,
                  source_to_detector, pixel_h_size, pixel_v_size, mask_radius, beam_harden,
                  full_vox_origin, voxel_size, niterations, nthreads, regularize, norm_r,
                  is_pixels_in_log=True, real_norms=False):
    return _reconstruct(N.CGLS_TIKHONOV, pixels, angles, pixels_per_voxel, source_to_sample,
                        source_to_detector, pixel_h_size, pixel_v_size, mask_radius,
                        niterations, nthreads, is_pixels_in_log, regularize, norm_r,
                        real_norms=real_norms)


def cgls_TVreg(pixels, angles, h_offsets, v_offsets, pixels_per_voxel, source_to_sample,
               source_to_detector, pixel_h_size, pixel_v_size, mask_radius, beam_harden,
               full_vox_origin, voxel_size, niterations, nthreads, regularize, norm_r,
               is_pixels_in_log=True, real_norms=False):
    return _reconstruct(N.CGLS_TV, pixels, angles, pixels_per_voxel, source_to_sample,
                        source_to_detector, pixel_h_size, pixel_v_size, mask_radius,
                        niterations, nthreads, is_pixels_in_log, regularize, norm_r,
                        real_norms=real_norms)


def create_sinogram(source_x, source_y, source_z, detector_x, h_pixels, v_pixels, angles,
                    voxels, grid_offset, voxel_size):
    """Cone forward projection with explicit geometry
    (conebeam_wrapper.cpp:346-400): angles in radians, output
    (n_angles, n_h, n_v)."""
    vol = N.f32(voxels, "voxels", 3)
    # the reference reads every geometry value through float32
    h = np.asarray(h_pixels, np.float32).astype(np.float64)
    v = np.asarray(v_pixels, np.float32).astype(np.float64)
    a = np.asarray(angles, np.float32).astype(np.float64)
    g = N.Geometry()
    g.kind = N.CONE
    keep = [np.ascontiguousarray(x) for x in (a, h, v)]
    g.angles, g.h_pixels, g.v_pixels = (x.ctypes.data for x in keep)
    g.n_angles, g.n_h, g.n_v = len(a), len(h), len(v)
    f = lambda x: float(np.float32(x))  # noqa: E731
    g.source = (ctypes.c_double * 3)(f(source_x), f(source_y), f(source_z))
    g.detector_x = f(detector_x)
    go = np.asarray(grid_offset, np.float32)
    vs = np.asarray(voxel_size, np.float32)
    g.origin = (ctypes.c_double * 3)(*(float(x) for x in go[:3]))
    g.voxel_size = (ctypes.c_double * 3)(*(float(x) for x in vs[:3]))
    g.nx, g.ny, g.nz = vol.shape
    out = np.zeros((len(a), len(h), len(v)), np.float32)
    N.check(N.lib.ccpi_cb_create_sinogram(ctypes.byref(g), vol, out), "create_sinogram")
    return out


def reconstruct_explicit(algorithm, source, detector_x, h_pixels, v_pixels, angles, sino,
                         grid_offset, voxel_size, shape, niterations, regularize=0.0,
                         norm_r=None, backprojector="gather"):
    """A cone-beam solver on an explicit geometry with host arrays
    (``ccpi_reconstruct``; the reference's reconstruction_alg::reconstruct
    on an explicitly set instrument, Core/src/algorithms.hpp:13-20).
    algorithm: "cgls", "sirt", "mlem", "cgls_tikhonov" or "cgls_TVreg";
    angles in radians; sino (n_angles, n_h, n_v) log data; returns the
    clamped volume of `shape`; norm_r (optional, one entry per iteration)
    receives |A^T r| for the CGLS family.  backprojector: "gather" (the
    default, deterministic: b2D bit for bit) or "scatter" (the CGLS family
    back-projects with the ray-driven scatter, ``CCPI_RECON_CONE_SCATTER``:
    faster, equal to float rounding)."""
    algs = {"cgls": N.CGLS, "sirt": N.SIRT, "mlem": N.MLEM, "cgls_tikhonov": N.CGLS_TIKHONOV,
            "cgls_TVreg": N.CGLS_TV}
    if algorithm not in algs:
        raise ValueError(f"unknown algorithm {algorithm!r}")
    a, h, v = (np.ascontiguousarray(x, np.float64) for x in (angles, h_pixels, v_pixels))
    s = N.f32(sino, "sino", 3)
    if s.shape != (len(a), len(h), len(v)):
        raise ValueError(f"sino has shape {s.shape}, the geometry needs "
                         f"{(len(a), len(h), len(v))}")
    g = N.Geometry()
    g.kind = N.CONE
    g.angles, g.h_pixels, g.v_pixels = a.ctypes.data, h.ctypes.data, v.ctypes.data
    g.n_angles, g.n_h, g.n_v = len(a), len(h), len(v)
    g.source = (ctypes.c_double * 3)(*(float(x) for x in source))
    g.detector_x = float(detector_x)
    g.origin = (ctypes.c_double * 3)(*(float(x) for x in grid_offset))
    g.voxel_size = (ctypes.c_double * 3)(*(float(x) for x in voxel_size))
    g.nx, g.ny, g.nz = (int(x) for x in shape)
    out = np.zeros(tuple(int(x) for x in shape), np.float32)
    norms = np.zeros(max(int(niterations), 1), np.float64)
    forms = {"gather": 0, "scatter": N.RECON_CONE_SCATTER}
    if backprojector not in forms:
        raise ValueError(f"unknown backprojector {backprojector!r}")
    N.check(N.lib.ccpi_reconstruct_flags(ctypes.byref(g), algs[algorithm], s.ctypes.data,
                                         int(niterations), float(regularize),
                                         norms.ctypes.data, out.ctypes.data,
                                         forms[backprojector]), "reconstruct_explicit")
    if norm_r is not None:
        nr = np.asarray(norm_r)
        n = min(int(niterations), nr.shape[0])
        nr[:n] = norms[:n]
    return out


# ---- demonstration phantom of the Nikon XTek instrument
# (Nikon_XTek::create_phantom / build_phantom / initialise_phantom_volume,
# Core/src/Readers/xtek.cpp:131-175, :392-457, :825-894; wrappers
# conebeam_wrapper.cpp:238-310)
_PH_PIXEL = 0.390625


def _phantom_geometry():
    """Source x, detector x, detector coordinates (512 columns = 512 rows),
    250 angles in radians and the mask radius of the XTek phantom."""
    source_x, detector_x = -250.0, 737.0
    c = 0
    while c < 1000 and not (-99.8046875 + float(c) * _PH_PIXEL >= 100.0 + 0.001):
        c += 1
    pix = -99.8046875 + np.arange(c, dtype=np.float64) * _PH_PIXEL
    step = 2.0 * np.pi / 250.0
    phi = np.arange(250, dtype=np.float64) * step
    mask_radius = -source_x * np.sin(np.arctan(pix[-1] / (detector_x - source_x)))
    return source_x, detector_x, pix, phi, float(mask_radius)


def _phantom_volume(mask_radius):
    """512^3 volume of three unit cubes and its voxel size / origin."""
    n = 512
    vsize = 2.0 * mask_radius / n
    x = np.zeros((n, n, n), np.float32)
    x[107:189, 107:189, 57:139] = 1.0
    x[189:271, 189:271, 139:221] = 1.0
    x[271:353, 271:353, 221:303] = 1.0
    return x, vsize, -(vsize * n) / 2.0


def create_phantom():
    """(pixels (250, 512, 512) float32 projections, angles (250,) float32
    degrees, source_x = 250.0, detector_x = 987.0, pixel_h_size,
    pixel_v_size, mask_radius), as the reference returns them.  The
    projections are this library's cone-beam forward projection of the
    three-cube phantom; the reference projects it with its generic 3-D
    Siddon routine (instrument::forward_project), which traces the same line
    integrals with different float rounding."""
    source_x, detector_x, pix, phi, mask_radius = _phantom_geometry()
    vol, vsize, off = _phantom_volume(mask_radius)
    g = N.Geometry()
    g.kind = N.CONE
    keep = [np.ascontiguousarray(phi), np.ascontiguousarray(pix), np.ascontiguousarray(pix)]
    g.angles, g.h_pixels, g.v_pixels = (x.ctypes.data for x in keep)
    g.n_angles, g.n_h, g.n_v = len(phi), len(pix), len(pix)
    g.source = (ctypes.c_double * 3)(source_x, 0.0, 0.0)
    g.detector_x = detector_x
    g.origin = (ctypes.c_double * 3)(off, off, off)
    g.voxel_size = (ctypes.c_double * 3)(vsize, vsize, vsize)
    g.nx = g.ny = g.nz = vol.shape[0]
    out = np.zeros((len(phi), len(pix), len(pix)), np.float32)
    N.check(N.lib.ccpi_cb_create_sinogram(ctypes.byref(g), vol, out), "create_phantom")
    angles = (phi * 180.0 / np.pi).astype(np.float32)
    return (out, angles, -source_x, detector_x - source_x, _PH_PIXEL, _PH_PIXEL, mask_radius)


def create_phantom_volume():
    """(voxels (512, 512, 512) float32, angles (250,) float32 degrees,
    h_pixels (512,) float32, v_pixels (512,) float32, source_x = 250.0,
    detector_x = 987.0, pixel_h_size, pixel_v_size, mask_radius): the
    phantom volume without projecting it, as the reference returns it."""
    source_x, detector_x, pix, phi, mask_radius = _phantom_geometry()
    vol, _, _ = _phantom_volume(mask_radius)
    angles = (phi * 180.0 / np.pi).astype(np.float32)
    p32 = pix.astype(np.float32)
    return (vol, angles, p32, p32.copy(), -source_x, detector_x - source_x, _PH_PIXEL,
            _PH_PIXEL, mask_radius)
