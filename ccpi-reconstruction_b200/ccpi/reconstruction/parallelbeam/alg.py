"""``ccpi.reconstruction.parallelbeam.alg`` on a B200.

Same functions, argument order, conventions and outputs as the reference
module (Wrappers/Python/src/diamond_module.cpp:32-50, signatures in
diamond_wrapper.hpp / diamond_wrapper.cpp):

* ``pixels``: (n_angles, n_v, n_h) projections; transmission unless
  ``is_pixels_in_log`` (then -log is not applied);
* ``angles`` in degrees (read as float32, as the reference reads them);
* ``rotation_centre``: detector column of the rotation axis; a value <= 0
  means "centre of the detector" (no shift), as in the reference;
* ``resolution``: detector pixels per voxel edge;
* result: a new float32 volume (nx, ny, nz), x slowest, z fastest, on the
  grid the reference derives from the detector (rows padded to a multiple
  of 4 voxels), clamped at zero.

Deviations, all on inputs the reference does not check: arrays of other
dtypes are converted to float32 (the reference reinterprets their bytes),
bad shapes raise ValueError and failures raise RuntimeError instead of
printing a message and returning a (1, 1, 1) zero array.  ``nthreads`` is
accepted and ignored.  ``norm_r`` behaves as in the reference (zero-filled
when its first element is nonzero); pass ``real_norms=True`` to receive the
per-iteration |A^T r| instead.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _native as N

__all__ = ["cgls", "cgls_conv", "sirt", "mlem", "cgls_tikhonov", "cgls_TVreg",
           "cgls_step", "cgls_conv_step", "sirt_step", "mlem_step", "cgls_tikhonov_step",
           "cgls_TVreg_step", "pb_forward_project", "pb_backward_project",
           "pb_setup_geometry_from_image", "pb_setup_geometry_from_acquisition", "grid",
           "reconstruct_batched"]


def grid(n_angles, n_v, n_h, rotation_centre, resolution):
    """(nx, ny, nz, n_v_padded, v_offset) of the reconstruction grid."""
    dims = np.zeros(5, np.int32)
    N.check(N.lib.ccpi_pb_grid(int(n_angles), int(n_v), int(n_h), float(rotation_centre),
                               int(resolution), dims), "parallelbeam grid")
    return tuple(int(d) for d in dims)


def _reconstruct(alg, pixels, angles, rotation_centre, resolution, niterations, nthreads,
                 is_pixels_in_log, regularize=0.0, norm_r=None, x0=None, real_norms=False):
    pix = N.f32(pixels, "pixels", 3)
    ang = N.f32(angles, "angles", 1)
    na, nv, nh = pix.shape
    if ang.shape[0] != na:
        raise ValueError(f"Number of projections ({na}) doesn't match angle array "
                         f"({ang.shape[0]})")
    niterations = int(niterations)
    if niterations < 0:
        raise ValueError("niterations must be >= 0")
    nx, ny, nz, _, _ = grid(na, nv, nh, rotation_centre, resolution)
    out = np.zeros((nx, ny, nz), np.float32)
    x0p = None
    if x0 is not None:
        x0a = N.f32(x0, "last_iteration_volume", 3)
        if x0a.shape != out.shape:
            raise ValueError(f"last_iteration_volume has shape {x0a.shape}, the grid is "
                             f"{out.shape}")
        x0p = x0a.ctypes.data
    norms = np.zeros(max(niterations, 1), np.float64)
    N.check(N.lib.ccpi_pb_reconstruct(alg, pix, na, nv, nh, ang, float(rotation_centre),
                                      int(resolution), niterations, int(nthreads),
                                      int(bool(is_pixels_in_log)), float(regularize), x0p,
                                      norms.ctypes.data, out),
            "parallelbeam reconstruction")
    if norm_r is not None:
        nr = np.asarray(norm_r)
        n = min(niterations, nr.shape[0]) if nr.ndim == 1 else 0
        if real_norms:
            nr[:n] = norms[:n]
        elif n and nr[0] != 0:
            # diamond_wrapper.cpp:99-108 overwrites norm_r with zeros
            nr[:n] = 0
    return out


def cgls(pixels, angles, rotation_centre, resolution, niterations, nthreads, is_pixels_in_log):
    return _reconstruct(N.CGLS, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log)


def cgls_conv(pixels, angles, rotation_centre, resolution, niterations, nthreads, norm_r,
              is_pixels_in_log, real_norms=False):
    return _reconstruct(N.CGLS, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, norm_r=norm_r, real_norms=real_norms)


def sirt(pixels, angles, rotation_centre, resolution, niterations, nthreads, is_pixels_in_log):
    return _reconstruct(N.SIRT, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log)


def mlem(pixels, angles, rotation_centre, resolution, niterations, nthreads, is_pixels_in_log):
    return _reconstruct(N.MLEM, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log)


def cgls_tikhonov(pixels, angles, rotation_centre, resolution, niterations, nthreads,
                  regularize, norm_r, is_pixels_in_log, real_norms=False):
    return _reconstruct(N.CGLS_TIKHONOV, pixels, angles, rotation_centre, resolution,
                        niterations, nthreads, is_pixels_in_log, regularize, norm_r,
                        real_norms=real_norms)


def cgls_TVreg(pixels, angles, rotation_centre, resolution, niterations, nthreads, regularize,
               norm_r, is_pixels_in_log, real_norms=False):
    return _reconstruct(N.CGLS_TV, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, regularize, norm_r, real_norms=real_norms)


_ALGS = {"cgls": N.CGLS, "sirt": N.SIRT, "mlem": N.MLEM, "cgls_tikhonov": N.CGLS_TIKHONOV,
         "cgls_TVreg": N.CGLS_TV}


def reconstruct_batched(algorithm, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, regularize=None):
    """Many independent problems of uneven sizes in one go (no reference
    counterpart; each result equals the single call ``algorithm(pixels[i],
    angles[i], rotation_centre[i], resolution, niterations, nthreads,
    [regularize[i], zeros,] is_pixels_in_log)``).

    algorithm: "cgls", "sirt", "mlem", "cgls_tikhonov" or "cgls_TVreg";
    pixels / angles: sequences of (n_angles, n_v, n_h) arrays and angle
    lists; rotation_centre: a number or one per problem; regularize: one
    weight per problem for the regularised solvers.  Returns the list of
    volumes.  Every problem's kernels go into one CUDA graph per iteration.
    """
    del nthreads
    if algorithm not in _ALGS:
        raise ValueError(f"unknown algorithm {algorithm!r}")
    n = len(pixels)
    if len(angles) != n:
        raise ValueError("pixels and angles must have the same length")
    pix = [N.f32(p, "pixels", 3) for p in pixels]
    ang = [N.f32(a, "angles", 1) for a in angles]
    cor = np.broadcast_to(np.asarray(rotation_centre, np.float64), (n,)).copy()
    na = np.array([p.shape[0] for p in pix], np.int32)
    nv = np.array([p.shape[1] for p in pix], np.int32)
    nh = np.array([p.shape[2] for p in pix], np.int32)
    for i in range(n):
        if ang[i].shape[0] != na[i]:
            raise ValueError(f"problem {i}: number of projections ({na[i]}) doesn't match "
                             f"angle array ({ang[i].shape[0]})")
    reg = None
    if regularize is not None:
        reg = np.broadcast_to(np.asarray(regularize, np.float64), (n,)).copy()
    outs = []
    for i in range(n):
        gx, gy, gz, _, _ = grid(na[i], nv[i], nh[i], cor[i], resolution)
        outs.append(np.zeros((gx, gy, gz), np.float32))
    ptrs = lambda arrs: (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])  # noqa: E731
    N.check(N.lib.ccpi_pb_reconstruct_batched(
        n, _ALGS[algorithm], ptrs(pix), na, nv, nh, ptrs(ang), cor, int(resolution),
        int(niterations), int(bool(is_pixels_in_log)),
        reg.ctypes.data if reg is not None else None, ptrs(outs)), "batched reconstruction")
    return outs


# ---- warm-start forms (diamond_wrapper.cpp:140-411): the previous volume
# is copied, never modified.  CGLS restarts its Krylov recursion from the
# data (the residual ignores x0), MLEM resets x to 1, SIRT continues.
def cgls_step(pixels, angles, rotation_centre, resolution, niterations, nthreads,
              is_pixels_in_log, last_iteration_volume):
    return _reconstruct(N.CGLS, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, x0=last_iteration_volume)


def cgls_conv_step(pixels, angles, rotation_centre, resolution, niterations, nthreads, norm_r,
                   is_pixels_in_log, last_iteration_volume, real_norms=False):
    return _reconstruct(N.CGLS, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, norm_r=norm_r, x0=last_iteration_volume,
                        real_norms=real_norms)


def sirt_step(pixels, angles, rotation_centre, resolution, niterations, nthreads,
              is_pixels_in_log, last_iteration_volume):
    return _reconstruct(N.SIRT, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, x0=last_iteration_volume)


def mlem_step(pixels, angles, rotation_centre, resolution, niterations, nthreads,
              is_pixels_in_log, last_iteration_volume):
    return _reconstruct(N.MLEM, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, x0=last_iteration_volume)


def cgls_tikhonov_step(pixels, angles, rotation_centre, resolution, niterations, nthreads,
                       regularize, norm_r, is_pixels_in_log, last_iteration_volume,
                       real_norms=False):
    return _reconstruct(N.CGLS_TIKHONOV, pixels, angles, rotation_centre, resolution,
                        niterations, nthreads, is_pixels_in_log, regularize, norm_r,
                        x0=last_iteration_volume, real_norms=real_norms)


def cgls_TVreg_step(pixels, angles, rotation_centre, resolution, niterations, nthreads,
                    regularize, norm_r, is_pixels_in_log, last_iteration_volume,
                    real_norms=False):
    return _reconstruct(N.CGLS_TV, pixels, angles, rotation_centre, resolution, niterations,
                        nthreads, is_pixels_in_log, regularize, norm_r,
                        x0=last_iteration_volume, real_norms=real_norms)


# ---- projector calls (diamond_wrapper.cpp:421-823)
def pb_forward_project(volume, angles, resolution):
    """Volume (vx, vy, vz) -> projections (n_angles, n_v_padded, max(vx, vy))
    on a detector derived from the volume (centre at width / 2)."""
    vol = N.f32(volume, "volume", 3)
    ang = N.f32(angles, "angles", 1)
    dims = np.zeros(3, np.int32)
    N.check(N.lib.ccpi_pb_forward_project(vol, *vol.shape, ang, ang.shape[0], int(resolution),
                                          None, dims), "pb_forward_project")
    out = np.zeros(tuple(dims), np.float32)
    N.check(N.lib.ccpi_pb_forward_project(vol, *vol.shape, ang, ang.shape[0], int(resolution),
                                          out.ctypes.data, dims), "pb_forward_project")
    return out


def pb_backward_project(stack, angles, rotation_center, resolution):
    """Projections (n_angles, n_v, n_h) -> volume on the reconstruction grid."""
    st = N.f32(stack, "stack", 3)
    ang = N.f32(angles, "angles", 1)
    if ang.shape[0] != st.shape[0]:
        raise ValueError("Number of projections doesn't match angle array")
    dims = np.zeros(3, np.int32)
    N.check(N.lib.ccpi_pb_backward_project(st, *st.shape, ang, float(rotation_center),
                                           int(resolution), None, dims), "pb_backward_project")
    out = np.zeros(tuple(dims), np.float32)
    N.check(N.lib.ccpi_pb_backward_project(st, *st.shape, ang, float(rotation_center),
                                           int(resolution), out.ctypes.data, dims),
            "pb_backward_project")
    return out


def pb_setup_geometry_from_image(volume, angles, resolution):
    vol = np.asarray(volume)
    width = max(vol.shape[0], vol.shape[1])
    na = int(np.asarray(angles).shape[0])
    _, _, _, nvp, _ = grid(na, vol.shape[2], width, width / 2.0, resolution)
    return {"n_angles": na, "n_h": width, "n_v": nvp, "output_volume_x": vol.shape[0],
            "output_volume_y": vol.shape[1], "output_volume_z": vol.shape[2]}


def pb_setup_geometry_from_acquisition(stack, angles, rotation_center, resolution):
    st = np.asarray(stack)
    na = int(np.asarray(angles).shape[0])
    nx, ny, nz, nvp, _ = grid(na, st.shape[1], st.shape[2], rotation_center, resolution)
    return {"n_angles": na, "n_h": st.shape[2], "n_v": nvp, "output_volume_x": nx,
            "output_volume_y": ny, "output_volume_z": nz}
