"""ctypes binding of libccpi_b200.so (the C ABI in include/ccpi_b200.h).

The library is looked up next to the package (``ccpi-reconstruction_b200/``)
or at the path in ``CCPI_B200_LIB``.  A missing library is an ImportError:
the reconstruction path has no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB_PATH = os.environ.get("CCPI_B200_LIB", os.path.join(_PKG_ROOT, "libccpi_b200.so"))

CGLS, SIRT, MLEM, CGLS_TIKHONOV, CGLS_TV = 0, 1, 2, 3, 4
PARALLEL, CONE = 0, 1
SOLVE_PLAIN = 1
RECON_CONE_SCATTER = 1

_c_int, _c_dbl, _vp, _sz = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class Geometry(ctypes.Structure):
    """Mirror of ``ccpi_geometry`` (radians; reference frame and layouts)."""
    _fields_ = [("kind", _c_int), ("n_angles", _c_int), ("n_h", _c_int), ("n_v", _c_int),
                ("angles", _vp), ("h_pixels", _vp), ("v_pixels", _vp),
                ("source", _c_dbl * 3), ("detector_x", _c_dbl),
                ("origin", _c_dbl * 3), ("voxel_size", _c_dbl * 3),
                ("nx", _c_int), ("ny", _c_int), ("nz", _c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libccpi_b200.so not found at {LIB_PATH}; build it with "
            "`make -C ccpi-reconstruction_b200/csrc` (or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    lib.ccpi_last_error.restype = ctypes.c_char_p
    lib.ccpi_version.restype = _c_int
    lib.ccpi_pb_grid.argtypes = [_c_int, _c_int, _c_int, _c_dbl, _c_int, _i32p]
    lib.ccpi_pb_reconstruct.argtypes = [_c_int, _f32p, _c_int, _c_int, _c_int, _f32p, _c_dbl,
                                        _c_int, _c_int, _c_int, _c_int, _c_dbl, _vp, _vp, _f32p]
    lib.ccpi_pb_geometry.argtypes = [_c_int, _c_int, _c_int, _f32p, _c_dbl, _c_int, _f64p,
                                     _f64p, _f64p, P(Geometry)]
    lib.ccpi_pb_pack.argtypes = [_vp, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp]
    lib.ccpi_pb_reconstruct_batched.argtypes = [_c_int, _c_int, P(_vp), _i32p, _i32p, _i32p,
                                                P(_vp), _f64p, _c_int, _c_int, _c_int, _vp,
                                                P(_vp)]
    lib.ccpi_pb_aml_ring_artefacts.argtypes = [_f32p, _c_int, _c_int, _c_int, ctypes.c_float,
                                               ctypes.c_float, _c_int, _f32p]
    lib.ccpi_ring_filter_aml.argtypes = [_vp, _c_int, _c_int, _c_int, _c_dbl, _c_dbl, _c_int,
                                         _vp]
    lib.ccpi_pb_high_peaks.argtypes = [_f32p, _c_int, _c_int, _c_int, _c_dbl, _c_int, _c_int,
                                       _f32p]
    lib.ccpi_pb_column_ring_artefacts.argtypes = [_f32p, _c_int, _c_int, _c_int, _c_int, _f32p]
    lib.ccpi_high_peaks.argtypes = [_vp, _c_int, _c_int, _c_int, _c_dbl, _c_int, _vp]
    lib.ccpi_measure_gather.argtypes = [ctypes.c_ulonglong, _vp, _f64p]
    lib.ccpi_ring_filter_column.argtypes = [_vp, _c_int, _c_int, _c_int, _vp]
    lib.ccpi_pb_forward_project.argtypes = [_f32p, _c_int, _c_int, _c_int, _f32p, _c_int,
                                            _c_int, _vp, _i32p]
    lib.ccpi_pb_backward_project.argtypes = [_f32p, _c_int, _c_int, _c_int, _f32p, _c_dbl,
                                             _c_int, _vp, _i32p]
    lib.ccpi_cb_grid.argtypes = [_c_int, _c_int, _c_int, _c_int] + [_c_dbl] * 5 + [_i32p, _f64p]
    lib.ccpi_cb_find_centre.argtypes = [_f32p, _c_int, _c_int, _c_int, _f32p, _c_dbl, _c_dbl,
                                        _c_dbl, P(_c_dbl)]
    lib.ccpi_cb_reconstruct.argtypes = [_c_int, _f32p, _c_int, _c_int, _c_int, _f32p, _c_int] + \
        [_c_dbl] * 5 + [_c_int, _c_int, _c_int, _c_dbl, _vp, _f32p]
    lib.ccpi_cb_create_sinogram.argtypes = [P(Geometry), _f32p, _f32p]
    lib.ccpi_reconstruct.argtypes = [P(Geometry), _c_int, _vp, _c_int, _c_dbl, _vp, _vp]
    lib.ccpi_reconstruct_flags.argtypes = [P(Geometry), _c_int, _vp, _c_int, _c_dbl, _vp, _vp,
                                           _c_int]
    lib.ccpi_plan_create.argtypes = [P(Geometry), P(_vp)]
    lib.ccpi_plan_autotune.argtypes = [_vp, _vp, _i32p]
    lib.ccpi_plan_set_cone_backprojector.argtypes = [_vp, _c_int]
    lib.ccpi_plan_destroy.argtypes = [_vp]
    lib.ccpi_plan_destroy.restype = None
    lib.ccpi_plan_voxels.argtypes = [_vp]
    lib.ccpi_plan_voxels.restype = ctypes.c_longlong
    lib.ccpi_plan_pixels.argtypes = [_vp]
    lib.ccpi_plan_pixels.restype = ctypes.c_longlong
    lib.ccpi_forward.argtypes = [_vp, _vp, _vp, _vp]
    lib.ccpi_backward.argtypes = [_vp, _vp, _vp, _vp]
    lib.ccpi_forward_batch.argtypes = [_vp, _c_int, _vp, _vp, _vp]
    lib.ccpi_backward_batch.argtypes = [_vp, _c_int, _vp, _vp, _vp]
    lib.ccpi_solve_workspace_bytes.argtypes = [_vp, _c_int, _c_int]
    lib.ccpi_solve_workspace_bytes.restype = _sz
    lib.ccpi_solve.argtypes = [_vp, _c_int, _vp, _vp, _c_int, _c_dbl, _vp, _c_int, _vp, _sz, _vp]
    lib.ccpi_solve_batched.argtypes = [_c_int, P(_vp), _c_int, P(_vp), P(_vp), _c_int, _vp, _vp]
    lib.ccpi_session_create.argtypes = [_vp, _c_int, _vp, _vp, _c_dbl, _c_int, _c_int, _vp,
                                        P(_vp)]
    lib.ccpi_session_run.argtypes = [_vp, _c_int]
    lib.ccpi_session_finish.argtypes = [_vp, _vp]
    lib.ccpi_session_destroy.argtypes = [_vp]
    lib.ccpi_session_destroy.restype = None
    lib.ccpi_shard_create.argtypes = [_vp, _c_int, _vp, _vp, _c_dbl, _c_int, _vp, _vp, _vp,
                                      _vp, _vp, P(_vp)]
    lib.ccpi_shard_stage.argtypes = [_vp, _c_int]
    lib.ccpi_shard_finish.argtypes = [_vp, _vp]
    lib.ccpi_shard_destroy.argtypes = [_vp]
    lib.ccpi_shard_destroy.restype = None
    return lib


lib = _load()


def check(rc: int, what: str):
    if rc != 0:
        msg = lib.ccpi_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")


def f32(a, name, ndim):
    """float32, C-contiguous view or copy of an array with `ndim` dimensions
    (the reference reinterprets its buffers without checks; this raises)."""
    arr = np.asarray(a)
    if arr.ndim != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions, got shape {arr.shape}")
    if not np.issubdtype(arr.dtype, np.floating) and not np.issubdtype(arr.dtype, np.integer):
        raise TypeError(f"{name} must be a real array, got {arr.dtype}")
    return np.ascontiguousarray(arr, dtype=np.float32)
