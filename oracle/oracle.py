"""Python access to the CPU oracles (TEST INFRASTRUCTURE ONLY).

Two libraries, both built by ``oracle/Makefile``:

* ``oracle/librestate.so`` -- this project's CPU restatement of the
  reference's projectors and solvers (``oracle/restate.cpp``), float build
  (the reference's arithmetic, bit for bit) and double build (FP64 oracle).
* ``oracle/_ref/libccpi_ref.so`` -- the reference's own iterative core
  (CCPi-Reconstruction ``Core/src``) compiled from its sources, with C entry
  points mirroring its Python wrappers (``oracle/ref_harness.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.

Geometry helpers here restate the reference's numpy front-ends
(``Core/src/diamond.cpp:35-86,394-501``, ``Core/src/instruments.cpp:35-64``,
``Core/src/Readers/xtek.cpp:57-129,367-380,760-798``) so that the
restatement can be driven with the same inputs as the Python API.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATE_SO = os.path.join(HERE, "librestate.so")
REF_SO = os.path.join(HERE, "_ref", "libccpi_ref.so")

CGLS, SIRT, MLEM, TIKHONOV, TV = 0, 1, 2, 3, 4
ALG_NAMES = {"cgls": CGLS, "sirt": SIRT, "mlem": MLEM,
             "cgls_tikhonov": TIKHONOV, "cgls_TVreg": TV}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_c_int, _c_dbl, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


class _RsGeometry(ctypes.Structure):
    _fields_ = [("kind", _c_int), ("na", _c_int), ("nh", _c_int), ("nv", _c_int),
                ("angles", _vp), ("h_pixels", _vp), ("v_pixels", _vp),
                ("source", _c_dbl * 3), ("detector_x", _c_dbl),
                ("origin", _c_dbl * 3), ("size", _c_dbl * 3),
                ("nx", _c_int), ("ny", _c_int), ("nz", _c_int)]


@dataclass
class Geometry:
    """Explicit projector geometry (radians, reference layouts)."""
    kind: int  # 0 parallel, 1 cone
    angles: np.ndarray
    h_pixels: np.ndarray
    v_pixels: np.ndarray
    origin: tuple
    size: tuple
    shape: tuple  # (nx, ny, nz)
    source: tuple = (0.0, 0.0, 0.0)
    detector_x: float = 0.0
    _keep: list = field(default_factory=list, repr=False)

    @property
    def sino_shape(self):
        return (len(self.angles), len(self.h_pixels), len(self.v_pixels))

    def c_struct(self) -> _RsGeometry:
        a = np.ascontiguousarray(self.angles, np.float64)
        h = np.ascontiguousarray(self.h_pixels, np.float64)
        v = np.ascontiguousarray(self.v_pixels, np.float64)
        self._keep = [a, h, v]
        g = _RsGeometry()
        g.kind = self.kind
        g.na, g.nh, g.nv = len(a), len(h), len(v)
        g.angles, g.h_pixels, g.v_pixels = a.ctypes.data, h.ctypes.data, v.ctypes.data
        g.source = (_c_dbl * 3)(*self.source)
        g.detector_x = float(self.detector_x)
        g.origin = (_c_dbl * 3)(*self.origin)
        g.size = (_c_dbl * 3)(*self.size)
        g.nx, g.ny, g.nz = self.shape
        return g


# --------------------------------------------------------------- restatement
_rs = None


def restate():
    global _rs
    if _rs is None:
        if not os.path.exists(RESTATE_SO):
            raise FileNotFoundError(f"{RESTATE_SO} missing: run `make -C oracle`")
        lib = ctypes.CDLL(RESTATE_SO)
        gp = ctypes.POINTER(_RsGeometry)
        for suf, p in (("f32", _f32p), ("f64", _f64p)):
            getattr(lib, f"rs_fp_{suf}").argtypes = [gp, p, p]
            getattr(lib, f"rs_bp_{suf}").argtypes = [gp, p, p]
            fn = getattr(lib, f"rs_solve_{suf}")
            fn.argtypes = [gp, _c_int, p, p, _c_int, _c_dbl, _vp]
            fn.restype = _c_int
            getattr(lib, f"rs_regularize_{suf}").argtypes = [_c_int, _c_int, _c_int, _c_int, p, p]
        lib.rs_neglog_f32.argtypes = [_f32p, _f32p, ctypes.c_longlong]
        lib.rs_expneg_f32.argtypes = [_f32p, _f32p, ctypes.c_longlong]
        lib.rs_aml_ring_f32.argtypes = [_f32p, _c_int, _c_int, _c_int, _c_dbl, _c_dbl, _c_int]
        lib.rs_high_peaks_f32.argtypes = [_f32p, _c_int, _c_int, _c_int, _c_dbl, _c_int]
        lib.rs_high_peaks_f32.restype = _c_int
        lib.rs_column_ring_f32.argtypes = [_f32p, _c_int, _c_int, _c_int]
        _rs = lib
    return _rs


def _dt(fp64):
    return (np.float64, "f64") if fp64 else (np.float32, "f32")


def forward(geom: Geometry, vol, fp64=False):
    dt, suf = _dt(fp64)
    vol = np.ascontiguousarray(vol, dt)
    out = np.zeros(geom.sino_shape, dt)
    g = geom.c_struct()
    getattr(restate(), f"rs_fp_{suf}")(ctypes.byref(g), vol, out)
    return out


def backward(geom: Geometry, pix, fp64=False):
    dt, suf = _dt(fp64)
    pix = np.ascontiguousarray(pix, dt)
    out = np.zeros(geom.shape, dt)
    g = geom.c_struct()
    getattr(restate(), f"rs_bp_{suf}")(ctypes.byref(g), pix, out)
    return out


def solve(geom: Geometry, alg: int, sino, niter, lam=0.0, x0=None, fp64=False,
          want_norms=False):
    dt, suf = _dt(fp64)
    sino = np.ascontiguousarray(sino, dt)
    x = np.zeros(geom.shape, dt) if x0 is None else np.array(x0, dt, order="C")
    norms = np.zeros(max(niter, 1), np.float64)
    g = geom.c_struct()
    rc = getattr(restate(), f"rs_solve_{suf}")(ctypes.byref(g), alg, sino, x, niter,
                                               float(lam), norms.ctypes.data)
    if rc:
        raise RuntimeError(f"rs_solve failed ({rc})")
    return (x, norms[:niter]) if want_norms else x


def neglog(p):
    """-log(p) with the C library's logf (the reference's float log)."""
    p = np.ascontiguousarray(p, np.float32)
    out = np.empty_like(p)
    restate().rs_neglog_f32(p, out, p.size)
    return out


def expneg(p):
    """exp(-p) with the C library's expf (the reference wrapper's way back
    from logs to transmission)."""
    p = np.ascontiguousarray(p, np.float32)
    out = np.empty_like(p)
    restate().rs_expneg_f32(p, out, p.size)
    return out


def regularize(alg, a, fp64=False):
    dt, suf = _dt(fp64)
    a = np.ascontiguousarray(a, dt)
    b = np.zeros_like(a)
    getattr(restate(), f"rs_regularize_{suf}")(alg, *a.shape, a, b)
    return b


# ----------------------------------------------------- numpy front-end rules
def v_alignment(n, ppv, cone=False, align=4):
    """instrument::calc_v_alignment (Core/src/instruments.cpp:35-64) with the
    conda build's 16-byte alignment (4 floats).  Returns (n_padded, offset)."""
    nvox = -(-n // ppv)
    blocks = -(-nvox // align)
    if cone and blocks % 2:
        blocks += 1
    npix = blocks * align * ppv
    return npix, (npix - n) // 2


def parallel_api_geometry(na, nv, nh, angles_deg, cor, ppv):
    """Diamond numpy geometry and voxel grid (diamond.cpp:35-86, :453-501,
    voxels.cpp:12-46).  Returns (Geometry, nv_pad, v_offset)."""
    nv_pad, voff = v_alignment(nv, ppv)
    shift = (cor - nh / 2.0) if cor > 0.0 else 0.0
    h0 = -((nh - 1) * 1.0) / 2.0 - shift
    h = h0 + np.arange(nh, dtype=np.float64) * 1.0
    v0 = -((nv_pad - 1) * 1.0) / 2.0
    v = v0 + np.arange(nv_pad, dtype=np.float64) * 1.0
    ang = math.pi * (np.asarray(angles_deg, np.float32).astype(np.float64) / 180.0)
    hrange = h[1] - h[0]
    hmax = max(abs(h[0]), abs(h[-1]))
    n = int(math.ceil((2.0 * hmax) / hrange))
    nx = -(-n // ppv)
    hvox = hrange * ppv
    while (-hvox * nx / 2.0 >= h[0]) or (hvox * nx / 2.0 <= h[-1]):
        nx += 1
    vvox = (v[1] - v[0]) * ppv
    nz = -(-nv_pad // ppv)
    size = (hvox, hvox, vvox)
    origin = tuple(-size[i] * n_ / 2.0 for i, n_ in enumerate((nx, nx, nz)))
    g = Geometry(0, ang, h, v, origin, size, (nx, nx, nz))
    return g, nv_pad, voff


def parallel_api_sinogram(pixels, nv_pad, voff, is_log):
    """Diamond::read_scans (diamond.cpp:394-451): (na, nv, nh) numpy ->
    (na, nh, nv_pad) with zero padding rows and -log when not in log."""
    p = np.asarray(pixels, np.float32)
    na, nv, nh = p.shape
    out = np.zeros((na, nh, nv_pad), np.float32)
    data = p if is_log else neglog(p)
    out[:, :, voff:voff + nv] = np.transpose(data, (0, 2, 1))
    return out


# ------------------------------------------------------------ reference .so
_ref = None


class quiet:
    """Silence the reference's progress and error prints (it writes to the
    process's stdout/stderr from C++) for the duration of a call."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        sys.stderr.flush()
        self._saved = (os.dup(1), os.dup(2))
        null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(null, 1)
        os.dup2(null, 2)
        os.close(null)
        return self

    def __exit__(self, *exc):
        os.dup2(self._saved[0], 1)
        os.dup2(self._saved[1], 2)
        os.close(self._saved[0])
        os.close(self._saved[1])
        return False


def reference_available():
    return os.path.exists(REF_SO)


def reference():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle ref`")
        lib = ctypes.CDLL(REF_SO)
        lib.ref_set_pad_factor.argtypes = [_c_dbl]
        lib.ref_pb_geometry.argtypes = [_c_int, _c_int, _c_int, _c_dbl, _c_int, _i32p, _f64p]
        lib.ref_pb_reconstruct.argtypes = [_c_int, _f32p, _c_int, _c_int, _c_int, _f32p, _c_dbl,
                                           _c_int, _c_int, _c_int, _c_int, _c_dbl, _vp, _f32p]
        lib.ref_pb_forward_project.argtypes = [_f32p, _c_int, _c_int, _c_int, _f32p, _c_int,
                                               _c_int, _vp, ctypes.POINTER(_c_int)]
        lib.ref_pb_backward_project.argtypes = [_f32p, _c_int, _c_int, _c_int, _f32p, _c_dbl,
                                                _c_int, _f32p]
        for nm in ("ref_pb_f2d", "ref_pb_b2d"):
            getattr(lib, nm).argtypes = [_f64p, _c_int, _f64p, _c_int, _f64p, _c_int, _f64p,
                                         _f64p, _c_int, _c_int, _c_int, _f32p, _f32p]
        for nm in ("ref_cb_f2d", "ref_cb_b2d"):
            getattr(lib, nm).argtypes = [_c_dbl] * 4 + [_f64p, _c_int, _f64p, _c_int, _f64p,
                                                        _c_int, _f64p, _f64p, _c_int, _c_int,
                                                        _c_int, _f32p, _f32p]
        lib.ref_cb_geometry.argtypes = [_vp, _c_int, _c_int, _c_int, _vp, _c_int] + \
            [_c_dbl] * 5 + [_c_int, _i32p, _f64p]
        lib.ref_cb_reconstruct.argtypes = [_c_int, _f32p, _c_int, _c_int, _c_int, _f32p,
                                           _c_int] + [_c_dbl] * 5 + [_c_int, _c_int, _c_int,
                                                                     _c_dbl, _f32p]
        lib.ref_cb_phantom_volume.argtypes = [_f32p, _f32p, _f32p, _f32p, _f64p]
        lib.ref_aml_ring.argtypes = [_f32p, _c_int, _c_int, _c_int, _c_dbl, _c_dbl, _c_int]
        lib.ref_high_peaks.argtypes = [_f32p, _c_int, _c_int, _c_int, _c_dbl, _c_int]
        lib.ref_column_ring.argtypes = [_f32p, _c_int, _c_int, _c_int]
        lib.ref_aml_ring_artefacts.argtypes = [_f32p, _c_int, _c_int, _c_int, ctypes.c_float,
                                               ctypes.c_float, _c_int, _f32p]
        lib.ref_cb_solve_explicit.argtypes = [_c_int] + [_c_dbl] * 4 + [
            _f64p, _c_int, _f64p, _c_int, _f64p, _c_int, _f32p, _f64p, _f64p, _c_int, _c_int,
            _c_int, _c_int, _c_dbl, _c_int, _f32p]
        _ref = lib
    return _ref


def ref_forward(geom: Geometry, vol):
    lib = reference()
    vol = np.ascontiguousarray(vol, np.float32)
    out = np.zeros(geom.sino_shape, np.float32)
    a, h, v = (np.ascontiguousarray(x, np.float64) for x in (geom.angles, geom.h_pixels, geom.v_pixels))
    o, s = np.array(geom.origin, np.float64), np.array(geom.size, np.float64)
    if geom.kind == 0:
        lib.ref_pb_f2d(h, len(h), v, len(v), a, len(a), o, s, *geom.shape, vol, out)
    else:
        lib.ref_cb_f2d(*geom.source, geom.detector_x, h, len(h), v, len(v), a, len(a), o, s,
                       *geom.shape, vol, out)
    return out


def ref_backward(geom: Geometry, pix):
    lib = reference()
    pix = np.ascontiguousarray(pix, np.float32)
    out = np.zeros(geom.shape, np.float32)
    a, h, v = (np.ascontiguousarray(x, np.float64) for x in (geom.angles, geom.h_pixels, geom.v_pixels))
    o, s = np.array(geom.origin, np.float64), np.array(geom.size, np.float64)
    if geom.kind == 0:
        lib.ref_pb_b2d(h, len(h), v, len(v), a, len(a), o, s, *geom.shape, pix, out)
    else:
        lib.ref_cb_b2d(*geom.source, geom.detector_x, h, len(h), v, len(v), a, len(a), o, s,
                       *geom.shape, pix, out)
    return out


def ref_pb_geometry(na, nv, nh, cor, ppv):
    dims = np.zeros(4, np.int32)
    geom = np.zeros(4, np.float64)
    rc = reference().ref_pb_geometry(na, nv, nh, float(cor), ppv, dims, geom)
    if rc:
        raise RuntimeError("reference geometry failed")
    return dims, geom


def ref_pb_reconstruct(alg, pixels, angles_deg, cor, ppv, niter, is_log, lam=0.0, x0=None,
                       nthreads=1):
    pixels = np.ascontiguousarray(pixels, np.float32)
    na, nv, nh = pixels.shape
    dims, _ = ref_pb_geometry(na, nv, nh, cor, ppv)
    out = np.zeros(tuple(dims[:3]), np.float32)
    # cgls_regularize::reconstruct updates r_vox (a volume) with sinogram
    # extents (Core/src/Algorithms/cgls.cpp:386): pad every allocation by
    # the overrun ratio so that those writes land in padding
    pad = _reg_pad(alg, na * nh * int(dims[3]), int(dims[0]) * int(dims[1]) * int(dims[2]))
    x0p = None
    if x0 is not None:
        x0 = np.ascontiguousarray(x0, np.float32)
        x0p = x0.ctypes.data
    reference().ref_set_pad_factor(pad)
    try:
        rc = reference().ref_pb_reconstruct(alg, pixels, na, nv, nh,
                                            np.ascontiguousarray(angles_deg, np.float32),
                                            float(cor), ppv, niter, nthreads, int(bool(is_log)),
                                            float(lam), x0p, out)
    finally:
        reference().ref_set_pad_factor(0.0)
    if rc:
        raise RuntimeError(f"reference reconstruct failed ({rc})")
    return out


def ref_pb_forward_project(volume, angles_deg, ppv):
    volume = np.ascontiguousarray(volume, np.float32)
    vx, vy, vz = volume.shape
    na = len(angles_deg)
    a = np.ascontiguousarray(angles_deg, np.float32)
    nvp = _c_int(0)
    lib = reference()
    lib.ref_pb_forward_project(volume, vx, vy, vz, a, na, ppv, None, ctypes.byref(nvp))
    out = np.zeros((na, nvp.value, max(vx, vy)), np.float32)
    lib.ref_pb_forward_project(volume, vx, vy, vz, a, na, ppv, out.ctypes.data, ctypes.byref(nvp))
    return out


def ref_pb_backward_project(stack, angles_deg, cor, ppv):
    stack = np.ascontiguousarray(stack, np.float32)
    na, nv, nh = stack.shape
    dims, _ = ref_pb_geometry(na, nv, nh, cor, ppv)
    out = np.zeros(tuple(dims[:3]), np.float32)
    reference().ref_pb_backward_project(stack, na, nv, nh,
                                        np.ascontiguousarray(angles_deg, np.float32), float(cor),
                                        ppv, out)
    return out


def ref_cb_geometry(na, nh, nv, ppv, s2s, s2d, px_h, px_v, mask_radius, pixels=None,
                    angles_deg=None, is_log=True):
    dims = np.zeros(4, np.int32)
    geom = np.zeros(7, np.float64)
    pp = None if pixels is None else np.ascontiguousarray(pixels, np.float32)
    ap = None if angles_deg is None else np.ascontiguousarray(angles_deg, np.float32)
    rc = reference().ref_cb_geometry(None if pp is None else pp.ctypes.data, na, nh, nv,
                                     None if ap is None else ap.ctypes.data, ppv, float(s2s),
                                     float(s2d), float(px_h), float(px_v), float(mask_radius),
                                     int(bool(is_log)), dims, geom)
    if rc:
        raise RuntimeError(f"reference cone geometry failed ({rc})")
    return dims, geom


def _reg_pad(alg, n_pix, n_vox):
    """Padding factor for the reference's allocations in its regularised
    CGLS: cgls_regularize::reconstruct updates r_vox (a volume) with
    sinogram extents (Core/src/Algorithms/cgls.cpp:386), so every allocation
    is padded by the overrun ratio and those writes land in padding."""
    return max(0.0, n_pix / max(n_vox, 1) - 1.0) + 0.05 if alg in (3, 4) else 0.0


def ref_cb_reconstruct(alg, pixels, angles_deg, ppv, s2s, s2d, px_h, px_v, mask_radius, niter,
                       is_log, lam=0.0, nthreads=1):
    pixels = np.ascontiguousarray(pixels, np.float32)
    na, nh, nv = pixels.shape
    dims, _ = ref_cb_geometry(na, nh, nv, ppv, s2s, s2d, px_h, px_v, mask_radius)
    out = np.zeros(tuple(dims[:3]), np.float32)
    reference().ref_set_pad_factor(
        _reg_pad(alg, na * nh * int(dims[3]), int(dims[0]) * int(dims[1]) * int(dims[2])))
    try:
        rc = reference().ref_cb_reconstruct(alg, pixels, na, nh, nv,
                                            np.ascontiguousarray(angles_deg, np.float32), ppv,
                                            float(s2s), float(s2d), float(px_h), float(px_v),
                                            float(mask_radius), niter, nthreads,
                                            int(bool(is_log)), float(lam), out)
    finally:
        reference().ref_set_pad_factor(0.0)
    if rc:
        raise RuntimeError(f"reference cone reconstruct failed ({rc})")
    return out


def ref_cb_solve_explicit(geom: Geometry, alg, sino, niter, lam=0.0, nthreads=1):
    lib = reference()
    a, h, v = (np.ascontiguousarray(x, np.float64) for x in (geom.angles, geom.h_pixels, geom.v_pixels))
    out = np.zeros(geom.shape, np.float32)
    lib.ref_set_pad_factor(_reg_pad(alg, len(a) * len(h) * len(v), int(np.prod(geom.shape))))
    try:
        rc = lib.ref_cb_solve_explicit(alg, *geom.source, geom.detector_x, h, len(h), v, len(v),
                                       a, len(a), np.ascontiguousarray(sino, np.float32),
                                       np.array(geom.origin, np.float64),
                                       np.array(geom.size, np.float64), *geom.shape, niter,
                                       float(lam), nthreads, out)
    finally:
        lib.ref_set_pad_factor(0.0)
    if rc:
        raise RuntimeError(f"reference explicit cone solve failed ({rc})")
    return out


# ------------------------------------------------------- synthetic geometries
def cone_geometry(n_vox, vox_size, n_angles, n_det, pix_size, s2o, o2d, full_circle=True,
                  n_det_v=None):
    """Explicit cone geometry in the reference's frame: source at (-s2o,0,0),
    detector plane at x = o2d, centred voxel grid and detector."""
    nv = n_det if n_det_v is None else n_det_v
    span = 2.0 * math.pi if full_circle else math.pi
    ang = np.arange(n_angles, dtype=np.float64) * (span / n_angles)
    h = (np.arange(n_det, dtype=np.float64) - (n_det - 1) / 2.0) * pix_size
    v = (np.arange(nv, dtype=np.float64) - (nv - 1) / 2.0) * pix_size
    nx, ny, nz = (n_vox,) * 3 if np.isscalar(n_vox) else n_vox
    size = (vox_size,) * 3
    origin = (-nx * vox_size / 2.0, -ny * vox_size / 2.0, -nz * vox_size / 2.0)
    return Geometry(1, ang, h, v, origin, size, (nx, ny, nz), source=(-s2o, 0.0, 0.0),
                    detector_x=o2d)


def parallel_geometry(shape, n_angles, nh, nv=None, cor_shift=0.0, span=math.pi):
    """Explicit parallel geometry: unit pixels, centred grid and detector,
    detector column i at i - (nh-1)/2 - cor_shift."""
    nx, ny, nz = shape
    nv = nz if nv is None else nv
    ang = np.arange(n_angles, dtype=np.float64) * (span / n_angles)
    h = np.arange(nh, dtype=np.float64) - (nh - 1) / 2.0 - cor_shift
    v = np.arange(nv, dtype=np.float64) - (nv - 1) / 2.0
    return Geometry(0, ang, h, v, (-nx / 2.0, -ny / 2.0, -nz / 2.0), (1.0, 1.0, 1.0),
                    (nx, ny, nz))


# ------------------------------------------------------- AML ring filter
def aml_ring(p, param_n, param_r, num_series):
    """The restatement's AML ring filter on a log sinogram (na, nh, nv);
    returns the filtered copy (Core/src/diamond.cpp:660-808)."""
    lib = restate()
    out = np.array(p, np.float32, order="C")
    na, nh, nv = out.shape
    rc = lib.rs_aml_ring_f32(out, na, nh, nv, float(param_n), float(param_r), int(num_series))
    if rc:
        raise ValueError("AML ring filter: parameters out of range")
    return out


def ref_aml_ring(p, param_n, param_r, num_series):
    """The reference's remove_aml_ring_artefacts on a log sinogram (na, nh, nv)."""
    out = np.array(p, np.float32, order="C")
    na, nh, nv = out.shape
    with quiet():
        reference().ref_aml_ring(out, na, nh, nv, float(param_n), float(param_r),
                                 int(num_series))
    return out


def ref_aml_ring_artefacts(pixels, param_n, param_r, num_series):
    """parallelbeam.filters.aml_ring_artefacts as the reference's wrapper
    computes it: (na, nv, nh) transmission in and out."""
    pixels = np.ascontiguousarray(pixels, np.float32)
    na, nv, nh = pixels.shape
    out = np.zeros_like(pixels)
    with quiet():
        reference().ref_aml_ring_artefacts(pixels, na, nv, nh, float(param_n), float(param_r),
                                           int(num_series), out)
    return out


# ------------------------------------- high-peaks and column ring filters
def high_peaks(p, jump, num_pix):
    """The restatement's high-peaks filter on a log sinogram (na, nh, nv);
    returns the filtered copy (Core/src/diamond.cpp:513-617)."""
    out = np.array(p, np.float32, order="C")
    na, nh, nv = out.shape
    if restate().rs_high_peaks_f32(out, na, nh, nv, float(jump), int(num_pix)):
        raise ValueError("high peaks filter: parameters out of range")
    return out


def column_ring(p):
    """The restatement's column ring filter on a log sinogram (na, nh, nv);
    returns the filtered copy (Core/src/diamond.cpp:619-658)."""
    out = np.array(p, np.float32, order="C")
    na, nh, nv = out.shape
    restate().rs_column_ring_f32(out, na, nh, nv)
    return out


def ref_high_peaks(p, jump, num_pix):
    """The reference's Diamond::high_peaks_before on (na, nh, nv) logs."""
    out = np.array(p, np.float32, order="C")
    na, nh, nv = out.shape
    with quiet():
        reference().ref_high_peaks(out, na, nh, nv, float(jump), int(num_pix))
    return out


def ref_column_ring(p):
    """The reference's remove_column_ring_artefacts on (na, nh, nv) logs."""
    out = np.array(p, np.float32, order="C")
    na, nh, nv = out.shape
    with quiet():
        reference().ref_column_ring(out, na, nh, nv)
    return out


def ref_cb_phantom_volume():
    """conebeam.create_phantom_volume from the reference: (vol, angles deg,
    h_pixels, v_pixels, source_x, detector_x, pixel_h, pixel_v,
    mask_radius)."""
    vol = np.zeros((512, 512, 512), np.float32)
    ang = np.zeros(250, np.float32)
    h = np.zeros(512, np.float32)
    v = np.zeros(512, np.float32)
    sc = np.zeros(5, np.float64)
    with quiet():
        reference().ref_cb_phantom_volume(vol, ang, h, v, sc)
    return (vol, ang, h, v) + tuple(float(x) for x in sc)
