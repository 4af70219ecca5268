"""Device-level access: plans, projectors and solvers on torch CUDA tensors.

PyTorch is only the plumbing here (device memory and the current stream);
every operation is a call into libccpi_b200.so.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native as N


class Plan:
    """Device tables of one explicit geometry (``ccpi_plan_create``).

    kind: "parallel" or "cone"; angles in radians; h_pixels / v_pixels the
    detector coordinates; origin / voxel_size / shape the voxel grid.
    """

    def __init__(self, kind, angles, h_pixels, v_pixels, origin, voxel_size, shape,
                 source=(0.0, 0.0, 0.0), detector_x=0.0):
        self.kind = kind
        self._arrays = [np.ascontiguousarray(x, np.float64) for x in (angles, h_pixels, v_pixels)]
        g = N.Geometry()
        g.kind = N.PARALLEL if kind == "parallel" else N.CONE
        g.angles, g.h_pixels, g.v_pixels = (a.ctypes.data for a in self._arrays)
        g.n_angles, g.n_h, g.n_v = (len(a) for a in self._arrays)
        g.source = (ctypes.c_double * 3)(*source)
        g.detector_x = float(detector_x)
        g.origin = (ctypes.c_double * 3)(*origin)
        g.voxel_size = (ctypes.c_double * 3)(*voxel_size)
        g.nx, g.ny, g.nz = shape
        self.shape = tuple(int(s) for s in shape)
        self.sino_shape = (g.n_angles, g.n_h, g.n_v)
        self.geometry = g
        h = ctypes.c_void_p()
        N.check(N.lib.ccpi_plan_create(ctypes.byref(g), ctypes.byref(h)), "ccpi_plan_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def autotune(self, device=None):
        """Pick the fastest projector launch shapes for this plan
        (``ccpi_plan_autotune``); call before solving.  Returns the choice
        (grid or cone rows per lane, back projector slices per lane or 0)."""
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else device
        chosen = np.zeros(2, np.int32)
        N.check(N.lib.ccpi_plan_autotune(self._h,
                                         ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream),
                                         chosen), "ccpi_plan_autotune")
        return int(chosen[0]), int(chosen[1])

    def set_cone_backprojector(self, scatter):
        """Cone beam: 1 = ray-driven scatter back projector (float atomics),
        0 = the deterministic voxel gather (``ccpi_plan_set_cone_backprojector``)."""
        N.check(N.lib.ccpi_plan_set_cone_backprojector(self._h, int(bool(scatter))),
                "ccpi_plan_set_cone_backprojector")

    def close(self):
        if self._h:
            N.lib.ccpi_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _stream(t):
        return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)

    def _check(self, t, shape, name):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
        if tuple(t.shape[-3:]) != tuple(shape):
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {shape}")

    def forward(self, vol, out=None):
        """out = A vol on torch's current stream."""
        self._check(vol, self.shape, "volume")
        if out is None:
            out = torch.empty(self.sino_shape, device=vol.device, dtype=torch.float32)
        self._check(out, self.sino_shape, "sinogram")
        N.check(N.lib.ccpi_forward(self._h, ctypes.c_void_p(vol.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), self._stream(vol)),
                "ccpi_forward")
        return out

    def backward(self, sino, out=None):
        """out = A^T sino on torch's current stream."""
        self._check(sino, self.sino_shape, "sinogram")
        if out is None:
            out = torch.empty(self.shape, device=sino.device, dtype=torch.float32)
        self._check(out, self.shape, "volume")
        N.check(N.lib.ccpi_backward(self._h, ctypes.c_void_p(sino.data_ptr()),
                                    ctypes.c_void_p(out.data_ptr()), self._stream(sino)),
                "ccpi_backward")
        return out

    def _batch(self, name, src, out, in_shape, out_shape):
        if src.dim() != 4 or out.dim() != 4 or src.shape[0] != out.shape[0]:
            raise ValueError(f"{name}: expected (n, ...) input and output of one batch size")
        self._check(src, in_shape, "input")
        self._check(out, out_shape, "output")
        N.check(getattr(N.lib, name)(self._h, int(src.shape[0]), ctypes.c_void_p(src.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), self._stream(src)), name)
        return out

    def forward_batch(self, vol, out):
        """out[b] = A vol[b] for a (n, nx, ny, nz) batch (``ccpi_forward_batch``)."""
        return self._batch("ccpi_forward_batch", vol, out, self.shape, self.sino_shape)

    def backward_batch(self, sino, out):
        """out[b] = A^T sino[b] for a (n, n_angles, n_h, n_v) batch."""
        return self._batch("ccpi_backward_batch", sino, out, self.sino_shape, self.shape)

    def workspace_bytes(self, alg, niterations):
        return int(N.lib.ccpi_solve_workspace_bytes(self._h, int(alg), int(niterations)))

    def solve(self, alg, sino, x, niterations, regularize=0.0, plain=False, workspace=None,
              want_norms=False):
        """Run a solver in place on x (blocking)."""
        self._check(sino, self.sino_shape, "sinogram")
        self._check(x, self.shape, "volume")
        norms = np.zeros(max(int(niterations), 1), np.float64)
        ws, wsb = None, 0
        if workspace is not None:
            ws, wsb = ctypes.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
        N.check(N.lib.ccpi_solve(self._h, int(alg), ctypes.c_void_p(sino.data_ptr()),
                                 ctypes.c_void_p(x.data_ptr()), int(niterations),
                                 float(regularize), norms.ctypes.data,
                                 N.SOLVE_PLAIN if plain else 0, ws, wsb, self._stream(x)),
                "ccpi_solve")
        return (x, norms[:niterations]) if want_norms else x


class Session:
    """A prepared solver (``ccpi_session_*``): set-up once, then run
    iterations in graph launches on torch's current stream."""

    def __init__(self, plan, alg, sino, x, max_iterations, regularize=0.0, plain=False):
        plan._check(sino, plan.sino_shape, "sinogram")
        plan._check(x, plan.shape, "volume")
        self.plan, self.sino, self.x = plan, sino, x
        self.alg = int(alg)
        self.done = 0
        h = ctypes.c_void_p()
        N.check(N.lib.ccpi_session_create(plan.handle, self.alg, ctypes.c_void_p(sino.data_ptr()),
                                          ctypes.c_void_p(x.data_ptr()), float(regularize),
                                          int(max_iterations), N.SOLVE_PLAIN if plain else 0,
                                          plan._stream(x), ctypes.byref(h)),
                "ccpi_session_create")
        self._h = h

    def run(self, n):
        N.check(N.lib.ccpi_session_run(self._h, int(n)), "ccpi_session_run")
        self.done += int(n)

    def finish(self):
        norms = np.zeros(max(self.done, 1), np.float64)
        N.check(N.lib.ccpi_session_finish(self._h, norms.ctypes.data), "ccpi_session_finish")
        return norms[:self.done]

    def close(self):
        if self._h:
            N.lib.ccpi_session_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batched(plans, alg, sinos, xs, niterations, regularize=None):
    """Solve independent problems together (one graph per iteration)."""
    n = len(plans)
    arr = lambda vals: (ctypes.c_void_p * n)(*vals)  # noqa: E731
    hp = arr([p.handle.value for p in plans])
    sp = arr([s.data_ptr() for s in sinos])
    xp = arr([x.data_ptr() for x in xs])
    reg = None
    if regularize is not None:
        reg_arr = np.ascontiguousarray(regularize, np.float64)
        reg = reg_arr.ctypes.data
    stream = ctypes.c_void_p(torch.cuda.current_stream(xs[0].device).cuda_stream) if n else None
    N.check(N.lib.ccpi_solve_batched(n, hp, int(alg), sp, xp, int(niterations), reg, stream),
            "ccpi_solve_batched")
    return xs


def parallel_plan(shape, n_angles, n_h, n_v=None, cor_shift=0.0, span=math.pi, angles=None):
    """Plan for a centred parallel-beam geometry with unit pixels and voxels."""
    nx, ny, nz = shape
    nv = nz if n_v is None else n_v
    ang = np.arange(n_angles) * (span / n_angles) if angles is None else np.asarray(angles)
    h = np.arange(n_h) - (n_h - 1) / 2.0 - cor_shift
    v = np.arange(nv) - (nv - 1) / 2.0
    return Plan("parallel", ang, h, v, (-nx / 2.0, -ny / 2.0, -nz / 2.0), (1.0, 1.0, 1.0), shape)


def cone_plan(n_vox, vox_size, n_angles, n_det, pix_size, s2o, o2d, n_det_v=None,
              full_circle=True):
    """Plan for a centred cone-beam geometry: source at (-s2o, 0, 0),
    detector plane at x = o2d."""
    nx, ny, nz = (n_vox,) * 3 if np.isscalar(n_vox) else n_vox
    nv = n_det if n_det_v is None else n_det_v
    span = 2 * math.pi if full_circle else math.pi
    ang = np.arange(n_angles) * (span / n_angles)
    h = (np.arange(n_det) - (n_det - 1) / 2.0) * pix_size
    v = (np.arange(nv) - (nv - 1) / 2.0) * pix_size
    origin = (-nx * vox_size / 2.0, -ny * vox_size / 2.0, -nz * vox_size / 2.0)
    return Plan("cone", ang, h, v, origin, (vox_size,) * 3, (nx, ny, nz),
                source=(-s2o, 0.0, 0.0), detector_x=o2d)


def parallel_api_plan(n_angles, n_v, n_h, angles_deg, rotation_centre, resolution):
    """Plan on the grid parallelbeam.alg derives from a sinogram shape
    (``ccpi_pb_geometry``).  Returns (plan, n_v_padded, v_offset)."""
    ang_deg = np.ascontiguousarray(angles_deg, np.float32)
    if ang_deg.shape != (int(n_angles),):
        raise ValueError("angles must have n_angles entries")
    dims = np.zeros(5, np.int32)
    N.check(N.lib.ccpi_pb_grid(int(n_angles), int(n_v), int(n_h), float(rotation_centre),
                               int(resolution), dims), "ccpi_pb_grid")
    nvp, voff = int(dims[3]), int(dims[4])
    ang = np.zeros(int(n_angles), np.float64)
    h = np.zeros(int(n_h), np.float64)
    v = np.zeros(nvp, np.float64)
    g = N.Geometry()
    N.check(N.lib.ccpi_pb_geometry(int(n_angles), int(n_v), int(n_h), ang_deg,
                                   float(rotation_centre), int(resolution), ang, h, v,
                                   ctypes.byref(g)), "ccpi_pb_geometry")
    plan = Plan("parallel", ang, h, v, tuple(g.origin), tuple(g.voxel_size), (g.nx, g.ny, g.nz))
    return plan, nvp, voff


def pack_parallel(pixels, n_v_padded, v_offset, out=None):
    """(n_angles, n_v, n_h) CUDA tensor -> (n_angles, n_h, n_v_padded), the
    layout the device solvers take (``ccpi_pb_pack``)."""
    if not (pixels.is_cuda and pixels.dtype == torch.float32 and pixels.is_contiguous()):
        raise ValueError("pixels must be a contiguous float32 CUDA tensor")
    na, nv, nh = pixels.shape
    if out is None:
        out = torch.empty((na, nh, int(n_v_padded)), device=pixels.device, dtype=torch.float32)
    N.check(N.lib.ccpi_pb_pack(ctypes.c_void_p(pixels.data_ptr()), na, nv, nh, int(n_v_padded),
                               int(v_offset), ctypes.c_void_p(out.data_ptr()),
                               ctypes.c_void_p(torch.cuda.current_stream(pixels.device).cuda_stream)),
            "ccpi_pb_pack")
    return out


def ring_filter_aml(sino, param_n, param_r, num_series):
    """AML ring-artefact filter (``ccpi_ring_filter_aml``) on a log sinogram
    in the internal layout (n_angles, n_h, n_v), in place, on torch's
    current stream; returns sino."""
    if not (sino.is_cuda and sino.dtype == torch.float32 and sino.is_contiguous()
            and sino.dim() == 3):
        raise ValueError("sinogram must be a contiguous 3-D float32 CUDA tensor")
    na, nh, nv = sino.shape
    N.check(N.lib.ccpi_ring_filter_aml(ctypes.c_void_p(sino.data_ptr()), na, nh, nv,
                                       float(param_n), float(param_r), int(num_series),
                                       ctypes.c_void_p(
                                           torch.cuda.current_stream(sino.device).cuda_stream)),
            "ccpi_ring_filter_aml")
    return sino


def _log_sinogram(sino):
    if not (sino.is_cuda and sino.dtype == torch.float32 and sino.is_contiguous()
            and sino.dim() == 3):
        raise ValueError("sinogram must be a contiguous 3-D float32 CUDA tensor")
    return sino.shape, ctypes.c_void_p(torch.cuda.current_stream(sino.device).cuda_stream)


def high_peaks(sino, jump, num_pix):
    """High-peaks filter (``ccpi_high_peaks``) on a log sinogram in the
    internal layout (n_angles, n_h, n_v), in place, on torch's current
    stream; returns sino."""
    (na, nh, nv), st = _log_sinogram(sino)
    N.check(N.lib.ccpi_high_peaks(ctypes.c_void_p(sino.data_ptr()), na, nh, nv, float(jump),
                                  int(num_pix), st), "ccpi_high_peaks")
    return sino


def ring_filter_column(sino):
    """Column ring-artefact filter (``ccpi_ring_filter_column``) on a log
    sinogram in the internal layout (n_angles, n_h, n_v), in place, on
    torch's current stream; returns sino."""
    (na, nh, nv), st = _log_sinogram(sino)
    N.check(N.lib.ccpi_ring_filter_column(ctypes.c_void_p(sino.data_ptr()), na, nh, nv, st),
            "ccpi_ring_filter_column")
    return sino
