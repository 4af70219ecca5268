"""``ccpi.reconstruction.parallelbeam.filters`` on a B200.

``aml_ring_artefacts(pixels, param_n, param_r, num_series)`` is the
reference's AML ring-artefact filter (Wrappers/Python/src/
diamond_module.cpp:58-68, diamond_wrapper.cpp:18-51): ``pixels`` is the
(n_angles, n_v, n_h) transmission stack; the filter runs on -log(pixels)
and the result is returned as transmission again, a new float32 array of
the same shape.  Deviation, on inputs the reference does not check:
parameters it rejects (param_n < 0, param_r <= 0, num_series outside
[1, 100]) raise RuntimeError instead of printing a message and returning
the data unfiltered.
"""
from __future__ import annotations

import numpy as np

from .. import _native as N

__all__ = ["aml_ring_artefacts"]


def aml_ring_artefacts(pixels, param_n, param_r, num_series):
    pix = N.f32(pixels, "pixels", 3)
    na, nv, nh = pix.shape
    out = np.empty_like(pix)
    N.check(N.lib.ccpi_pb_aml_ring_artefacts(pix, na, nv, nh, float(param_n), float(param_r),
                                             int(num_series), out),
            "aml_ring_artefacts")
    return out
