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

The reference's other two sinogram pre-processing steps, which it runs only
when a Diamond data file's configuration asks for them
(Core/src/diamond.cpp:383-387) and which have no Python call there, are
here as well, on the same (n_angles, n_v, n_h) layout:

``high_peaks(pixels, jump, num_pix, is_pixels_in_log=False)`` is
CCPi::Diamond::high_peaks_before (diamond.cpp:513-617): num_pix rounds of a
top-to-bottom and a bottom-to-top pass over the angles that limit every drop
between neighbouring angles to ``jump``.

``column_ring_artefacts(pixels, is_pixels_in_log=False)`` is
CCPi::remove_column_ring_artefacts (diamond.cpp:619-658): every detector
element loses its mean over the angles.

Both run on -log(pixels) and return transmission, as aml_ring_artefacts
does, unless ``is_pixels_in_log`` is true, in which case logs go in and
come out unchanged in form.  jump < 0 and num_pix outside [1, n_angles),
which the reference reports and skips, raise RuntimeError.
"""
from __future__ import annotations

import numpy as np

from .. import _native as N

__all__ = ["aml_ring_artefacts", "high_peaks", "column_ring_artefacts"]


def aml_ring_artefacts(pixels, param_n, param_r, num_series):
    pix = N.f32(pixels, "pixels", 3)
    na, nv, nh = pix.shape
    out = np.empty_like(pix)
    N.check(N.lib.ccpi_pb_aml_ring_artefacts(pix, na, nv, nh, float(param_n), float(param_r),
                                             int(num_series), out),
            "aml_ring_artefacts")
    return out


def high_peaks(pixels, jump, num_pix, is_pixels_in_log=False):
    pix = N.f32(pixels, "pixels", 3)
    na, nv, nh = pix.shape
    out = np.empty_like(pix)
    N.check(N.lib.ccpi_pb_high_peaks(pix, na, nv, nh, float(jump), int(num_pix),
                                     int(bool(is_pixels_in_log)), out),
            "high_peaks")
    return out


def column_ring_artefacts(pixels, is_pixels_in_log=False):
    pix = N.f32(pixels, "pixels", 3)
    na, nv, nh = pix.shape
    out = np.empty_like(pix)
    N.check(N.lib.ccpi_pb_column_ring_artefacts(pix, na, nv, nh, int(bool(is_pixels_in_log)),
                                                out),
            "column_ring_artefacts")
    return out
