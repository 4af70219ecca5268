"""Host-side parts of the C-ABI library that run without a GPU: symbol
exports, the numpy-path geometry (grids, padding, centre search) and the
Python wrappers' argument checking."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden

HEADER = os.path.join(ROOT, "include", "ccpi_b200.h")
LIB = os.path.join(ROOT, "ccpi-reconstruction_b200", "libccpi_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ccpi_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    syms = declared_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(lib, s), s


def test_parallel_grid_matches_reference():
    from ccpi.reconstruction.parallelbeam import alg
    for row in golden("pb_grids")["rows"]:
        na, nv, nh, cor, ppv = int(row[0]), int(row[1]), int(row[2]), row[3], int(row[4])
        nx, ny, nz, nvp, voff = alg.grid(na, nv, nh, cor, ppv)
        assert [nx, ny, nz, nvp] == [int(x) for x in row[5:9]]


def test_cone_grid_matches_reference():
    from ccpi.reconstruction.conebeam import alg
    for row in golden("cb_grids")["rows"]:
        na, nh, nv, ppv = (int(x) for x in row[:4])
        dims, geo = alg.grid(na, nh, nv, ppv, *row[4:9])
        assert list(dims[:4]) == [int(x) for x in row[9:13]]
        assert np.array_equal(np.array(geo), row[13:18])


def test_cone_centre_search_matches_reference():
    from ccpi.reconstruction.conebeam import alg
    d = golden("cb_centre")
    sino = d["sino"]
    na, nh, nv = sino.shape
    dims, _ = alg.grid(na, nh, nv, 1, float(d["s2s"]), float(d["s2d"]), float(d["px"]),
                       float(d["px"]), float(d["mask_radius"]))
    nvp, voff = dims[3], dims[4]
    padded = np.zeros((na, nh, nvp), np.float32)
    padded[:, :, voff:voff + nv] = sino
    y = alg.find_centre(padded, d["angles"], float(d["s2s"]), float(d["s2d"]), float(d["px"]))
    assert y == d["geom"][5]


def test_wrapper_rejects_bad_inputs():
    from ccpi.reconstruction.parallelbeam import alg
    with pytest.raises(ValueError):
        alg.cgls(np.zeros((4, 5)), np.zeros(4), 0.0, 1, 2, 1, True)
    with pytest.raises(ValueError):
        alg.sirt(np.zeros((4, 5, 6)), np.zeros(3), 0.0, 1, 2, 1, True)
    with pytest.raises(TypeError):
        alg.mlem(np.zeros((4, 5, 6), np.complex64), np.zeros(4), 0.0, 1, 2, 1, True)
    with pytest.raises(RuntimeError):
        alg.grid(0, 4, 4, 0.0, 1)


def test_setup_geometry_dicts():
    from ccpi.reconstruction.parallelbeam import alg
    d = alg.pb_setup_geometry_from_acquisition(np.zeros((91, 8, 160)), np.zeros(91), 0.0, 1)
    assert d == {"n_angles": 91, "n_h": 160, "n_v": 8, "output_volume_x": 160,
                 "output_volume_y": 160, "output_volume_z": 8}
    d = alg.pb_setup_geometry_from_image(np.zeros((24, 20, 7)), np.zeros(16), 1)
    assert d["n_h"] == 24 and d["n_v"] == 8 and d["output_volume_z"] == 7
