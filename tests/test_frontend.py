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


def test_high_peaks_parameters_checked_before_any_device_work():
    """jump < 0 and num_pix outside [1, n_angles) are errors of the call
    itself (the reference reports them and leaves the data unfiltered,
    diamond.cpp:520-527), raised before the filter touches a GPU."""
    from ccpi.reconstruction.parallelbeam import filters
    pix = np.full((6, 2, 5), 0.5, np.float32)
    for jump, npix in [(-0.1, 1), (0.1, 0), (0.1, 6)]:
        with pytest.raises(RuntimeError, match="high peaks"):
            filters.high_peaks(pix, jump, npix)
    with pytest.raises(ValueError):
        filters.column_ring_artefacts(np.zeros((4, 5)))


def test_setup_geometry_dicts():
    from ccpi.reconstruction.parallelbeam import alg
    d = alg.pb_setup_geometry_from_acquisition(np.zeros((91, 8, 160)), np.zeros(91), 0.0, 1)
    assert d == {"n_angles": 91, "n_h": 160, "n_v": 8, "output_volume_x": 160,
                 "output_volume_y": 160, "output_volume_z": 8}
    d = alg.pb_setup_geometry_from_image(np.zeros((24, 20, 7)), np.zeros(16), 1)
    assert d["n_h"] == 24 and d["n_v"] == 8 and d["output_volume_z"] == 7


@pytest.mark.parametrize("vshape,na,ppv", [((24, 20, 7), 16, 1), ((31, 40, 13), 9, 2),
                                           ((64, 64, 16), 180, 1)])
def test_setup_geometry_dicts_match_reference(vshape, na, ppv):
    """pb_setup_geometry_from_image / _from_acquisition
    (diamond_wrapper.cpp:559-631, :760-823) give the reference's numbers:
    its padded row count and, from a sinogram, its reconstruction grid."""
    import oracle as O
    if not O.reference_available():
        pytest.skip("oracle/_ref/libccpi_ref.so not built")
    from ccpi.reconstruction.parallelbeam import alg
    vx, vy, vz = vshape
    width = max(vx, vy)
    d = alg.pb_setup_geometry_from_image(np.zeros(vshape, np.float32), np.zeros(na), ppv)
    dims, _ = O.ref_pb_geometry(na, vz, width, width / 2.0, ppv)
    assert d == {"n_angles": na, "n_h": width, "n_v": int(dims[3]), "output_volume_x": vx,
                 "output_volume_y": vy, "output_volume_z": vz}
    nv, nh, cor = vz + 3, width + 5, width / 2.0 + 1.25
    d = alg.pb_setup_geometry_from_acquisition(np.zeros((na, nv, nh), np.float32), np.zeros(na),
                                               cor, ppv)
    dims, _ = O.ref_pb_geometry(na, nv, nh, cor, ppv)
    assert d == {"n_angles": na, "n_h": nh, "n_v": int(dims[3]), "output_volume_x": int(dims[0]),
                 "output_volume_y": int(dims[1]), "output_volume_z": int(dims[2])}


@pytest.mark.parametrize("na,nv,nh,cor,ppv", [(30, 7, 40, 0.0, 1), (45, 16, 64, 33.25, 2),
                                              (12, 5, 33, 16.0, 1)])
def test_pb_geometry_matches_oracle_front_end(na, nv, nh, cor, ppv):
    """ccpi_pb_geometry gives the geometry the oracle's restatement of the
    Diamond front-end gives (grid, detector coordinates, angles)."""
    import ctypes
    import oracle as O
    from ccpi.reconstruction import _native as N
    deg = np.linspace(0, 180, na, endpoint=False).astype(np.float32)
    dims = np.zeros(5, np.int32)
    assert N.lib.ccpi_pb_grid(na, nv, nh, cor, ppv, dims) == 0
    ang = np.zeros(na)
    h = np.zeros(nh)
    v = np.zeros(int(dims[3]))
    g = N.Geometry()
    assert N.lib.ccpi_pb_geometry(na, nv, nh, deg, cor, ppv, ang, h, v, ctypes.byref(g)) == 0
    og, nvp, voff = O.parallel_api_geometry(na, nv, nh, deg, cor, ppv)
    assert (g.nx, g.ny, g.nz) == tuple(og.shape) and (nvp, voff) == (dims[3], dims[4])
    assert np.array_equal(ang, og.angles) and np.array_equal(h, og.h_pixels)
    assert np.array_equal(v, og.v_pixels)
    assert tuple(g.origin) == tuple(og.origin) and tuple(g.voxel_size) == tuple(og.size)


def test_create_phantom_volume_equals_reference():
    """conebeam.create_phantom_volume: the reference's volume, angles,
    detector coordinates and scalars, exactly (its test_conebeam.py:17-27
    checks the same scalars of create_phantom)."""
    import oracle as O
    from ccpi.reconstruction.conebeam import alg
    ours = alg.create_phantom_volume()
    assert ours[1].shape == (250,) and ours[0].shape == (512, 512, 512)
    assert ours[4:] == (250.0, 987.0, 0.390625, 0.390625, 25.151547886198443)
    if not O.reference_available():
        pytest.skip("reference library not built")
    ref = O.ref_cb_phantom_volume()
    for a, b in zip(ours[:4], ref[:4]):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    assert ours[4:] == ref[4:]
