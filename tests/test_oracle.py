"""The oracle (CPU restatement, oracle/restate.cpp) against the golden
fixtures the reference itself produced (tests/golden/make_golden.py), and
against the reference compiled from its sources when that build is present.
The float build of the restatement is expected to agree bit for bit."""
import numpy as np
import pytest

import oracle as O
from conftest import golden, golden_names, max_rel, rel_l2


def geom_from(d, kind):
    shape = tuple(int(s) for s in d["shape"])
    g = O.Geometry(kind, d["angles"], d["h"], d["v"], tuple(d["origin"]), tuple(d["size"]), shape)
    if kind == 1:
        g.source = tuple(d["source"])
        g.detector_x = float(d["detector_x"])
    return g


@pytest.mark.parametrize("name", ["pb0", "pb1", "pb2"])
def test_parallel_projectors_bit_exact(name):
    d = golden(name)
    g = geom_from(d, 0)
    assert np.array_equal(O.forward(g, d["vol"]), d["fp"])
    assert np.array_equal(O.backward(g, d["pix"]), d["bp"])


@pytest.mark.parametrize("name", ["cb0", "cb1"])
def test_cone_projectors_bit_exact(name):
    d = golden(name)
    g = geom_from(d, 1)
    assert np.array_equal(O.forward(g, d["vol"]), d["fp"])
    assert np.array_equal(O.backward(g, d["pix"]), d["bp"])


@pytest.mark.parametrize("name", golden_names("api_"))
def test_parallel_api_solvers_bit_exact(name):
    d = golden(name)
    pix = d["pixels"]
    na, nv, nh = pix.shape
    g, nvp, voff = O.parallel_api_geometry(na, nv, nh, d["angles"], float(d["cor"]), int(d["ppv"]))
    sino = O.parallel_api_sinogram(pix, nvp, voff, bool(d["is_log"]))
    rec = O.solve(g, int(d["alg"]), sino, int(d["niter"]), lam=float(d["lam"]))
    assert rec.shape == d["out"].shape
    assert np.array_equal(rec, d["out"]), max_rel(rec, d["out"])


@pytest.mark.parametrize("name", golden_names("step_"))
def test_parallel_step_forms_bit_exact(name):
    d = golden(name)
    pix = d["pixels"]
    na, nv, nh = pix.shape
    g, nvp, voff = O.parallel_api_geometry(na, nv, nh, d["angles"], 0.0, 1)
    sino = O.parallel_api_sinogram(pix, nvp, voff, False)
    rec = O.solve(g, int(d["alg"]), sino, int(d["niter"]), x0=d["x0"])
    assert np.array_equal(rec, d["out"])


def test_parallel_grids_match_reference():
    for row in golden("pb_grids")["rows"]:
        na, nv, nh, cor, ppv = int(row[0]), int(row[1]), int(row[2]), row[3], int(row[4])
        g, nvp, voff = O.parallel_api_geometry(na, nv, nh, np.zeros(na, np.float32), cor, ppv)
        assert list(g.shape) + [nvp] == [int(x) for x in row[5:9]]
        assert g.h_pixels[0] == row[9] and g.v_pixels[0] == row[10]
        assert g.size[0] == row[11] and g.size[2] == row[12]


def test_fp64_oracle_close_to_reference():
    d = golden("pb2")
    g = geom_from(d, 0)
    assert max_rel(O.forward(g, d["vol"], fp64=True), d["fp"]) < 1e-6
    d = golden("cb1")
    g = geom_from(d, 1)
    assert max_rel(O.backward(g, d["pix"], fp64=True), d["bp"]) < 1e-5


def test_fp64_solver_error_of_reference_is_small():
    # the reference's own FP32 rounding after 6 CGLS iterations is ~2e-4
    d = golden("api_alg0_cor0.0_ppv1")
    pix = d["pixels"]
    na, nv, nh = pix.shape
    g, nvp, voff = O.parallel_api_geometry(na, nv, nh, d["angles"], 0.0, 1)
    sino = O.parallel_api_sinogram(pix, nvp, voff, False)
    r64 = O.solve(g, O.CGLS, sino, int(d["niter"]), fp64=True)
    assert rel_l2(r64, d["out"]) < 5e-4


@pytest.mark.skipif(not O.reference_available(), reason="reference oracle not built")
def test_restatement_matches_compiled_reference_random():
    rng = np.random.default_rng(7)
    for shape, na, nh, shift in [((18, 22, 4), 29, 26, 0.37), ((12, 12, 8), 8, 20, 0.0)]:
        g = O.parallel_geometry(shape, na, nh, cor_shift=shift)
        vol = rng.random(shape).astype(np.float32)
        pix = rng.random(g.sino_shape).astype(np.float32)
        assert np.array_equal(O.forward(g, vol), O.ref_forward(g, vol))
        assert np.array_equal(O.backward(g, pix), O.ref_backward(g, pix))
    g = O.cone_geometry(14, 1.0, 17, 20, 1.0, 30.0, 30.0)
    vol = rng.random(g.shape).astype(np.float32)
    pix = rng.random(g.sino_shape).astype(np.float32)
    with O.quiet():
        assert np.array_equal(O.forward(g, vol), O.ref_forward(g, vol))
        assert np.array_equal(O.backward(g, pix), O.ref_backward(g, pix))


def test_neglog_uses_float_log():
    p = np.array([0.5, 1.0, 0.25, 0.9999], np.float32)
    assert np.array_equal(O.neglog(p), -np.log(p).astype(np.float32)) or \
        max_rel(O.neglog(p), -np.log(p.astype(np.float64))) < 1e-7


@pytest.mark.parametrize("name", golden_names("aml"))
def test_aml_restatement_equals_reference(name):
    """The restatement of the AML ring filter equals the reference's
    remove_aml_ring_artefacts bit for bit, and the fixture is the reference
    wrapper's output."""
    if not O.reference_available():
        pytest.skip("reference library not built")
    d = golden(name)
    pn, pr, ns = float(d["param_n"]), float(d["param_r"]), int(d["num_series"])
    p = np.ascontiguousarray(O.neglog(d["pixels"]).transpose(0, 2, 1))  # (na, nh, nv)
    assert np.array_equal(O.aml_ring(p, pn, pr, ns), O.ref_aml_ring(p, pn, pr, ns))
    assert np.array_equal(O.ref_aml_ring_artefacts(d["pixels"], pn, pr, ns), d["out"])


@pytest.mark.parametrize("name", golden_names("hp"))
def test_high_peaks_restatement_equals_golden(name):
    """The restatement of Diamond::high_peaks_before equals the reference's
    output stored in the fixture, bit for bit (and the reference itself
    when it is built)."""
    d = golden(name)
    jump, npix = float(d["jump"]), int(d["num_pix"])
    assert np.array_equal(O.high_peaks(d["logs"], jump, npix), d["out"])
    if O.reference_available():
        assert np.array_equal(O.ref_high_peaks(d["logs"], jump, npix), d["out"])


@pytest.mark.parametrize("name", golden_names("colring"))
def test_column_ring_restatement_equals_golden(name):
    d = golden(name)
    assert np.array_equal(O.column_ring(d["logs"]), d["out"])
    if O.reference_available():
        assert np.array_equal(O.ref_column_ring(d["logs"]), d["out"])


@pytest.mark.parametrize("seed", range(4))
def test_prefilters_restatement_equal_reference_random(seed):
    """Random sizes, jumps (zero, tiny, larger than any drop) and rounds up
    to n_angles - 1 against the reference library."""
    if not O.reference_available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(100 + seed)
    na, nh, nv = int(rng.integers(2, 40)), int(rng.integers(1, 30)), int(rng.integers(1, 6))
    p = rng.uniform(-1.0, 3.0, (na, nh, nv)).astype(np.float32)
    jump = [0.0, 1e-3, 0.3, 1e9][seed]
    npix = int(rng.integers(1, na))
    assert np.array_equal(O.high_peaks(p, jump, npix), O.ref_high_peaks(p, jump, npix))
    assert np.array_equal(O.column_ring(p), O.ref_column_ring(p))


def test_high_peaks_restatement_rejects_what_the_reference_rejects():
    p = np.ones((5, 3, 2), np.float32)
    for jump, npix in [(-0.1, 1), (0.1, 0), (0.1, 5)]:
        with pytest.raises(ValueError):
            O.high_peaks(p, jump, npix)
        if O.reference_available():  # reported and skipped: data unchanged
            assert np.array_equal(O.ref_high_peaks(p, jump, npix), p)
