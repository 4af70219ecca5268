"""The sinogram filters against the reference: the AML ring-artefact filter
(parallelbeam.filters.aml_ring_artefacts), the high-peaks filter and the
column ring filter, through the reference-facing calls on the golden stacks
and through the device calls on log sinograms, all bit for bit."""
import numpy as np
import pytest

import oracle as O
from conftest import golden, golden_names, max_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names("aml"))
def test_aml_ring_artefacts_vs_reference(name, cuda):
    from ccpi.reconstruction.parallelbeam import filters
    d = golden(name)
    out = filters.aml_ring_artefacts(d["pixels"], float(d["param_n"]), float(d["param_r"]),
                                     int(d["num_series"]))
    assert out.shape == d["out"].shape and out.dtype == np.float32
    assert np.array_equal(out, d["out"]), max_rel(out, d["out"])


@pytest.mark.parametrize("seed,ns", [(0, 1), (1, 2), (2, 4)])
def test_device_ring_filter_vs_restatement(seed, ns, cuda):
    import torch
    from ccpi.reconstruction.device import ring_filter_aml
    rng = np.random.default_rng(seed)
    na, nh, nv = int(rng.integers(20, 80)), int(rng.integers(8, 60)), int(rng.integers(1, 6))
    p = rng.uniform(0.0, 2.0, (na, nh, nv)).astype(np.float32)
    pn, pr = float(rng.uniform(0, 1)), float(rng.uniform(0.001, 0.2))
    t = torch.from_numpy(p).to(cuda)
    ring_filter_aml(t, pn, pr, ns)
    assert np.array_equal(t.cpu().numpy(), O.aml_ring(p, pn, pr, ns))


def test_ring_filter_rejects_bad_parameters(cuda):
    from ccpi.reconstruction.parallelbeam import filters
    pix = np.full((10, 2, 12), 0.5, np.float32)
    for args in [(-0.1, 0.01, 1), (0.1, 0.0, 1), (0.1, 0.01, 0), (0.1, 0.01, 101)]:
        with pytest.raises(RuntimeError):
            filters.aml_ring_artefacts(pix, *args)


@pytest.mark.parametrize("name", golden_names("hp"))
def test_high_peaks_vs_reference(name, cuda):
    import torch
    from ccpi.reconstruction.device import high_peaks
    from ccpi.reconstruction.parallelbeam import filters
    d = golden(name)
    jump, npix = float(d["jump"]), int(d["num_pix"])
    t = torch.from_numpy(d["logs"]).to(cuda)
    high_peaks(t, jump, npix)
    assert np.array_equal(t.cpu().numpy(), d["out"])
    # the (n_angles, n_v, n_h) call on logs, and on transmission
    logs = np.ascontiguousarray(d["logs"].transpose(0, 2, 1))
    out = filters.high_peaks(logs, jump, npix, is_pixels_in_log=True)
    assert np.array_equal(out, d["out"].transpose(0, 2, 1))
    trans = O.expneg(logs)
    want = O.expneg(O.high_peaks(O.neglog(trans).transpose(0, 2, 1), jump, npix)
                    .transpose(0, 2, 1))
    assert np.array_equal(filters.high_peaks(trans, jump, npix), want)


@pytest.mark.parametrize("name", golden_names("colring"))
def test_column_ring_vs_reference(name, cuda):
    import torch
    from ccpi.reconstruction.device import ring_filter_column
    from ccpi.reconstruction.parallelbeam import filters
    d = golden(name)
    t = torch.from_numpy(d["logs"]).to(cuda)
    ring_filter_column(t)
    assert np.array_equal(t.cpu().numpy(), d["out"])
    logs = np.ascontiguousarray(d["logs"].transpose(0, 2, 1))
    out = filters.column_ring_artefacts(logs, is_pixels_in_log=True)
    assert np.array_equal(out, d["out"].transpose(0, 2, 1))
    trans = O.expneg(logs)
    want = O.expneg(O.column_ring(O.neglog(trans).transpose(0, 2, 1)).transpose(0, 2, 1))
    assert np.array_equal(filters.column_ring_artefacts(trans), want)


@pytest.mark.parametrize("seed", range(3))
def test_device_prefilters_vs_restatement(seed, cuda):
    import torch
    from ccpi.reconstruction.device import high_peaks, ring_filter_column
    rng = np.random.default_rng(40 + seed)
    na, nh, nv = int(rng.integers(2, 200)), int(rng.integers(1, 90)), int(rng.integers(1, 40))
    p = rng.uniform(-1.0, 3.0, (na, nh, nv)).astype(np.float32)
    jump, npix = float(rng.choice([0.0, 0.01, 0.5])), int(rng.integers(1, na))
    t = torch.from_numpy(p).to(cuda)
    high_peaks(t, jump, npix)
    assert np.array_equal(t.cpu().numpy(), O.high_peaks(p, jump, npix))
    t = torch.from_numpy(p).to(cuda)
    ring_filter_column(t)
    assert np.array_equal(t.cpu().numpy(), O.column_ring(p))


def test_prefilters_full_size_properties(cuda):
    """A 720 x 768 x 256 log sinogram (the parallel-beam bench size): after
    the column filter every element's mean over the angles is within float
    rounding of zero; a high-peaks pass with a jump larger than any drop
    changes nothing beyond the rounding of p[a+1] + (p[a] - p[a+1]), and
    one round leaves no drop between neighbouring angles below -jump in the
    top-to-bottom direction (checked on a slab against the restatement)."""
    import torch
    from ccpi.reconstruction.device import high_peaks, ring_filter_column
    g = torch.Generator(device=cuda).manual_seed(5)
    t = torch.rand((720, 768, 256), device=cuda, generator=g) * 2.0 + 0.5
    ring_filter_column(t)
    m = t.double().mean(dim=0)
    assert float(m.abs().max()) < 1e-5
    t = torch.rand((720, 768, 256), device=cuda, generator=g) * 2.0
    ref = t.clone()
    high_peaks(t, 1e9, 2)
    assert float((t - ref).abs().max()) < 1e-5
    slab = ref[:, 100:104, :].contiguous().cpu().numpy()
    t = ref.clone()
    high_peaks(t, 0.05, 1)
    assert np.array_equal(t[:, 100:104, :].cpu().numpy(), O.high_peaks(slab, 0.05, 1))


def test_prefilters_reject_bad_parameters(cuda):
    from ccpi.reconstruction.parallelbeam import filters
    pix = np.full((10, 2, 12), 0.5, np.float32)
    for jump, npix in [(-0.1, 1), (0.1, 0), (0.1, 10)]:
        with pytest.raises(RuntimeError):
            filters.high_peaks(pix, jump, npix)
