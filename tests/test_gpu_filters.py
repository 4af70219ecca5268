"""The AML ring-artefact filter (parallelbeam.filters.aml_ring_artefacts)
against the reference: the reference-facing call on the golden stacks and
the device call on a log sinogram, both bit for bit."""
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
