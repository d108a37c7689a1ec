"""The clover field as a FullTensor4D at the boundary (CalculateClover<1, 1>,
observables/clover.hpp:94-152; TopChargeClover(const FullTensor&),
topological_charge.hpp:202-231) against the reference's own functions
(tests/golden/ref_tensor_4x6x8x10.npz: 48 sampled sites with all 16 matrices, full-tensor
checksums and Q).  FP64: 1e-12 of the largest entry; two-row FP32 storage: 1e-5 (products in
FP64 from the stored links)."""
import os

import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import checksums, haar_links_numpy, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def tens(oracle):
    d = dict(np.load(os.path.join(GOLDEN, "ref_tensor_4x6x8x10.npz")))
    ext = tuple(int(e) for e in d["ext"])
    seed, hb, n = (int(v) for v in d["seeds"])
    d["ext"] = ext
    d["U"] = oracle.heatbath(ext, haar_links_numpy(ext, seed), 6.0, n, hb, 0)
    np.testing.assert_allclose(checksums(d["U"]), d["U_ck"], rtol=1e-13)
    return d


def test_tensor_against_reference(tens):
    G = lt.GaugeField(tens["ext"])
    G.upload(tens["U"])
    T = lt.CalculateClover(G)
    assert rel_err(T.data[tens["sites"]], tens["tensor"]) < 1e-12
    scale = np.abs(T.data).sum()
    assert np.all(np.abs(checksums(T.data) - tens["tensor_ck"]) <= 1e-12 * scale * np.array([1, 1, 97]))
    # C_{nu mu} = C_{mu nu}^dag and a zero diagonal, as the reference stores them
    M = T.data[..., 0] + 1j * T.data[..., 1]
    assert np.array_equal(M, np.conj(np.swapaxes(np.swapaxes(M, 1, 2), 3, 4)))
    assert not np.any(M[:, [0, 1, 2, 3], [0, 1, 2, 3]])


def test_topcharge_from_tensor(tens):
    G = lt.GaugeField(tens["ext"])
    G.upload(tens["U"])
    T = lt.CalculateClover(G)
    q_ref = float(tens["Q"])
    assert lt.TopChargeClover(T) == pytest.approx(q_ref, rel=1e-11, abs=1e-13)
    assert lt.TopChargeClover(G) == pytest.approx(q_ref, rel=1e-11, abs=1e-13)
    # a tensor given from the host (not computed by this handle): a detached copy, edited
    T2 = lt.FullTensor(tens["ext"])
    T2.data[:] = T.data
    assert lt.TopChargeClover(T2) == pytest.approx(q_ref, rel=1e-11, abs=1e-13)
    T2.data[:, 0, 1] *= 2.0          # F_01 = C_01 - C_10 no longer anti-Hermitian in the same way
    assert lt.TopChargeClover(T2) != pytest.approx(q_ref, rel=1e-6)


def test_tensor_fp32_12(tens):
    G = lt.GaugeField(tens["ext"], "fp32_12")
    G.upload(tens["U"])
    T = lt.CalculateClover(G)
    assert rel_err(T.data[tens["sites"]], tens["tensor"]) < 1e-5
