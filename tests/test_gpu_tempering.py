"""The tempering swap against the reference's own MetadynamicsTemperingKernel.

tests/golden/ref_tempering.npz holds five runs of MetadynamicsTemperingKernel::operator()
(updates/tempering.hpp:51-72) on two thermalised 8^4 fields -- the unbiased stream's links
(Gluon) and the biased stream's (Gluon_temper) -- with the reference driver's bias
(SU3_main.cpp:566-578) after the recorded deposits and with the recorded CV_current: the
candidate charge CV_new (MetaCharge: Q after n_smear_meta Euler-flow steps of rho), CV_old,
delta_V_tempering, the kernel's uniform, the decision and CV_current afterwards.

Here: the same bias through lt_bias_*; CV_new from lt_metad_charge (stout steps of rho: the
Euler flow step of step size rho is the stout step of parameter rho); the decision and dV
from lt_tempering_swap with scales (0, 1) -- the reference's two-stream rule -- given the
reference's uniform; on acceptance the link storage of the two handles is exchanged.
FP64: CV_new to 1e-11, dV to 1e-10 absolute, identical decisions.
"""
import os

import numpy as np
import pytest

import lettuce_b200 as lt
from lettuce_b200.tempering import metad_charge
from ltref import checksums, haar_links_numpy

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def temper(oracle):
    d = dict(np.load(os.path.join(GOLDEN, "ref_tempering.npz")))
    ext = tuple(int(e) for e in d["ext"])
    sa, sb, ha, hb, n = (int(v) for v in d["seeds"])
    d["ext"] = ext
    d["Ua"] = oracle.heatbath(ext, haar_links_numpy(ext, sa), 6.0, n, ha, 0)
    d["Ub"] = oracle.heatbath(ext, haar_links_numpy(ext, sb), 6.0, n, hb, 0)
    np.testing.assert_allclose(checksums(d["Ua"]), d["Ua_ck"], rtol=1e-13)
    np.testing.assert_allclose(checksums(d["Ub"]), d["Ub_ck"], rtol=1e-13)
    return d


def test_cases_cover_both_decisions(temper):
    acc = temper["out"][:, 4]
    assert 0 < acc.sum() < len(acc)


@pytest.mark.parametrize("case", range(5))
def test_swap_matches_reference(temper, case):
    d = temper
    ext, rho = d["ext"], float(d["rho"])
    cv_new, cv_old, dV, u, accepted, cv_after = d["out"][case]
    off = int(np.sum(d["n_dep"][:case]))
    deposits = d["deposits"][off:off + int(d["n_dep"][case])]
    bias = lt.MetaBiasPotential(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0)
    if deposits.size:
        bias.UpdatePotential(deposits)
    A, B = lt.GaugeField(ext), lt.GaugeField(ext)
    A.upload(d["Ua"])
    B.upload(d["Ub"])
    q_a = metad_charge(A, rho, 4)
    assert q_a == pytest.approx(cv_new, rel=1e-11, abs=1e-11)
    assert cv_old == pytest.approx(float(d["cv_old"][case]))
    acc, dE = lt.TemperingSwap(A, B, bias, 0.0, 1.0, q_a, cv_old, u)
    assert dE == pytest.approx(dV, rel=1e-10, abs=1e-10)
    assert acc == bool(accepted)
    # the reference's CV_current afterwards: the candidate's charge on acceptance
    assert (q_a if acc else cv_old) == pytest.approx(cv_after, rel=1e-11, abs=1e-11)
    want_a, want_b = (d["Ub"], d["Ua"]) if acc else (d["Ua"], d["Ub"])
    assert np.array_equal(A.download(), want_a)
    assert np.array_equal(B.download(), want_b)
