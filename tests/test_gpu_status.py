"""Failure detection without a GPU fault: the handle's device status word.

Kernels record conditions in a status word that the host reads (lt_status_word); nothing
here traps, hangs or faults a GPU.  The failures are made on the host side: a NaN uploaded
into one link, a unitarity defect uploaded into another, and a coupling so small that the
heatbath's accept/reject loop runs into the reference's 10-retry cap
(updates/heatbath.hpp:72-76) and takes the unit matrix.
"""
import numpy as np
import pytest

import lettuce_b200 as lt

pytestmark = pytest.mark.gpu

EXT = (4, 4, 4, 8)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp32_12"])
def test_healthy_field_has_clean_status(prec):
    G = lt.GaugeField(EXT, prec)
    G.SetToHaarRandom(3)
    lt.UpdateSweeps(G, 6.0, 3, 1, 4, seed=1)
    dev = G.check_links()
    assert dev < (1e-13 if prec == "fp64" else 2e-6), dev
    assert G.status_word() == 0


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp32_12"])
def test_nonfinite_and_unitarity_defects_are_flagged(prec):
    G = lt.GaugeField(EXT, prec)
    U = lt.haar_links(EXT, 4)
    U[5, 2, 0, 1, 0] = np.nan
    G.upload(U)
    G.check_links()
    assert G.status_word(clear=True) & lt.STATUS_NONFINITE
    assert G.status_word() == 0                      # cleared
    U = lt.haar_links(EXT, 4)
    U[7, 1, 1] *= 1.01                               # row 1 of one link no longer unit
    G.upload(U)
    dev = G.check_links()
    assert dev > 1e-3
    assert G.status_word(clear=True) == lt.STATUS_UNITARITY


@pytest.mark.parametrize("prec", ["fp64", "fp32_12"])
def test_heatbath_retry_cap_is_reported(prec):
    G = lt.GaugeField(EXT, prec)
    G.SetToHaarRandom(5)
    assert G.status_word() == 0
    lt.UpdateSweeps(G, 1e-3, 1, 1, 0, seed=2)        # lambda^2 ~ 1e3: every proposal rejected
    assert G.status_word(clear=True) & lt.STATUS_HB_CAP
    assert G.check_links() < 1e-4                    # the unit-matrix fallback keeps links in SU(3)
