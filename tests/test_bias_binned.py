"""The Gaussian-free binned bias update (the metadynamics configuration's "binned weights").

The reference deposits well-tempered Gaussians (metadynamics.hpp:103-147); the binned deposit
is not in the reference, so its checker is the C oracle's independent restatement
(or_bias_update_binned; parity unpinned against the reference) plus the properties that
define it.  All host code: no GPU is needed.
"""
import ctypes as C

import numpy as np
import pytest

import lettuce_b200 as lt
from lettuce_b200 import _lib

ARGS = (-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0)


def oracle_bias(oracle, cvs, symmetric=False, args=ARGS):
    b = oracle.lib.or_bias_create(*args)
    for cv in cvs:
        oracle.lib.or_bias_update_binned(b, cv)
        if symmetric:
            oracle.lib.or_bias_update_binned(b, -cv)
    # grid values through the potential at the grid points (interpolation weight 0 there)
    n = args[2]
    bw = (args[1] - args[0]) / n
    xs = [args[0] + i * bw for i in range(n)]
    g = np.array([oracle.lib.or_bias_potential(b, x) for x in xs])
    pot = lambda x: oracle.lib.or_bias_potential(b, x)   # noqa: E731
    return b, g, pot


def binned(cvs, symmetric=False, args=ARGS):
    b = lt.MetaBiasPotential(*args)
    b.SetUpdateMode("binned")
    assert b.GetUpdateMode() == "binned"
    if len(cvs):
        (b.UpdatePotentialSymmetric if symmetric else b.UpdatePotential)(np.asarray(cvs))
    return b


@pytest.mark.parametrize("symmetric", [False, True])
def test_matches_oracle(oracle, symmetric):
    rng = np.random.default_rng(5)
    cvs = np.concatenate([rng.normal(0.0, 2.0, 300), [7.999, -8.0, 8.0, 9.3, -11.0, 0.0, 0.02, -7.98]])
    b = binned(cvs, symmetric)
    ob, og, opot = oracle_bias(oracle, cvs, symmetric)
    # a CV on a grid point up to rounding may leave a share of order 1e-16 * weight on the
    # neighbouring point in one restatement and not in the other: compare to 1e-12 of weight
    np.testing.assert_allclose(b.grid()[:-1], og, rtol=1e-13, atol=1e-12 * ARGS[3])
    probes = np.linspace(-9.0, 9.0, 721)
    np.testing.assert_allclose([b.ReturnPotential(x) for x in probes], [opot(x) for x in probes],
                               rtol=1e-13, atol=1e-12 * ARGS[3])
    oracle.lib.or_bias_destroy(ob)


def test_deposit_adds_weight_of_area():
    """Without tempering (huge well_tempered_parameter) every in-range deposit raises the sum
    of the grid values by exactly `weight` (the two shares add up to it)."""
    args = (-8.0, 8.0, 800, 0.05, 0.08, 1e300, 1000.0)
    rng = np.random.default_rng(1)
    cvs = rng.uniform(-7.9, 7.9, 50)
    b = binned(cvs, args=args)
    g = b.grid()
    assert g.sum() == pytest.approx(50 * 0.05, rel=1e-13)
    # a deposit exactly on a grid point raises that point (and its potential) by `weight`
    b2 = binned([1.0], args=args)
    assert b2.ReturnPotential(1.0) == pytest.approx(0.05, rel=1e-13)
    assert np.count_nonzero(b2.grid()) == 1


def test_linear_split_between_bracketing_points():
    args = (-8.0, 8.0, 800, 1.0, 0.08, 1e300, 1000.0)
    bw = 16.0 / 800
    cv = -8.0 + 37 * bw + 0.25 * bw
    g = binned([cv], args=args).grid()
    assert np.flatnonzero(g).tolist() == [37, 38]
    assert g[37] == pytest.approx(0.75, rel=1e-12)
    assert g[38] == pytest.approx(0.25, rel=1e-12)


def test_well_tempered_increments_shrink():
    """Deposits at one point: each increment is weight exp(-V/wt), so V follows
    V_{n+1} = V_n + w exp(-V_n / wt)."""
    args = (-8.0, 8.0, 800, 0.5, 0.08, 2.0, 1000.0)
    b = binned([], args=args)
    v = 0.0
    for _ in range(40):
        b.UpdatePotential(0.0)
        v += 0.5 * np.exp(-v / 2.0)
    assert b.ReturnPotential(0.0) == pytest.approx(v, rel=1e-13)


def test_symmetric_and_out_of_range():
    b = binned([1.234, -3.3], symmetric=True)
    g = b.grid()
    np.testing.assert_allclose(g, g[::-1], rtol=1e-13, atol=1e-12 * ARGS[3])
    flat = binned([8.0, 9.5, -8.01, float("nan")])
    assert not np.any(flat.grid())


def test_mode_is_checked_and_default_is_gaussian():
    b = lt.MetaBiasPotential(*ARGS)
    assert b.GetUpdateMode() == "gaussian"
    assert lt.lib().lt_bias_set_update_mode(b.handle, 7) == _lib.LT_ERR_ARG
    assert lt.lib().lt_bias_set_update_mode(None, 1) == _lib.LT_ERR_ARG
    m = C.c_int()
    assert lt.lib().lt_bias_get_update_mode(None, C.byref(m)) == _lib.LT_ERR_ARG
