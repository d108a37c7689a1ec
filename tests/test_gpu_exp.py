"""The device SU(3) exponential on the reference's own edge cases, branch by branch.

Inputs: golden4["exp_in"] (generic, Taylor-branch, sign-flip and zero matrices) and
tests/golden/ref_exp.npz (every range of the spectral bound c1 = tr(Q^2)/2 that selects a
branch of the device exponential, negative determinants, exactly and nearly degenerate
spectra -- theta = 0 and w -> 0, the Taylor switches of xi_0 and xi_1 -- and the zero
matrix).  Expected values: the reference's SU3::exp (math/su3_exp.hpp:204-283, :419-432)
run on the same inputs by the reference harness.

Each branch runs through the test entry point lt_su3_exp_test:
  * FP64: the dispatch the flow, stout and HMC kernels use, the closed form on every input,
    and each series (tiny, short, long term counts) on the inputs inside its range -- 1e-12 absolute (entries are O(1));
  * FP32 (the arithmetic of both FP32 storages): the same branches, within 4e-6 max(1, c1)
    (the input is rounded to FP32 and Q^2 carries c1-sized entries).
The outputs must also be unitary with unit determinant to the arithmetic's precision.
"""
import ctypes as C
import os

import numpy as np
import pytest

import lettuce_b200 as lt
from lettuce_b200 import _lib

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DISPATCH, CLOSED, SHORT, LONG, TINY = 0, 1, 2, 3, 4


@pytest.fixture(scope="module")
def cases(golden4):
    d = dict(np.load(os.path.join(GOLDEN, "ref_exp.npz")))
    q = np.concatenate([golden4["exp_in"].reshape(-1, 18), d["exp_in"].reshape(-1, 18)])
    e = np.concatenate([golden4["exp_out"].reshape(-1, 18), d["exp_out"].reshape(-1, 18)])
    Q = (q[:, 0::2] + 1j * q[:, 1::2]).reshape(-1, 3, 3)
    c1 = 0.5 * np.einsum("nij,nji->n", Q, Q).real
    return np.ascontiguousarray(q), e, c1


def device_exp(q, prec, path):
    out = np.empty_like(q)
    _lib.check(lt.lib().lt_su3_exp_test(q, out, q.shape[0], _lib.PREC[prec], path))
    return out


def unitarity(out):
    M = (out[:, 0::2] + 1j * out[:, 1::2]).reshape(-1, 3, 3)
    u = np.abs(np.einsum("nij,nkj->nik", M, M.conj()) - np.eye(3)).max()
    return u, np.abs(np.linalg.det(M) - 1).max()


def test_inputs_cover_every_branch(cases):
    _, _, c1 = cases
    assert np.sum(c1 > 0.5) >= 16
    assert np.sum((c1 > 1 / 32) & (c1 <= 0.5)) >= 16
    assert np.sum((c1 > 1 / 512) & (c1 <= 1 / 32)) >= 16
    assert np.sum((c1 > 0) & (c1 <= 1 / 512)) >= 16
    assert np.sum(c1 == 0) >= 1


@pytest.mark.parametrize("path", [DISPATCH, CLOSED])
def test_fp64_against_reference(cases, path):
    q, ref, _ = cases
    out = device_exp(q, "fp64", path)
    assert np.abs(out - ref).max() < 1e-12
    u, d = unitarity(out)
    assert u < 1e-13 and d < 1e-13


@pytest.mark.parametrize("path,limit", [(TINY, 1 / 512), (SHORT, 1 / 32), (LONG, 0.5)])
def test_fp64_series_in_range(cases, path, limit):
    q, ref, c1 = cases
    m = c1 <= limit
    out = device_exp(np.ascontiguousarray(q[m]), "fp64", path)
    assert np.abs(out - ref[m]).max() < 1e-12


@pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
@pytest.mark.parametrize("path", [DISPATCH, CLOSED])
def test_fp32_against_reference(cases, prec, path):
    q, ref, c1 = cases
    out = device_exp(q, prec, path)
    err = np.abs(out - ref).max(axis=1)
    assert np.all(err < 4e-6 * np.maximum(1.0, c1)), err.max()
    u, d = unitarity(out)
    assert u < 2e-6 * max(1.0, c1.max()) and d < 2e-6 * max(1.0, c1.max())


@pytest.mark.parametrize("path,limit", [(TINY, 1 / 512), (SHORT, 1 / 32), (LONG, 0.5)])
def test_fp32_series_in_range(cases, path, limit):
    q, ref, c1 = cases
    m = c1 <= limit
    out = device_exp(np.ascontiguousarray(q[m]), "fp32", path)
    assert np.abs(out - ref[m]).max() < 2e-6


def test_sign_flip_is_conjugation(cases):
    """exp(-iQ) = exp(iQ)^dagger for Hermitian Q: the reference's signflip branch."""
    q, _, _ = cases
    a = device_exp(q, "fp64", DISPATCH)
    b = device_exp(np.ascontiguousarray(-q), "fp64", DISPATCH)
    A = (a[:, 0::2] + 1j * a[:, 1::2]).reshape(-1, 3, 3)
    B = (b[:, 0::2] + 1j * b[:, 1::2]).reshape(-1, 3, 3)
    assert np.abs(B - np.conj(np.transpose(A, (0, 2, 1)))).max() < 1e-13


def test_kernels_built_for_sm100a():
    bv, pv = C.c_int(), C.c_int()
    _lib.check(lt.lib().lt_device_arch(C.byref(bv), C.byref(pv)))
    assert bv.value == 100
