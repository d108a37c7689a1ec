"""The Zeuthen flow (Ramos and Sint, arXiv:1508.05552): not in the reference, so its checker
is the C oracle's restatement (or_flow_zeuthen; parity unpinned against the reference) and
the properties that define it.  CPU: the oracle's own gauge covariance and small-step limit.
GPU (marked): the CUDA path against the oracle for every integrator and storage format, and
gauge covariance of the device flow.
"""
import numpy as np
import pytest

from ltref import haar_links_numpy, rel_err

EXTS = [(4, 4, 4, 4), (4, 6, 4, 8)]


def to_c(U):
    return U[..., 0] + 1j * U[..., 1]


def from_c(M):
    out = np.empty(M.shape + (2,))
    out[..., 0], out[..., 1] = M.real, M.imag
    return out


def gauge_transform(ext, U, seed):
    """U_mu(x) -> G(x) U_mu(x) G(x + mu)^dag with Haar-random G (reference site order)."""
    V = int(np.prod(ext))
    G = to_c(haar_links_numpy(ext, seed)[:, 0])          # one SU(3) matrix per site
    M = to_c(U)
    idx = np.arange(V).reshape(ext)
    out = np.empty_like(M)
    for mu in range(4):
        fwd = np.roll(idx, -1, axis=mu).reshape(-1)
        out[:, mu] = G @ M[:, mu] @ np.conj(np.transpose(G[fwd], (0, 2, 1)))
    return from_c(out)


@pytest.fixture(scope="module")
def starts(oracle):
    return {ext: oracle.heatbath(ext, haar_links_numpy(ext, 31), 6.0, 6, 4, 0) for ext in EXTS}


@pytest.mark.parametrize("ext", EXTS)
def test_oracle_gauge_covariant(oracle, starts, ext):
    U = starts[ext]
    Ug = gauge_transform(ext, U, 77)
    F = oracle.flow_zeuthen(ext, U, 0.02, 3)
    Fg = oracle.flow_zeuthen(ext, Ug, 0.02, 3)
    assert rel_err(Fg, gauge_transform(ext, F, 77)) < 1e-12
    assert oracle.energy(ext, Fg) == pytest.approx(oracle.energy(ext, F), rel=1e-12)


def test_oracle_small_step_is_luescher_weisz_plus_correction(oracle, starts):
    """One Euler step of size eps differs from the Luescher-Weisz Euler step by
    eps * Algebra(nabla* nabla X / 12) in the exponent: O(eps), vanishing with eps, and the
    two flows agree at eps -> 0 to first order."""
    ext = EXTS[0]
    U = starts[ext]
    d = []
    for eps in (1e-3, 5e-4):
        z = oracle.flow_zeuthen(ext, U, eps, 1, 0)
        with oracle.action((2, 5.0 / 3.0, -1.0 / 12.0)):
            lw = oracle.flow(ext, U, eps, 1, 0)
        d.append(np.abs(z - lw).max())
    assert d[0] > 0 and d[1] / d[0] == pytest.approx(0.5, rel=0.02)


@pytest.mark.gpu
class TestDevice:
    @pytest.mark.parametrize("ext", EXTS)
    @pytest.mark.parametrize("integ", [0, 1, 2, 3])
    def test_fp64_against_oracle(self, oracle, starts, ext, integ):
        import lettuce_b200 as lt
        U = starts[ext]
        G, H = lt.GaugeField(ext), lt.GaugeField(ext)
        G.upload(U)
        integrator = (lt.Euler, lt.RK2, lt.RK3, lt.RK3W7)[integ]
        lt.GradientFlowKernel(G, H, integrator, lt.ZeuthenFlow(), 0.02)(4)
        assert rel_err(H.download(), oracle.flow_zeuthen(ext, U, 0.02, 4, integ)) < 1e-12

    @pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
    def test_fp32_against_oracle(self, oracle, starts, prec):
        import lettuce_b200 as lt
        ext = EXTS[1]
        U = starts[ext]
        G, H = lt.GaugeField(ext, prec), lt.GaugeField(ext, prec)
        G.upload(U)
        lt.GradientFlowKernel(G, H, lt.RK3, lt.ZeuthenFlow(), 0.02)(4)
        assert rel_err(H.download(), oracle.flow_zeuthen(ext, U, 0.02, 4, 2)) < 1e-5

    def test_gauge_covariant_and_flow_kind_resets(self, oracle, starts):
        import lettuce_b200 as lt
        ext = EXTS[1]
        U = starts[ext]
        out = []
        for W in (U, gauge_transform(ext, U, 5)):
            G, H = lt.GaugeField(ext), lt.GaugeField(ext)
            G.upload(W)
            flow = lt.GradientFlowKernel(G, H, lt.RK3, lt.ZeuthenFlow(), 0.02)
            p, q, e = flow.Measure(3, 2)
            out.append((p, q, e, H.download()))
        np.testing.assert_allclose(out[1][0], out[0][0], rtol=1e-12)
        np.testing.assert_allclose(out[1][2], out[0][2], rtol=1e-12)
        assert np.max(np.abs(out[1][1] - out[0][1])) < 1e-12
        assert rel_err(out[1][3], gauge_transform(ext, out[0][3], 5)) < 1e-12
        # the same handle flows with the Wilson force again once the kernel says so
        G, H = lt.GaugeField(ext), lt.GaugeField(ext)
        G.upload(U)
        lt.GradientFlowKernel(G, H, lt.RK3, lt.ZeuthenFlow(), 0.02)(1)
        lt.GradientFlowKernel(G, H, lt.RK3, None, 0.02)(2)
        assert rel_err(H.download(), oracle.flow_rk3(ext, U, 0.02, 2)) < 1e-12
