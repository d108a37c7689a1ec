"""Statistical and derivative checks of the stochastic and adjoint parts on the GPU.

* Heatbath + overrelaxation chains are chaotic, so against the reference they are compared
  statistically: the mean plaquette of a GPU chain at 8^4, beta = 6 must lie within 2 sigma
  (binned errors of both chains combined) of the reference chain in tests/golden/.
* HMC: <exp(-dH)> = 1 within its error.
* The hand-written adjoint of the metadynamics force is compared with symmetric finite
  differences of the stout-smeared clover charge, using the reference's own check pattern
  (LettuceGauge/numerical_derivative.hpp:71-249): left multiplication of one link by
  exp(+-i h lambda_a / 2) and dQ/dh vs Re tr(i lambda_a F).
"""
import numpy as np
import pytest

import lettuce_b200 as lt

pytestmark = pytest.mark.gpu

GELL_MANN = np.zeros((8, 3, 3), dtype=np.complex128)
GELL_MANN[0][0, 1] = GELL_MANN[0][1, 0] = 1
GELL_MANN[1][0, 1], GELL_MANN[1][1, 0] = -1j, 1j
GELL_MANN[2][0, 0], GELL_MANN[2][1, 1] = 1, -1
GELL_MANN[3][0, 2] = GELL_MANN[3][2, 0] = 1
GELL_MANN[4][0, 2], GELL_MANN[4][2, 0] = -1j, 1j
GELL_MANN[5][1, 2] = GELL_MANN[5][2, 1] = 1
GELL_MANN[6][1, 2], GELL_MANN[6][2, 1] = -1j, 1j
GELL_MANN[7] = np.diag([1, 1, -2]) / np.sqrt(3)


def exp_lambda(a, alpha):
    """exp(i alpha lambda_a / 2) (math/su3.hpp:135-260) via eigendecomposition."""
    w, v = np.linalg.eigh(GELL_MANN[a])
    return (v * np.exp(0.5j * alpha * w)) @ v.conj().T


def binned_mean_err(x, nbin=20):
    x = np.asarray(x)
    b = x[: len(x) // nbin * nbin].reshape(nbin, -1).mean(axis=1)
    return x.mean(), b.std(ddof=1) / np.sqrt(nbin)


def chains_mean_err(hist):
    """Mean and error of several independent chains: per chain the error of 10 bins, combined;
    never below the scatter of the chain means (slow modes at beta = 6 outlive short bins)."""
    hist = np.atleast_2d(np.asarray(hist))
    means, errs = zip(*(binned_mean_err(h, 10) for h in hist))
    n = len(means)
    err = np.sqrt(np.sum(np.square(errs))) / n
    if n > 1:
        err = max(err, np.std(means, ddof=1) / np.sqrt(n))
    return float(np.mean(means)), float(err)


@pytest.mark.parametrize("prec", ["fp64", "fp32_12"])
def test_heatbath_chain_matches_reference(golden_chain, prec):
    """Independent GPU chains vs independent reference chains (8^4, beta = 6, 1 HB + 4 OR per
    round, same thermalisation and length): mean plaquettes within 2 sigma."""
    ext = (8, 8, 8, 8)
    V = 8 ** 4
    ref_hist = golden_chain["plaq_norm"]
    n_therm, n_meas = int(golden_chain["n_therm"]), ref_hist.shape[1]
    hist = []
    for k in range(ref_hist.shape[0]):
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(100 + k)
        c = lt.UpdateSweeps(G, 6.0, n_therm, 1, 4, seed=31337 + k)
        plaq = []
        for _ in range(n_meas):
            c = lt.UpdateSweeps(G, 6.0, 1, 1, 4, seed=31337 + k, counter=c)
            plaq.append(lt.PlaquetteSum(G) / V / 18)
        hist.append(plaq)
    m_gpu, e_gpu = chains_mean_err(hist)
    m_ref, e_ref = chains_mean_err(ref_hist)
    sigma = np.hypot(e_gpu, e_ref)
    assert abs(m_gpu - m_ref) < 2 * sigma, (m_gpu, e_gpu, m_ref, e_ref)


def test_hmc_exp_minus_dH():
    ext = (8, 8, 8, 8)
    G = lt.GaugeField(ext, "fp64")
    G.SetToHaarRandom(8)
    lt.UpdateSweeps(G, 6.0, 50, 1, 4, seed=3)
    hmc = lt.HMCKernel(G, lt.WilsonAction(6.0), 1.0, seed=17)
    acc, x = 0, []
    for _ in range(60):
        acc += hmc(10, True)
        x.append(np.exp(-hmc.delta_H))
    m, e = binned_mean_err(x, 10)
    assert abs(m - 1.0) < 3 * e + 0.02, (m, e)
    assert acc > 30


def test_metad_force_finite_differences():
    """16^4, 4 stout steps rho = 0.12; 64 random links, all 8 generators."""
    ext = (16, 16, 16, 16)
    V = 16 ** 4
    G = lt.GaugeField(ext, "fp64")
    G.SetToHaarRandom(123)
    lt.UpdateSweeps(G, 6.0, 10, 1, 4, seed=5)
    bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
    k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4)
    F, q0 = k.CalculateTopologicalForce(dvdq=1.0)
    F = F[..., 0] + 1j * F[..., 1]
    # the same configuration on FP32 links (config 3 runs FP32 links with the FP64 bias)
    links = G.download()
    G32 = lt.GaugeField(ext, "fp32")
    G32.upload(links)
    k32 = lt.HMCMetaDKernel(G32, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4)
    F32, q32 = k32.CalculateTopologicalForce(dvdq=1.0)
    F32 = F32[..., 0] + 1j * F32[..., 1]
    assert q32 == pytest.approx(q0, abs=1e-5)
    rng = np.random.default_rng(7)
    h = 1e-4
    worst = {"fp64": [0.0, 0.0], "fp32": [0.0, 0.0]}
    for link in rng.choice(4 * V, size=64, replace=False):
        site, mu = divmod(int(link), 4)
        U0 = G.get_link(site, mu)
        fd = np.empty(8)
        for a in range(8):
            G.set_link(site, mu, exp_lambda(a, h) @ U0)
            qp = k.MetaCharge()
            G.set_link(site, mu, exp_lambda(a, -h) @ U0)
            qm = k.MetaCharge()
            fd[a] = 0.5 * (qp - qm) / h
        G.set_link(site, mu, U0)
        for name, FF in (("fp64", F), ("fp32", F32)):
            adj = np.array([np.real(np.trace(GELL_MANN[a] @ (1j * FF[site, mu]))) for a in range(8)])
            d = np.abs(adj - fd).max()
            worst[name][0] = max(worst[name][0], d)
            worst[name][1] = max(worst[name][1], d / max(np.abs(fd).max(), 1e-12))
    print("adjoint vs finite differences (max abs, max rel):", worst)
    assert worst["fp64"][0] < 1e-6, worst
    assert worst["fp32"][0] < 1e-6, worst
