"""GPU parity of the eleven molecular-dynamics integrators of the reference
(updates/hmc_gauge.hpp:19-377, updates/hmc_metadynamics.hpp:26-238) on HMCKernel and
HMCMetaDKernel, and of ParityUpdate (updates/parity_update.hpp:22-47).

FP64 links: links and momenta after a 3-step trajectory within 1e-10 of the reference fixture
(relative to the largest entry; the chains of exponentials and stout forces differ from the
reference only in summation order), H within 1e-11 relative.  The bias on the GPU is the
reference's grid potential holding V(Q) = 0.7 Q, whose derivative equals the slope to rounding.
ParityUpdate moves and conjugates links, so FP64 results are bit-identical.
"""
import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import haar_links_numpy, rel_err

pytestmark = pytest.mark.gpu

MD_CASES = [(i, False) for i in range(8)] + [(i, True) for i in (0, 1, 2, 3, 4, 5, 8, 9, 10)]
BY_ID = {i.ID: i for i in vars(lt.Integrators.HMC).values()}


def gpu(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


def linear_bias(slope):
    b = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
    b.GeneratePotentialFrom(lambda cv: slope * cv)
    return b


def kernel(G, integ, metad, g=None, slope=0.7, n_stout=None, beta=6.0, tau=0.5, seed=1):
    if metad:
        n = int(g["n_stout"]) if n_stout is None else n_stout
        return lt.HMCMetaDKernel(G, linear_bias(slope), lt.WilsonAction(beta), tau, 0.12, n, seed=seed,
                                 integrator=BY_ID[integ])
    return lt.HMCKernel(G, lt.WilsonAction(beta), tau, seed=seed, integrator=BY_ID[integ])


class TestIntegrators:
    @pytest.mark.parametrize("integ,metad", MD_CASES)
    def test_against_reference_fixture(self, golden_md, integ, metad):
        g = golden_md
        ext = tuple(int(e) for e in g["ext"])
        G = gpu(ext, g["U"])
        k = kernel(G, integ, metad, g)
        k.SetMomenta(g["P"])
        ho, hn = k.Integrate(int(g["n_step"]))
        key = f"{'metad' if metad else 'gauge'}{integ}"
        assert ho == pytest.approx(g[key + "_h"][0], rel=1e-11)
        assert hn == pytest.approx(g[key + "_h"][1], rel=1e-11)
        links = g["links"]
        assert rel_err(G.download().reshape(-1, 18)[links], g[key + "_U"]) < 1e-10
        assert rel_err(k.GetMomenta().reshape(-1, 18)[links], g[key + "_P"]) < 1e-10

    @pytest.mark.parametrize("integ", [8, 9, 10])
    def test_multiple_timescale_against_oracle(self, oracle, integ):
        """Another lattice, bias slope and stout depth than the fixture."""
        ext = (4, 4, 4, 6)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 31), 5.9, 4, 2, 0)
        P = oracle.random_momenta(ext, 5, 3)
        G = gpu(ext, U)
        k = kernel(G, integ, True, slope=-1.9, n_stout=2, beta=5.9, tau=0.3)
        k.SetMomenta(P)
        ho, hn = k.Integrate(2)
        U2, P2, oh, on = oracle.md_integrate(ext, U, P, 5.9, 0.3, 2, integ, True, 0.12, 2, -1.9)
        assert rel_err(G.download(), U2) < 1e-10 and rel_err(k.GetMomenta(), P2) < 1e-10
        assert ho == pytest.approx(oh, rel=1e-11) and hn == pytest.approx(on, rel=1e-11)

    @pytest.mark.parametrize("integ", [1, 5, 8, 10])
    def test_reversibility(self, oracle, integ):
        ext = (4, 4, 4, 4)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 12), 6.0, 4, 8, 0)
        G = gpu(ext, U)
        k = kernel(G, integ, integ >= 8, slope=1.3, n_stout=2)
        ho, hn = k.ReversibilityTest(4, counter=2)
        assert abs(hn - ho) < 1e-9 * abs(ho)
        assert rel_err(G.download(), U) < 1e-9

    def test_trajectory_matches_oracle(self, oracle):
        """lt_md_trajectory with OMF_4: the Philox momenta and the dynamics of the oracle."""
        ext = (4, 4, 4, 4)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 13), 6.0, 4, 8, 0)
        G = gpu(ext, U)
        k = lt.HMCKernel(G, lt.WilsonAction(6.0), 1.0, seed=77, counter=5, integrator=lt.OMF_4)
        k(6, False)
        P = oracle.random_momenta(ext, 77, 5)
        U2, _, ho, hn = oracle.md_integrate(ext, U, P, 6.0, 1.0, 6, 5)
        assert k.delta_H == pytest.approx(hn - ho, rel=1e-8, abs=1e-10)
        assert rel_err(G.download(), U2) < 1e-10
        assert k.counter.value == 6

    @pytest.mark.parametrize("integ", [lt.OMF_4, lt.OMF_2_OMF_4, lt.Leapfrog_OMF_4])
    def test_metad_trajectories_update_bias(self, oracle, integ):
        ext = (8, 8, 8, 8)
        U = oracle.heatbath(ext, lt.haar_links(ext, 42), 6.0, 5, 99, 0)
        G = gpu(ext, U, "fp32_12")
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4, seed=11, integrator=integ)
        acc = [k(8, True) for _ in range(3)]
        assert sum(acc) >= 2
        assert bias.grid().max() > 0.0
        assert np.allclose(bias.grid(), bias.grid()[::-1])
        assert abs(k.cv) < 8

    def test_fp32_storage(self, oracle):
        ext = (8, 8, 8, 8)
        U = oracle.heatbath(ext, lt.haar_links(ext, 4), 6.0, 4, 3, 0)
        P = oracle.random_momenta(ext, 6, 0)
        _, _, oh, on = oracle.md_integrate(ext, U, P, 6.0, 0.5, 4, 5)
        for prec in ("fp32", "fp32_12"):
            G = gpu(ext, U, prec)
            k = lt.HMCKernel(G, lt.WilsonAction(6.0), 0.5, integrator=lt.OMF_4)
            k.SetMomenta(P)
            ho, hn = k.Integrate(4)
            assert ho == pytest.approx(oh, rel=1e-6) and hn == pytest.approx(on, rel=1e-6)

    def test_kernel_rejects_foreign_integrators(self):
        G = lt.GaugeField((4, 4, 4, 4))
        with pytest.raises(ValueError):
            lt.HMCKernel(G, lt.WilsonAction(6.0), integrator=lt.Leapfrog_OMF_4)
        with pytest.raises(ValueError):
            lt.HMCMetaDKernel(G, linear_bias(1.0), lt.WilsonAction(6.0), integrator=lt.OMF_4_friction_slow)
        G.upload(lt.haar_links((4, 4, 4, 4), 1))
        k = lt.HMCKernel(G, lt.WilsonAction(6.0))
        k.RandomMomentum(0)
        with pytest.raises(lt.LettuceError):   # the C ABI refuses a bias-only integrator without a bias
            lt.api.check(lt.api.lib().lt_md_integrate(G.handle, None, 8, 6.0, 1.0, 2, 0.12, 4, None, None))


class TestParity:
    def test_against_reference_fixture(self, golden_md):
        g = golden_md
        ext = tuple(int(e) for e in g["ext"])
        G = gpu(ext, g["U"])
        lt.ParityUpdate(G)
        R = G.download()
        assert np.array_equal(R.reshape(-1, 18)[g["links"]], g["parity_U"])

    def test_against_oracle_and_involution(self, oracle):
        ext = (6, 4, 8, 10)
        U = haar_links_numpy(ext, 21)
        G = gpu(ext, U)
        lt.ParityUpdate(G)
        assert np.array_equal(G.download(), oracle.parity_update(ext, U))
        lt.ParityUpdate(G)
        assert np.array_equal(G.download(), U)

    @pytest.mark.parametrize("prec", ["fp64", "fp32", "fp32_12"])
    def test_charge_flips_action_kept(self, oracle, prec):
        ext = (8, 8, 8, 8)
        U = oracle.heatbath(ext, lt.haar_links(ext, 8), 6.0, 5, 2, 0)
        G = gpu(ext, U, prec)
        lt.StoutSmearingN(G, G, 5, 0.12)
        q, s = lt.TopChargeClover(G), lt.WilsonAction(6.0).Action(G)
        lt.ParityUpdate(G)
        tol = 1e-12 if prec == "fp64" else 1e-5
        assert lt.TopChargeClover(G) == pytest.approx(-q, rel=tol, abs=tol)
        assert lt.WilsonAction(6.0).Action(G) == pytest.approx(s, rel=tol)


@pytest.mark.parametrize("prec", ["fp64", "fp32_12"])
def test_metad_trajectories_with_binned_bias(oracle, prec):
    """MetaD-HMC with the Gaussian-free binned deposits (the metadynamics configuration):
    every trajectory deposits symmetrically at its path samples, so without tempering the grid
    sum grows by 2 weight per sample and the deposits form mirror pairs."""
    import lettuce_b200 as lt
    from ltref import haar_links_numpy
    ext = (8, 8, 8, 8)
    U = oracle.heatbath(ext, haar_links_numpy(ext, 12), 6.0, 10, 3, 0)
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 1e300, 1000)
    bias.SetUpdateMode("binned")
    hmc = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4, seed=9)
    sums = [0.0]
    for _ in range(3):
        hmc(10, True)
        g = bias.grid()
        sums.append(g.sum())
        assert np.allclose(g, g[::-1], rtol=1e-12, atol=1e-14)
    steps = np.diff(sums) / (2 * 0.05)
    assert np.all(steps >= 1) and np.allclose(steps, np.round(steps), atol=1e-9)
    assert np.count_nonzero(bias.grid()) <= 4 * int(round(sum(steps)))
