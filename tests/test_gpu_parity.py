"""GPU parity: the CUDA path (through the C ABI) against the C oracle on identical inputs.

FP64 tolerance: 1e-12 relative to the field's largest entry for single-call kernels and
whole RK3 flows (the only differences are summation order and libm rounding); chains of
molecular dynamics allow 1e-10.  FP32 storage: the tolerances stated per test.
"""
import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def gpu(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


@pytest.fixture(scope="module")
def therm4(oracle, golden4):
    """4^4 start thermalised by 10 oracle heatbath sweeps at beta = 6 (deterministic)."""
    return oracle.heatbath(golden4["ext"], golden4["U"], 6.0, 10, 1234, 0)


@pytest.fixture(scope="module")
def therm8(oracle):
    ext = (8, 8, 8, 8)
    U = lt.haar_links(ext, 42)
    return oracle.heatbath(ext, U, 6.0, 5, 99, 0)


class TestContainer:
    def test_roundtrip_fp64_exact(self, golden4):
        G = gpu(golden4["ext"], golden4["U"])
        assert np.array_equal(G.download(), golden4["U"])

    def test_roundtrip_fp32(self, golden4):
        G = gpu(golden4["ext"], golden4["U"], "fp32")
        assert rel_err(G.download(), golden4["U"]) < 1e-7

    def test_roundtrip_fp32_12(self, golden4):
        G = gpu(golden4["ext"], golden4["U"], "fp32_12")
        assert rel_err(G.download(), golden4["U"]) < 1e-6

    @pytest.mark.parametrize("ext", [(4, 6, 8, 10), (2, 4, 2, 6), (16, 16, 16, 16), (16, 8, 18, 32)])
    def test_repeated_upload_packs_on_host_identically(self, ext):
        """From its second upload on, a two-row FP32 handle packs the links into the stored
        format on the host threads (single- and multi-threaded by volume) and copies them in
        chunks; the stored field must be bit for bit the one the device conversion of the first
        upload makes."""
        U1, U2 = lt.haar_links(ext, 71), lt.haar_links(ext, 72)
        fresh = []
        for U in (U1, U2):
            F = lt.GaugeField(ext, "fp32_12")
            F.upload(U)            # first upload: device conversion
            fresh.append(F.download())
        G = lt.GaugeField(ext, "fp32_12")
        G.upload(U2)
        for k, U in enumerate((U1, U2, U1)):
            G.upload(U)            # packed on the host
            assert np.array_equal(G.download(), fresh[k % 2]), k

    @pytest.mark.parametrize("ext", [(16, 16, 16, 16), (16, 8, 18, 32)])
    def test_repeated_upload_from_pinned_memory_splits_identically(self, ext):
        """From pinned host memory the repeated upload sends a share of the sites (the last) as
        FP64 over PCIe (converted on the device) while the host threads pack the rest; the
        stored field is again bit for bit the device conversion's."""
        import torch
        U1, U2 = lt.haar_links(ext, 73), lt.haar_links(ext, 74)
        pinned = torch.empty(U1.size, dtype=torch.float64, pin_memory=True)
        host = pinned.numpy().reshape(U1.shape)
        fresh = []
        for U in (U1, U2):
            F = lt.GaugeField(ext, "fp32_12")
            F.upload(U)
            fresh.append(F.download())
        G = lt.GaugeField(ext, "fp32_12")
        V = int(np.prod(ext))
        assert G.upload_bytes(host) == V * 576            # first upload: the FP64 field
        G.upload(U1)
        assert G.upload_bytes(U1) == V * 4 * 48           # pageable: packed whole
        split = G.upload_bytes(host)
        assert V * 4 * 48 < split < V * 576               # pinned: partly FP64
        for k, U in enumerate((U1, U2, U1)):
            host[...] = U
            G.upload(host)
            assert np.array_equal(G.download(), fresh[k % 2]), k

    def test_identity_and_copy_swap(self, golden4):
        ext = golden4["ext"]
        A, B = gpu(ext, golden4["U"]), lt.GaugeField(ext)
        assert lt.PlaquetteSum(B) == pytest.approx(18.0 * int(np.prod(ext)), rel=1e-15)
        B.assign(A)
        assert np.array_equal(B.download(), golden4["U"])
        B.SetToIdentity()
        lt.Swap(A, B)
        assert np.array_equal(B.download(), golden4["U"])
        assert lt.PlaquetteSum(A) == pytest.approx(18.0 * int(np.prod(ext)), rel=1e-15)

    def test_single_link_access(self, golden4):
        ext = golden4["ext"]
        G = gpu(ext, golden4["U"])
        U = golden4["U"]
        for site, mu in [(0, 0), (5, 3), (255, 1)]:
            ref = U[site, mu, ..., 0] + 1j * U[site, mu, ..., 1]
            assert np.array_equal(G.get_link(site, mu), ref)
        G.set_link(7, 2, np.eye(3))
        assert np.array_equal(G.get_link(7, 2), np.eye(3))

    def test_bad_arguments_raise(self):
        with pytest.raises(lt.LettuceError):
            lt.GaugeField((4, 4, 4, 5))
        G = lt.GaugeField((4, 4, 4, 4))
        with pytest.raises(lt.LettuceError):
            G.get_link(256, 0)


class TestObservables:
    @pytest.mark.parametrize("which", ["hot", "therm"])
    def test_plaquette_action_clover(self, oracle, golden4, therm4, which):
        ext = golden4["ext"]
        U = golden4["U"] if which == "hot" else therm4
        G = gpu(ext, U)
        assert lt.PlaquetteSum(G) == pytest.approx(oracle.plaquette_sum(ext, U), rel=TOL)
        assert lt.WilsonAction(6.0).Action(G) == pytest.approx(oracle.wilson_action(ext, U, 6.0), rel=TOL)
        q, e = lt.CloverObservables(G)
        assert q == pytest.approx(oracle.topcharge(ext, U), rel=1e-10, abs=1e-13)
        assert e == pytest.approx(oracle.energy(ext, U), rel=TOL)

    def test_golden_values(self, golden4):
        """Directly against the reference's own numbers."""
        G = gpu(golden4["ext"], golden4["U"])
        assert lt.PlaquetteSum(G) == pytest.approx(float(golden4["plaq"]), rel=TOL)
        assert lt.TopChargeClover(G) == pytest.approx(float(golden4["Q"]), rel=1e-10, abs=1e-13)
        assert lt.EnergyDensityClover(G) == pytest.approx(float(golden4["E"]), rel=TOL)

    def test_uneven_extents(self, oracle, golden_odd):
        from ltref import haar_links_numpy
        ext = tuple(golden_odd["ext"])
        U = haar_links_numpy(ext, int(golden_odd["seed"]))
        G = gpu(ext, U)
        assert lt.PlaquetteSum(G) == pytest.approx(float(golden_odd["plaq"]), rel=TOL)
        q, e = lt.CloverObservables(G)
        assert q == pytest.approx(float(golden_odd["Q"]), rel=1e-10, abs=1e-13)
        assert e == pytest.approx(float(golden_odd["E"]), rel=TOL)
        S = lt.Staples(G)
        assert rel_err(S.reshape(-1, 18)[golden_odd["links"]], golden_odd["staples"]) < TOL

    def test_staples(self, oracle, therm8):
        ext = (8, 8, 8, 8)
        G = gpu(ext, therm8)
        assert rel_err(lt.Staples(G), oracle.staples(ext, therm8)) < TOL


class TestLocalUpdates:
    def test_overrelaxation_sweep(self, oracle, therm8):
        ext = (8, 8, 8, 8)
        G = gpu(ext, therm8)
        lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 1)
        assert rel_err(G.download(), oracle.overrelax(ext, therm8, 1)) < TOL

    @pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
    def test_overrelaxation_sweep_fp32(self, oracle, therm8, prec):
        """FP32 storage and arithmetic against the FP64 oracle: one deterministic sweep."""
        ext = (8, 8, 8, 8)
        G = gpu(ext, therm8, prec)
        lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 1)
        assert rel_err(G.download(), oracle.overrelax(ext, therm8, 1)) < 1e-5

    def test_overrelaxation_conserves_action(self, therm8):
        G = gpu((8, 8, 8, 8), therm8)
        p0 = lt.PlaquetteSum(G)
        lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 20)
        assert lt.PlaquetteSum(G) == pytest.approx(p0, rel=1e-12)

    def test_heatbath_sweep_same_stream(self, oracle, therm8):
        """One sweep from identical input with the identical Philox stream."""
        ext = (8, 8, 8, 8)
        G = gpu(ext, therm8)
        hb = lt.HeatbathKernel(G, lt.WilsonAction(6.0), seed=777, counter=5)
        lt.Iterator.Checkerboard(hb, 1)
        assert hb.counter.value == 6
        assert rel_err(G.download(), oracle.heatbath(ext, therm8, 6.0, 1, 777, 5)) < 1e-11

    def test_heatbath_sweep_fp32_storages_same_stream(self, therm8):
        """The FP32 sampler on two-row links (staged staple, third row rebuilt) against the same
        sampler on full FP32 links: same Philox stream, same proposals, so all links but those
        whose accept/reject comparison falls within FP32 rounding of its threshold agree to
        FP32 accuracy."""
        ext = (8, 8, 8, 8)
        out = []
        for prec in ("fp32", "fp32_12"):
            G = gpu(ext, therm8, prec)
            lt.Iterator.Checkerboard(lt.HeatbathKernel(G, lt.WilsonAction(6.0), seed=777, counter=5), 2)
            out.append(G.download())
        d = np.abs(out[0] - out[1]).reshape(-1, 18).max(axis=1)
        assert np.median(d) < 1e-5
        assert np.mean(d > 1e-3) < 0.01

    def test_heatbath_keeps_group(self, therm8):
        G = gpu((8, 8, 8, 8), therm8, "fp32")
        lt.Iterator.Checkerboard(lt.HeatbathKernel(G, lt.WilsonAction(6.0), seed=3), 3)
        M = G.download()
        M = (M[..., 0] + 1j * M[..., 1]).reshape(-1, 3, 3)
        err = np.abs(np.einsum("nij,nkj->nik", M, M.conj()) - np.eye(3)).max()
        assert err < 1e-6
        assert np.abs(np.linalg.det(M) - 1).max() < 1e-5


class TestSmearing:
    def test_flow_rk3(self, oracle, golden4):
        ext = golden4["ext"]
        G, H = gpu(ext, golden4["U"]), lt.GaugeField(ext)
        lt.GradientFlowKernel(G, H, lt.RK3, None, 0.01)(10)
        F = H.download()
        assert rel_err(F.reshape(-1, 18)[golden4["links"]], golden4["flow10"]) < TOL
        assert rel_err(F, oracle.flow_rk3(ext, golden4["U"], 0.01, 10)) < TOL

    def test_flow_resume_and_measure(self, golden4):
        ext = golden4["ext"]
        G, H = gpu(ext, golden4["U"]), lt.GaugeField(ext)
        flow = lt.GradientFlowKernel(G, H, lt.RK3, None, 0.01)
        p, q, e = flow.Measure(2, 5)
        np.testing.assert_allclose(p, golden4["flowm_plaq"], rtol=TOL)
        np.testing.assert_allclose(q, golden4["flowm_q"], rtol=1e-10, atol=1e-13)
        np.testing.assert_allclose(e, golden4["flowm_e"], rtol=TOL)
        flow(5)
        flow.Resume(5)
        assert rel_err(H.download().reshape(-1, 18)[golden4["links"]], golden4["flow10"]) < TOL

    def test_flow_to_t0(self, therm8):
        """t0 from t^2 E(t) = target: the step-by-step measurements (parity-checked above)
        interpolated here must give the library's t0."""
        ext = (8, 8, 8, 8)
        eps, target = 0.02, 0.05
        G, H = gpu(ext, therm8), lt.GaugeField(ext)
        flow = lt.GradientFlowKernel(G, H, lt.RK3, None, eps)
        t0, q = flow.FlowToT0(target, 2000)
        n = int(np.ceil(t0 / eps)) + 1
        _, _, e = flow.Measure(n, 1)
        t = eps * np.arange(1, n + 1)
        y = t * t * e
        k = int(np.argmax(y >= target))
        expect = t[k - 1] + (target - y[k - 1]) / (y[k] - y[k - 1]) * eps
        assert t0 == pytest.approx(expect, rel=1e-12)
        with pytest.raises(lt.LettuceError):
            flow.FlowToT0(target, 2)

    def test_stout(self, oracle, golden4):
        ext = golden4["ext"]
        G, H = gpu(ext, golden4["U"]), lt.GaugeField(ext)
        lt.StoutSmearingN(G, H, 4, 0.12)
        assert rel_err(H.download().reshape(-1, 18)[golden4["links"]], golden4["stout4"]) < TOL

    @pytest.mark.parametrize("prec,tol", [("fp32", 2e-6), ("fp32_12", 2e-6)])
    def test_flow_fp32_plaquette(self, oracle, therm8, prec, tol):
        """FP32 bulk flow vs the FP64 oracle: |dP| of the normalised plaquette after t = 0.2."""
        ext = (8, 8, 8, 8)
        V = 8 ** 4
        G, H = gpu(ext, therm8, prec), lt.GaugeField(ext, prec)
        lt.GradientFlowKernel(G, H, lt.RK3, None, 0.01)(20)
        ref = oracle.flow_rk3(ext, therm8, 0.01, 20)
        p32 = lt.PlaquetteSum(H) / V / 18
        p64 = oracle.plaquette_sum(ext, ref) / V / 18
        assert abs(p32 - p64) < tol


class TestHMC:
    def test_gauge_force(self, oracle, golden4):
        ext = golden4["ext"]
        G = gpu(ext, golden4["U"])
        F = lt.WilsonAction(6.0).Force(G)
        assert rel_err(F.reshape(-1, 18)[golden4["links"]], golden4["gforce"]) < TOL

    def test_random_momenta_same_stream(self, oracle, golden4):
        ext = golden4["ext"]
        G = gpu(ext, golden4["U"])
        hmc = lt.HMCKernel(G, lt.WilsonAction(6.0), 1.0, seed=9)
        hmc.RandomMomentum(3)
        assert rel_err(hmc.GetMomenta(), oracle.random_momenta(ext, 9, 3)) < 1e-13

    def test_omf2_against_reference(self, golden4):
        ext = golden4["ext"]
        G = gpu(ext, golden4["U"])
        hmc = lt.HMCKernel(G, lt.WilsonAction(6.0), 1.0)
        hmc.SetMomenta(golden4["P"])
        ho, hn = hmc.Integrate(10)
        assert ho == pytest.approx(golden4["omf2_h"][0], rel=TOL)
        assert hn == pytest.approx(golden4["omf2_h"][1], rel=1e-11)
        links = golden4["links"]
        assert rel_err(G.download().reshape(-1, 18)[links], golden4["omf2_U"]) < 1e-10
        assert rel_err(hmc.GetMomenta().reshape(-1, 18)[links], golden4["omf2_P"]) < 1e-10

    def test_reversibility(self, therm8):
        """ReversibilityTest (updates/hmc_gauge.hpp:585-599): integrate, flip momenta, integrate."""
        G = gpu((8, 8, 8, 8), therm8)
        hmc = lt.HMCKernel(G, lt.WilsonAction(6.0), 1.0, seed=4)
        hmc.RandomMomentum(0)
        ho, _ = hmc.Integrate(10)
        hmc.SetMomenta(-hmc.GetMomenta())
        _, hn = hmc.Integrate(10)
        assert abs(hn - ho) < 1e-8 * abs(ho)
        assert rel_err(G.download(), therm8) < 1e-10


class TestMetaD:
    def test_clover_derivative(self, golden4):
        G = gpu(golden4["ext"], golden4["U"])
        D = lt.CloverDerivative(G)
        assert rel_err(D.reshape(-1, 18)[golden4["links"]], golden4["cderiv"]) < TOL

    def test_metad_force_against_reference(self, golden4):
        G = gpu(golden4["ext"], golden4["U"])
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, int(golden4["metad_nstout"]))
        F, q = k.CalculateTopologicalForce(dvdq=1.0)
        assert q == pytest.approx(float(golden4["metad_q"]), rel=1e-11)
        assert rel_err(F.reshape(-1, 18)[golden4["links"]], golden4["metad"]) < 1e-11

    def test_metad_force_against_oracle(self, oracle, therm8):
        ext = (8, 8, 8, 8)
        G = gpu(ext, therm8)
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 3)
        F, q = k.CalculateTopologicalForce(dvdq=0.7)
        Fo, qo = oracle.metad_force(ext, therm8, 0.12, 3, 0.7)
        assert q == pytest.approx(qo, rel=1e-11, abs=1e-13)
        assert rel_err(F, Fo) < 1e-11

    @pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
    def test_metad_force_fp32(self, oracle, therm8, prec):
        """FP32 links: the whole chain in FP32 (the stout adjoint's exponential derivative
        from the series) against the FP64 oracle on the same rounded links: 1e-5 of the
        largest force entry, Q to 1e-5."""
        ext = (8, 8, 8, 8)
        G = gpu(ext, therm8, prec)
        W = G.download()
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4)
        F, q = k.CalculateTopologicalForce(dvdq=0.7)
        Fo, qo = oracle.metad_force(ext, W, 0.12, 4, 0.7)
        assert q == pytest.approx(qo, abs=1e-5)
        assert rel_err(F, Fo) < 1e-5

    @pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("fp32", 1e-4)])
    def test_metad_reversibility(self, therm8, prec, tol):
        """ReversibilityTest of the MetaD kernel (updates/hmc_metadynamics.hpp:657-674)."""
        G = gpu((8, 8, 8, 8), therm8, prec)
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        bias.GeneratePotentialFrom(lambda cv: 3.0 * np.sin(cv))
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4, seed=3)
        k.RandomMomentum(0)
        start = G.download()
        ho, _ = k.Integrate(10)
        k.SetMomenta(-k.GetMomenta())
        _, hn = k.Integrate(10)
        assert abs(hn - ho) < tol * abs(ho)
        assert rel_err(G.download(), start) < (1e-9 if prec == "fp64" else 1e-4)

    def test_metad_trajectories_accept_and_update_bias(self, therm8):
        G = gpu((8, 8, 8, 8), therm8)
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4, seed=11)
        acc = [k(10, True) for _ in range(4)]
        assert sum(acc) >= 2
        assert bias.grid().max() > 0.0   # the symmetric well-tempered deposits happened
        assert np.allclose(bias.grid(), bias.grid()[::-1])   # symmetric updates
        assert abs(k.cv) < 8

    def test_metad_omf2_against_reference(self, golden4):
        ext = golden4["ext"]
        G = gpu(ext, golden4["U"])
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        bias.GeneratePotentialFrom(lambda cv: 0.5 * cv)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, int(golden4["metad_nstout"]))
        k.SetMomenta(golden4["P"])
        ho, hn = k.Integrate(4)
        assert ho == pytest.approx(golden4["momf2_h"][0], rel=1e-11)
        assert hn == pytest.approx(golden4["momf2_h"][1], rel=1e-10)
        links = golden4["links"]
        assert rel_err(G.download().reshape(-1, 18)[links], golden4["momf2_U"]) < 1e-9
        assert rel_err(k.GetMomenta().reshape(-1, 18)[links], golden4["momf2_P"]) < 1e-9
