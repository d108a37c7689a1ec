"""GPU parity at the benchmarked sizes: the 32^4 configuration of the headline and the 16^4
configuration of the metadynamics force, against the reference's own code.

Inputs are regenerated here bit for bit (numpy Haar start plus one C-oracle heatbath sweep,
ltref.large_input) and checked against the checksum stored with the fixture.  Expected
outputs come from tests/golden/ref_32x32x32x32.npz, ref_flow_32x32x32x32.npz and
ref_metad_16x16x16x16.npz (written by tests/golden/gen_golden.py from the reference harness,
and, for the heatbath, from the C oracle's Philox stream): 256 sampled links plus full-field
checksums per output.  Where the reference harness is built (oracle/_ref), the whole field
is compared as well.

Tolerances: FP64, 1e-12 of the largest entry per link (heatbath 1e-11, as for the small
lattices; flows of 400 steps 1e-10 on Q); checksums within 1e-12 of the sum of |entries|.
Two-row FP32 links (the bench's storage) against the FP64 reference on the same input:
1e-5 of the largest entry for one sweep or 10 flow steps, and the normalised plaquette
within 1e-6 (the north star's bound) after the flow to t = 4.
"""
import os

import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import Reference, checksums, large_input, ref_available, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def ck_close(field, ck, tol=TOL):
    got = checksums(field)
    scale = np.abs(field).sum()
    assert np.all(np.abs(got - ck) <= tol * scale * np.array([1.0, 1.0, 97.0])), (got, ck)


def samples(field, links):
    return field.reshape(-1, 18)[links]


@pytest.fixture(scope="module")
def big(oracle):
    d = load("ref_32x32x32x32.npz")
    ext = tuple(int(e) for e in d["ext"])
    d["ext"] = ext
    d["U"] = large_input(ext, int(d["seed"]), int(d["hb_seed"]), oracle)
    np.testing.assert_allclose(checksums(d["U"]), d["U_ck"], rtol=1e-13)
    return d


def gpu(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


class TestBenchmarkedLattice:
    def test_overrelaxation_fp64(self, big):
        G = gpu(big["ext"], big["U"])
        lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 1)
        F = G.download()
        assert rel_err(samples(F, big["links"]), big["or1"]) < TOL
        ck_close(F, big["or1_ck"])
        assert lt.PlaquetteSum(G) == pytest.approx(float(big["or1_plaq"]), rel=TOL)
        if ref_available(big["ext"]):
            assert rel_err(F, Reference(big["ext"]).overrelax(big["U"], 1)) < TOL

    def test_heatbath_fp64_same_stream(self, big):
        """One FP64 sweep with the C oracle's Philox stream (seed 555, counter 3)."""
        G = gpu(big["ext"], big["U"])
        lt.Iterator.Checkerboard(lt.HeatbathKernel(G, lt.WilsonAction(6.0), seed=555, counter=3), 1)
        F = G.download()
        assert rel_err(samples(F, big["links"]), big["hb1_oracle"]) < 1e-11
        ck_close(F, big["hb1_oracle_ck"], 1e-11)

    def test_flow_rk3_fp64(self, big):
        ext = big["ext"]
        G, H = gpu(ext, big["U"]), lt.GaugeField(ext)
        lt.GradientFlowKernel(G, H, lt.RK3, None, 0.01)(10)
        F = H.download()
        assert rel_err(samples(F, big["links"]), big["flow10"]) < TOL
        ck_close(F, big["flow10_ck"])
        assert lt.PlaquetteSum(H) == pytest.approx(float(big["flow10_plaq"]), rel=TOL)
        assert lt.TopChargeClover(H) == pytest.approx(float(big["flow10_q"]), rel=1e-10, abs=1e-10)
        if ref_available(ext):
            assert rel_err(F, Reference(ext).flow_rk3(big["U"], 0.01, 10)) < TOL

    def test_observables_fp64(self, big):
        G = gpu(big["ext"], big["U"])
        assert lt.PlaquetteSum(G) == pytest.approx(float(big["plaq"]), rel=TOL)
        assert lt.TopChargeClover(G) == pytest.approx(float(big["Q"]), rel=1e-10, abs=1e-10)
        assert lt.EnergyDensityClover(G) == pytest.approx(float(big["E"]), rel=TOL)

    def test_overrelaxation_fp32_12(self, big):
        G = gpu(big["ext"], big["U"], "fp32_12")
        lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 1)
        F = G.download()
        assert rel_err(samples(F, big["links"]), big["or1"]) < 1e-5
        ck_close(F, big["or1_ck"], 1e-6)

    def test_flow_rk3_fp32_12(self, big):
        ext = big["ext"]
        G, H = gpu(ext, big["U"], "fp32_12"), lt.GaugeField(ext, "fp32_12")
        lt.GradientFlowKernel(G, H, lt.RK3, None, 0.01)(10)
        F = H.download()
        assert rel_err(samples(F, big["links"]), big["flow10"]) < 1e-5
        V = int(np.prod(ext))
        assert abs(lt.PlaquetteSum(H) - float(big["flow10_plaq"])) / V / 18 < 1e-6

    def test_heatbath_fp32_storages_same_stream(self, big):
        """The FP32 sampler on two-row links against the same sampler on 18-real FP32 links."""
        out = []
        for prec in ("fp32", "fp32_12"):
            G = gpu(big["ext"], big["U"], prec)
            lt.Iterator.Checkerboard(lt.HeatbathKernel(G, lt.WilsonAction(6.0), seed=555, counter=3), 1)
            out.append(G.download())
        d = np.abs(out[0] - out[1]).reshape(-1, 18).max(axis=1)
        assert np.median(d) < 1e-5
        assert np.mean(d > 1e-3) < 0.01


@pytest.fixture(scope="module")
def ref():
    return load("ref_flow_32x32x32x32.npz")


class TestFlowToFour:
    """The config-2 flow (RK3, eps = 0.01, t = 4) of the 32^4 input against the reference's
    FP64 flow: P, Q and E at t = 0.5, 1, ..., 4."""

    def flow(self, big, prec, ref):
        ext = big["ext"]
        G, H = gpu(ext, big["U"], prec), lt.GaugeField(ext, prec)
        p, q, e = lt.GradientFlowKernel(G, H, lt.RK3, None, float(ref["eps"])).Measure(len(ref["t"]),
                                                                                      int(ref["every"]))
        return np.asarray(p), np.asarray(q), np.asarray(e)

    def test_fp64(self, big, ref):
        p, q, e = self.flow(big, "fp64", ref)
        np.testing.assert_allclose(p, ref["plaq"], rtol=TOL)
        np.testing.assert_allclose(e, ref["E"], rtol=1e-11)
        assert np.max(np.abs(q - ref["Q"])) < 1e-10

    def test_fp32_12(self, big, ref):
        """Two-row FP32 links: the normalised plaquette within 1e-6 at every t.  The absolute
        |dQ| is reported, not held to 1e-6: this input is one heatbath sweep from a hot start, Q
        still moves by tens while it flows (-44 at t = 1, -4 at t = 4), and along those
        unstable directions the FP32 rounding of every stored stage grows about twofold per
        half unit of flow time (measured on a B200: 7e-6 at t = 0.5 and 1, 9.5e-4 at t = 4).
        The bounds below hold those measured values with a factor two to show regressions."""
        p, q, e = self.flow(big, "fp32_12", ref)
        V = int(np.prod(big["ext"]))
        dP = np.abs(p - ref["plaq"]) / V / 18
        dQ = np.abs(q - ref["Q"])
        print(f"32^4 FP32-12 flow vs reference FP64: max |dP| {dP.max():.2e}, |dQ| by t {dQ}")
        assert dP.max() < 1e-6
        assert dQ[:2].max() < 2e-5
        assert dQ.max() < 2e-3


@pytest.fixture(scope="module")
def m16(oracle):
    d = load("ref_metad_16x16x16x16.npz")
    ext = tuple(int(e) for e in d["ext"])
    d["ext"] = ext
    d["U"] = large_input(ext, int(d["seed"]), int(d["hb_seed"]), oracle)
    np.testing.assert_allclose(checksums(d["U"]), d["U_ck"], rtol=1e-13)
    return d


class TestMetaDForce16:
    def force(self, m16, prec):
        G = gpu(m16["ext"], m16["U"], prec)
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, int(m16["metad_nstout"]))
        return k.CalculateTopologicalForce(dvdq=1.0)

    def test_fp64(self, m16):
        F, q = self.force(m16, "fp64")
        assert q == pytest.approx(float(m16["metad_q"]), rel=1e-11, abs=1e-12)
        assert rel_err(samples(F, m16["links"]), m16["metad"]) < 1e-11
        ck_close(F, m16["metad_ck"], 1e-11)

    def test_fp32_12(self, m16):
        F, q = self.force(m16, "fp32_12")
        assert q == pytest.approx(float(m16["metad_q"]), abs=1e-4)
        assert rel_err(samples(F, m16["links"]), m16["metad"]) < 2e-5
