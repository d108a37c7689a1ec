"""GPU parity of the measurement bundle of the reference driver (SU3_main.cpp:89-235) and of
the four gradient-flow integrators (smearing/gradient_flow.hpp:31-168).

FP64 links: every observable within 1e-12 (relative, absolute floor 1e-14 for quantities that
are sums of cancelling terms such as charges) of the C oracle and of the reference fixture;
flowed fields within 1e-12 of the oracle.  FP32 storage: the observables are evaluated in
FP64 from the widened links, so the differences come from the storage rounding of the links
alone (1e-6 relative on actions and loops, 1e-5 absolute on charges).
"""
import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import haar_links_numpy, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
KEYS = ("Q_plaq", "S_improved", "W2", "W4", "W8")


def gpu(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


def gpu_measure(G, beta):
    m = lt.Measure(G, beta)
    return {"q_t": m["TopChargeClov_timeslice"], "e_t": m["E_clov_timeslice"], "Q_plaq": m["TopChargePlaq"],
            "S_improved": m["Improved_Action"], "W2": m["Wilson_loop(L=2)"], "W4": m["Wilson_loop(L=4)"],
            "W8": m["Wilson_loop(L=8)"], "P": m["Polyakov_loop"], "all": m}


def assert_bundle(mine, ref, rtol, atol_q):
    for k in ("S_improved", "W2", "W4", "W8"):
        assert mine[k] == pytest.approx(float(ref[k]), rel=rtol), k
    assert mine["Q_plaq"] == pytest.approx(float(ref["Q_plaq"]), rel=rtol, abs=atol_q)
    assert mine["P"] == pytest.approx(complex(ref["P"]), rel=rtol, abs=atol_q)
    np.testing.assert_allclose(mine["q_t"], ref["q_t"], rtol=rtol, atol=atol_q)
    np.testing.assert_allclose(mine["e_t"], ref["e_t"], rtol=rtol, atol=atol_q)


@pytest.fixture(scope="module")
def therm_odd(oracle):
    """4 x 6 x 8 x 10 start thermalised by the oracle: every extent different, t first."""
    ext = (4, 6, 8, 10)
    return ext, oracle.heatbath(ext, haar_links_numpy(ext, 5), 5.9, 6, 77, 0)


class TestBundle:
    def test_against_reference_fixture(self, golden_measure):
        g = golden_measure
        ext = tuple(int(e) for e in g["ext"])
        assert_bundle(gpu_measure(gpu(ext, g["U"]), 6.0), g, TOL, 1e-14)

    def test_against_oracle_odd(self, oracle, therm_odd):
        ext, U = therm_odd
        G = gpu(ext, U)
        assert_bundle(gpu_measure(G, 6.2), oracle.measure(ext, U, 6.2), TOL, 1e-14)

    def test_timeslice_sums(self, oracle, therm_odd):
        ext, U = therm_odd
        G = gpu(ext, U)
        m = gpu_measure(G, 6.0)
        assert m["q_t"].sum() == pytest.approx(lt.TopChargeClover(G), rel=1e-12, abs=1e-13)
        assert m["e_t"].sum() == pytest.approx(lt.EnergyDensityClover(G), rel=1e-12)
        assert m["all"]["E_clov"] == pytest.approx(lt.EnergyDensityClover(G), rel=1e-12)
        assert m["all"]["Wilson_Action"] == pytest.approx(
            1.0 - lt.PlaquetteSum(G) / (18.0 * G.Volume()), rel=1e-14)

    @pytest.mark.parametrize("L", [1, 2, 3, 5, 8, 12])
    def test_wilson_loop_sizes(self, oracle, therm_odd, L):
        """Doubling path for powers of two, one-step extension otherwise; loops longer than an
        extent wrap around the periodic lattice."""
        ext, U = therm_odd
        want = oracle.lib.or_wilson_loop(oracle._e(ext), np.ascontiguousarray(U), L)
        assert lt.WilsonLoop(gpu(ext, U), L) == pytest.approx(want, rel=TOL)

    def test_wilson_loop_chain(self, golden_measure):
        """WilsonLoop<start, end, reset> with the chain kept between calls, against the
        reference: the doubling sequence, an extension by single links, and a reset away from
        the origin followed by a non-contiguous extension (the reference's literal semantics)."""
        g = golden_measure
        G = gpu(tuple(int(e) for e in g["ext"]), g["U"])
        for (a, b, r), want in zip(g["wl_chain_seq"], g["wl_chain"]):
            assert lt.WilsonLoopChain(G, int(a), int(b), bool(r)) == pytest.approx(float(want), rel=TOL), (a, b, r)
        H = lt.GaugeField((4, 4, 4, 4))
        with pytest.raises(lt.LettuceError):   # nothing to extend
            lt.WilsonLoopChain(H, 2, 4, False)
        lt.WilsonLoop(G, 2)                    # the plain form drops the kept chain
        with pytest.raises(lt.LettuceError):
            lt.WilsonLoopChain(G, 2, 4, False)

    def test_unit_field(self):
        ext = (4, 4, 6, 4)
        G = lt.GaugeField(ext)
        m = gpu_measure(G, 6.0)
        for k in ("S_improved", "W2", "W4", "W8", "Q_plaq"):
            assert abs(m[k]) < 1e-15, k
        assert m["P"] == pytest.approx(3.0, abs=1e-15)   # tr 1 over the spatial volume, as the reference
        assert np.all(np.abs(m["q_t"]) < 1e-15) and np.all(np.abs(m["e_t"]) < 1e-15)

    def test_rectangular_coefficients(self, oracle, therm_odd):
        ext, U = therm_odd
        G = gpu(ext, U)
        for cp, cr in ((1.0, 0.0), (0.0, 1.0), (3.648, -0.331)):
            want = oracle.lib.or_rect_action(oracle._e(ext), np.ascontiguousarray(U), 6.0, cp, cr)
            assert lt.RectangularAction(6.0, cp, cr).Action(G) == pytest.approx(want, rel=TOL)
        wilson = lt.RectangularAction(6.0, 1.0, 0.0).Action(G)
        assert wilson == pytest.approx(lt.WilsonAction(6.0).Action(G), rel=1e-12)

    @pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
    def test_fp32_storage(self, oracle, therm_odd, prec):
        ext, U = therm_odd
        G = gpu(ext, U, prec)
        W = G.download()
        assert_bundle(gpu_measure(G, 6.0), oracle.measure(ext, W, 6.0), 1e-11, 1e-13)
        assert_bundle(gpu_measure(G, 6.0), oracle.measure(ext, U, 6.0), 1e-6, 1e-5)


class TestFlowIntegrators:
    @pytest.mark.parametrize("integ", [lt.Euler, lt.RK2, lt.RK3, lt.RK3W7])
    def test_against_fixture(self, golden_measure, integ):
        g = golden_measure
        ext = tuple(int(e) for e in g["ext"])
        A, B = gpu(ext, g["U"]), lt.GaugeField(ext)
        flow = lt.GradientFlowKernel(A, B, integ, None, 0.02)
        flow(5)
        F = B.download().reshape(-1, 18)
        assert rel_err(F[g["links"]], g[f"flow{integ.ID}"]) < TOL

    @pytest.mark.parametrize("integ", [lt.Euler, lt.RK2, lt.RK3, lt.RK3W7])
    def test_against_oracle_and_resume(self, oracle, therm_odd, integ):
        ext, U = therm_odd
        A, B = gpu(ext, U), lt.GaugeField(ext)
        flow = lt.GradientFlowKernel(A, B, integ, None, 0.015)
        flow(3)
        flow.Resume(4)
        want = oracle.flow(ext, U, 0.015, 7, integ.ID)
        assert rel_err(B.download(), want) < TOL
        assert np.array_equal(A.download(), U)

    @pytest.mark.parametrize("integ", [lt.Euler, lt.RK2, lt.RK3W7])
    def test_in_place(self, oracle, therm_odd, integ):
        ext, U = therm_odd
        A = gpu(ext, U)
        lt.GradientFlowKernel(A, A, integ, None, 0.01)(4)
        assert rel_err(A.download(), oracle.flow(ext, U, 0.01, 4, integ.ID)) < TOL

    def test_names(self):
        A = lt.GaugeField((4, 4, 4, 4))
        assert lt.GradientFlowKernel(A, A, lt.RK3W7).ReturnIntegratorName() == "RK3W7"
        with pytest.raises(ValueError):
            lt.GradientFlowKernel(A, A, object)


class TestObservablesDriver:
    def test_levels(self, oracle, therm_odd):
        """Observables(): level 0 on the field, then one level per smear_skip Euler steps."""
        ext, U = therm_odd
        G = gpu(ext, U)
        levels = lt.Observables(G, 6.0, 3, 2, 0.02)
        assert len(levels) == 4
        assert np.array_equal(G.download(), U)
        for k, lev in enumerate(levels):
            F = U if k == 0 else oracle.flow(ext, U, 0.02, 2 * k, 0)
            want = oracle.measure(ext, F, 6.0)
            assert lev["TopChargePlaq"] == pytest.approx(want["Q_plaq"], rel=1e-10, abs=1e-12)
            assert lev["Wilson_loop(L=4)"] == pytest.approx(want["W4"], rel=1e-10)
            np.testing.assert_allclose(lev["E_clov_timeslice"], want["e_t"], rtol=1e-10)
        # flow lowers the action monotonically
        acts = [lev["Wilson_Action"] for lev in levels]
        assert all(a > b for a, b in zip(acts, acts[1:]))
