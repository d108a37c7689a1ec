"""GPU parity of the rectangular gauge actions (GaugeAction::Rectangular<2>,
actions/gauge/rectangular_action.hpp:23-276: Luescher-Weisz, Iwasaki, DBW2) and of the sweeps
over Iterator::Checkerboard4 (iterators/iterators.hpp:141-166), with any action.

FP64 links: staples and flows within 1e-12 of the reference fixture, two overrelaxation
sweeps within 1e-10 (48 sub-sweeps of reflections amplify rounding), gauge MD within 1e-10
(H 1e-11).  The Checkerboard4 heatbath draws the oracle's Philox streams, so it is compared
with the oracle's own Checkerboard4 heatbath at 1e-11.
"""
import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import DBW2, IWASAKI, LUESCHER_WEISZ, haar_links_numpy, rel_err

pytestmark = pytest.mark.gpu

RECT = (("lw", LUESCHER_WEISZ), ("iwasaki", IWASAKI), ("dbw2", DBW2))
BY_ID = {i.ID: i for i in vars(lt.Integrators.HMC).values()}


def gpu(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


def action(act, beta=6.0):
    return lt.RectangularAction(beta, act[1], act[2])


class TestRectangularActions:
    @pytest.mark.parametrize("name,act", RECT)
    def test_staples(self, golden_rect, name, act):
        g = golden_rect
        G = gpu(tuple(g["ext"]), g["U"])
        S = action(act).Staple(G).reshape(-1, 18)
        assert rel_err(S[g["links"]], g[name + "_staple"]) < 1e-12

    @pytest.mark.parametrize("name", ["lw", "iwasaki", "dbw2", "wilson"])
    def test_overrelaxation_checkerboard4(self, golden_rect, name):
        g = golden_rect
        G = gpu(tuple(g["ext"]), g["U"])
        act = None if name == "wilson" else action(tuple(g[name + "_act"]))
        lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(G, act), 2)
        assert rel_err(G.download().reshape(-1, 18)[g["links"]], g[name + "_or4"]) < 1e-10

    @pytest.mark.parametrize("name,act", RECT)
    def test_md(self, golden_rect, name, act):
        g = golden_rect
        G = gpu(tuple(g["ext"]), g["U"])
        k = lt.HMCKernel(G, action(act), 0.5, integrator=BY_ID[int(g[name + "_md_integ"])])
        k.SetMomenta(g["P"])
        ho, hn = k.Integrate(3)
        assert ho == pytest.approx(g[name + "_md_h"][0], rel=1e-11)
        assert hn == pytest.approx(g[name + "_md_h"][1], rel=1e-11)
        assert rel_err(G.download().reshape(-1, 18)[g["links"]], g[name + "_md_U"]) < 1e-10
        assert rel_err(k.GetMomenta().reshape(-1, 18)[g["links"]], g[name + "_md_P"]) < 1e-10

    @pytest.mark.parametrize("name,act", RECT)
    def test_flow(self, golden_rect, name, act):
        g = golden_rect
        ext = tuple(g["ext"])
        A, B = gpu(ext, g["U"]), lt.GaugeField(ext)
        lt.GradientFlowKernel(A, B, lt.RK3, action(act), 0.02)(10)
        assert rel_err(B.download().reshape(-1, 18)[g["links"]], g[name + "_flow"]) < 1e-12

    @pytest.mark.parametrize("act", [None, LUESCHER_WEISZ, IWASAKI])
    def test_heatbath_checkerboard4_same_stream(self, oracle, act):
        ext = (8, 8, 4, 8)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 14), 6.0, 2, 3, 0)
        G = gpu(ext, U)
        hb = lt.HeatbathKernel(G, action(act) if act else lt.WilsonAction(6.0), seed=91, counter=2)
        lt.Iterator.Checkerboard4(hb, 2)
        assert hb.counter.value == 4
        assert rel_err(G.download(), oracle.heatbath4(ext, U, 6.0, 2, 91, 2, act)) < 1e-11

    def test_flow_methods_and_hmc_reversibility(self, oracle):
        ext = (8, 8, 8, 8)
        U = oracle.heatbath(ext, lt.haar_links(ext, 3), 6.0, 3, 1, 0)
        G = gpu(ext, U)
        k = lt.HMCKernel(G, lt.IwasakiAction(2.6), 1.0, integrator=lt.OMF_4)
        ho, hn = k.ReversibilityTest(8, counter=3)
        assert abs(hn - ho) < 1e-9 * abs(ho)
        assert rel_err(G.download(), U) < 1e-9
        # flow to t0 with the Luescher-Weisz action (the Symanzik flow) runs the same stages
        F = lt.GaugeField(ext)
        t0, _ = lt.GradientFlowKernel(G, F, lt.RK3, lt.LuescherWeiszAction(6.0), 0.02).FlowToT0(0.05)
        assert 0.0 < t0 < 5.0

    @pytest.mark.parametrize("make", [lt.LuescherWeiszAction, lt.IwasakiAction, lt.DBW2Action])
    def test_overrelaxation_conserves_its_action(self, golden_rect, make):
        g = golden_rect
        G = gpu(tuple(g["ext"]), g["U"])
        act = make(6.0)
        s0 = act.Action(G)
        lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(G, act), 5)
        assert act.Action(G) == pytest.approx(s0, rel=1e-12)
        assert lt.WilsonAction(6.0).Action(G) != pytest.approx(lt.WilsonAction(6.0).Action(gpu(tuple(g["ext"]), g["U"])),
                                                              rel=1e-9)

    def test_rules(self, oracle):
        ext = (8, 8, 8, 8)
        G = gpu(ext, lt.haar_links(ext, 2))
        with pytest.raises(lt.LettuceError):   # rectangles need Checkerboard4
            lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G, lt.DBW2Action(6.0)), 1)
        H = gpu((8, 8, 6, 8), haar_links_numpy((8, 8, 6, 8), 2))
        with pytest.raises(lt.LettuceError):   # Checkerboard4 needs extents divisible by 4
            lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(H), 1)
        # the Wilson action's Checkerboard4 visits the links in another order than Checkerboard
        A, B = gpu(ext, lt.haar_links(ext, 2)), gpu(ext, lt.haar_links(ext, 2))
        lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(A), 1)
        lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(B), 1)
        assert rel_err(A.download(), B.download()) > 1e-6
        assert lt.WilsonAction(6.0).Action(A) == pytest.approx(lt.WilsonAction(6.0).Action(B), rel=1e-12)

    @pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
    def test_fp32_storage(self, oracle, golden_rect, prec):
        g = golden_rect
        ext = tuple(g["ext"])
        G = gpu(ext, g["U"], prec)
        W = G.download()
        lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(G, lt.IwasakiAction(6.0)), 1)
        assert rel_err(G.download(), oracle.overrelax4(ext, W, 1, IWASAKI)) < 5e-5
        S = lt.LuescherWeiszAction(6.0).Staple(gpu(ext, W, prec))
        assert rel_err(S, oracle.action_staples(ext, W, LUESCHER_WEISZ)) < 1e-6

    @pytest.mark.parametrize("prec", ["fp32", "fp32_12"])
    def test_fp32_storage_wilson_checkerboard4(self, oracle, golden_rect, prec):
        """Checkerboard4 with the Wilson action on FP32 links (the two-row storage runs the
        staged-staple kernels): overrelaxation against the oracle; the heatbath of both FP32
        storages draws the same stream, so they agree but for accept/reject flips."""
        g = golden_rect
        ext = tuple(g["ext"])
        G = gpu(ext, g["U"], prec)
        W = G.download()
        lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(G), 1)
        assert rel_err(G.download(), oracle.overrelax4(ext, W, 1)) < 5e-5
        out = []
        for p in ("fp32", prec):
            H = gpu(ext, W, p)
            lt.Iterator.Checkerboard4(lt.HeatbathKernel(H, lt.WilsonAction(6.0), seed=9, counter=1), 1)
            out.append(H.download())
        d = np.abs(out[0] - out[1]).reshape(-1, 18).max(axis=1)
        assert np.median(d) < 1e-5
        assert np.mean(d > 1e-3) < 0.01

    def test_checkerboard4_thermalises_like_checkerboard(self):
        """Both iterators sample the same Wilson-action distribution: plaquettes after 30
        rounds from one start agree within the statistical spread of 8^4."""
        ext = (8, 8, 8, 8)
        A, B = lt.GaugeField(ext, "fp32"), lt.GaugeField(ext, "fp32")
        A.SetToHaarRandom(5)
        B.SetToHaarRandom(5)
        lt.UpdateSweeps(A, 6.0, 30, 1, 2, 1)
        lt.UpdateSweeps4(B, 6.0, 30, 1, 2, 2)
        pa, pb = (lt.PlaquetteSum(X) / (18 * 8 ** 4) for X in (A, B))
        assert pa == pytest.approx(pb, abs=0.01)
        assert 0.55 < pa < 0.65
