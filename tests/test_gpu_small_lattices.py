"""Edge cases of the geometry: the smallest lattices the container accepts (every extent 2,
where the forward and backward neighbours coincide), mixed extents with a 2, and lattices
whose extents make the multiply-shift coordinate divisions and the rectangle staple's
two-step shifts wrap.  Every kernel family against the C oracle at the FP64 tolerance.
"""
import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import IWASAKI, haar_links_numpy, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
EXTS = [(2, 2, 2, 2), (2, 4, 2, 6), (6, 2, 4, 2), (4, 4, 2, 12)]


def gpu(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


@pytest.fixture(scope="module", params=EXTS, ids=lambda e: "x".join(map(str, e)))
def lattice(request, oracle):
    ext = request.param
    return ext, oracle.heatbath(ext, haar_links_numpy(ext, sum(ext)), 5.8, 2, 7, 0)


def test_observables(oracle, lattice):
    ext, U = lattice
    G = gpu(ext, U)
    assert lt.PlaquetteSum(G) == pytest.approx(oracle.plaquette_sum(ext, U), rel=TOL)
    assert lt.TopChargeClover(G) == pytest.approx(oracle.topcharge(ext, U), rel=1e-10, abs=1e-13)
    assert lt.EnergyDensityClover(G) == pytest.approx(oracle.energy(ext, U), rel=TOL)
    m, want = lt.Measure(G, 6.0), oracle.measure(ext, U, 6.0)
    assert m["Wilson_loop(L=2)"] == pytest.approx(want["W2"], rel=TOL)
    assert m["Polyakov_loop"] == pytest.approx(want["P"], rel=TOL, abs=1e-14)
    np.testing.assert_allclose(m["TopChargeClov_timeslice"], want["q_t"], rtol=1e-10, atol=1e-13)


def test_staples_and_sweeps(oracle, lattice):
    ext, U = lattice
    G = gpu(ext, U)
    assert rel_err(lt.Staples(G), oracle.staples(ext, U)) < TOL
    lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 2)
    assert rel_err(G.download(), oracle.overrelax(ext, U, 2)) < 1e-11
    H = gpu(ext, U)
    hb = lt.HeatbathKernel(H, lt.WilsonAction(5.8), seed=5, counter=1)
    lt.Iterator.Checkerboard(hb, 1)
    assert rel_err(H.download(), oracle.heatbath(ext, U, 5.8, 1, 5, 1)) < 1e-11


def test_flow_stout_force(oracle, lattice):
    ext, U = lattice
    A, B = gpu(ext, U), lt.GaugeField(ext)
    lt.GradientFlowKernel(A, B, lt.RK3, None, 0.02)(3)
    assert rel_err(B.download(), oracle.flow_rk3(ext, U, 0.02, 3)) < TOL
    lt.StoutSmearingN(A, B, 2, 0.1)
    assert rel_err(B.download(), oracle.stout(ext, U, 0.1, 2)) < TOL
    assert rel_err(lt.WilsonAction(6.0).Force(A), oracle.gauge_force(ext, U, 6.0)) < TOL
    k = lt.HMCMetaDKernel(A, lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000), lt.WilsonAction(6.0), 1.0, 0.1, 2)
    F, q = k.CalculateTopologicalForce(dvdq=0.7)
    want, wq = oracle.metad_force(ext, U, 0.1, 2, 0.7)
    assert rel_err(F, want) < 1e-11
    assert q == pytest.approx(wq, rel=1e-10, abs=1e-13)


def test_two_row_fp32_staged_kernels(oracle, lattice):
    """The two-row FP32 kernels that stage their staple links through shared memory, on lattices
    whose blocks are partly empty (2^4 has 8 links per checkerboard plane): overrelaxation, the
    flow stage and stout smearing against the FP64 oracle at FP32 accuracy."""
    ext, U = lattice
    G = gpu(ext, U, "fp32_12")
    W = G.download()
    lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), 1)
    assert rel_err(G.download(), oracle.overrelax(ext, W, 1)) < 1e-5
    A, B = gpu(ext, W, "fp32_12"), lt.GaugeField(ext, "fp32_12")
    lt.GradientFlowKernel(A, B, lt.RK3, None, 0.02)(2)
    assert rel_err(B.download(), oracle.flow_rk3(ext, W, 0.02, 2)) < 1e-5
    lt.StoutSmearingN(A, B, 1, 0.1)
    assert rel_err(B.download(), oracle.stout(ext, W, 0.1, 1)) < 1e-5


def test_rectangle_staple(oracle, lattice):
    """x + 2 nu wraps onto x itself when the extent along nu is 2."""
    ext, U = lattice
    G = gpu(ext, U)
    S = lt.IwasakiAction(6.0).Staple(G)
    assert rel_err(S, oracle.action_staples(ext, U, IWASAKI)) < TOL


def test_parity_update(oracle, lattice):
    ext, U = lattice
    G = gpu(ext, U)
    lt.ParityUpdate(G)
    assert np.array_equal(G.download(), oracle.parity_update(ext, U))


@pytest.mark.parametrize("ext", [(4, 4, 4, 4), (8, 4, 12, 4)])
def test_checkerboard4_smallest(oracle, ext):
    U = oracle.heatbath(ext, haar_links_numpy(ext, 3), 6.0, 2, 1, 0)
    G = gpu(ext, U)
    lt.Iterator.Checkerboard4(lt.OverrelaxationSubgroupKernel(G, lt.IwasakiAction(6.0)), 1)
    assert rel_err(G.download(), oracle.overrelax4(ext, U, 1, IWASAKI)) < 1e-11
