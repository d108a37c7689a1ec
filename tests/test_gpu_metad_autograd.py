"""The adjoint metadynamics force through torch.autograd: torch.autograd.grad of the
SmearedCharge mirror (tests/metad_autograd.py) against central differences of the same
function, and torch.autograd.gradcheck on single links."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import lettuce_b200 as lt  # noqa: E402
from metad_autograd import SmearedCharge, force_components  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kernel():
    ext = (8, 8, 8, 8)
    G = lt.GaugeField(ext, "fp64")
    G.SetToHaarRandom(31)
    lt.UpdateSweeps(G, 6.0, 10, 1, 4, seed=9)
    bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
    return lt.HMCMetaDKernel(G, bias, lt.WilsonAction(6.0), 1.0, 0.12, 4)


def test_autograd_gradient_matches_central_differences(kernel):
    n = 4 * kernel.U.Volume()
    x = torch.zeros((n, 8), dtype=torch.float64, requires_grad=True)
    q = SmearedCharge.apply(x, kernel)
    assert q.item() == pytest.approx(kernel.MetaCharge(), rel=1e-14)
    (g,) = torch.autograd.grad(q, x)
    rng = np.random.default_rng(3)
    h = 1e-4
    worst = 0.0
    for l in rng.choice(n, size=12, replace=False):
        for a in range(8):
            e = torch.zeros((n, 8), dtype=torch.float64)
            e[l, a] = h
            fd = (SmearedCharge.apply(e, kernel) - SmearedCharge.apply(-e, kernel)).item() / (2 * h)
            worst = max(worst, abs(fd - g[l, a].item()))
    assert worst < 1e-6, worst
    # the force scales with dV/dQ: the gradient is the dV/dQ = 1 force
    F, _ = kernel.CalculateTopologicalForce(dvdq=-2.0)
    assert np.allclose(force_components(F), -2.0 * g.numpy(), rtol=1e-12, atol=1e-15)


def test_gradcheck_single_links(kernel):
    n = 4 * kernel.U.Volume()
    for l in (0, 123, n - 1):
        def f(y, l=l):
            x = torch.zeros((n, 8), dtype=torch.float64)
            x = x.index_put((torch.tensor([l]),), y.reshape(1, 8))
            return SmearedCharge.apply(x, kernel)
        y0 = torch.zeros(8, dtype=torch.float64, requires_grad=True)
        assert torch.autograd.gradcheck(f, (y0,), eps=1e-5, atol=1e-7, rtol=1e-4)
