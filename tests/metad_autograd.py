"""The metadynamics force of the C ABI mirrored as a torch.autograd.Function (test harness
only; the library does not depend on torch).

SmearedCharge.apply(x, kernel) is the stout-smeared clover charge Q(U') of the kernel's
field after the left multiplication U'(l) = exp(i x[l, a] lambda_a / 2) U(l) of every link l
(x: float64 tensor of shape (4V, 8), Gell-Mann generators lambda_a).  Its backward is the
hand-written adjoint lt_metad_force taken at U', contracted with the generators:
dQ/dx[l, a] = Re tr(i lambda_a F(l)), the pattern of the reference's numerical check
(LettuceGauge/numerical_derivative.hpp:71-249).  The backward is exact at x = 0, where the
derivative of exp(i x lambda / 2) is i lambda / 2; that is where the tests evaluate it.
"""
import numpy as np
import torch

GELL_MANN = np.zeros((8, 3, 3), dtype=np.complex128)
GELL_MANN[0][0, 1] = GELL_MANN[0][1, 0] = 1
GELL_MANN[1][0, 1], GELL_MANN[1][1, 0] = -1j, 1j
GELL_MANN[2][0, 0], GELL_MANN[2][1, 1] = 1, -1
GELL_MANN[3][0, 2] = GELL_MANN[3][2, 0] = 1
GELL_MANN[4][0, 2], GELL_MANN[4][2, 0] = -1j, 1j
GELL_MANN[5][1, 2] = GELL_MANN[5][2, 1] = 1
GELL_MANN[6][1, 2], GELL_MANN[6][2, 1] = -1j, 1j
GELL_MANN[7] = np.diag([1, 1, -2]) / np.sqrt(3)


def exp_generator(coef):
    """exp(i sum_a coef[a] lambda_a / 2) via the eigendecomposition of the Hermitian sum."""
    h = np.tensordot(coef, GELL_MANN, axes=1) / 2
    w, v = np.linalg.eigh(h)
    return (v * np.exp(1j * w)) @ v.conj().T


def _perturb(kernel, x):
    """Apply x to the kernel's field link by link (only nonzero rows); returns the saved links."""
    saved = []
    for l in np.nonzero(np.any(x != 0.0, axis=1))[0]:
        site, mu = divmod(int(l), 4)
        u0 = kernel.U.get_link(site, mu)
        saved.append((site, mu, u0))
        kernel.U.set_link(site, mu, exp_generator(x[l]) @ u0)
    return saved


def _restore(kernel, saved):
    for site, mu, u0 in reversed(saved):
        kernel.U.set_link(site, mu, u0)


def force_components(F):
    """Re tr(i lambda_a F(l)) for a force field in the reference layout -> (4V, 8)."""
    F = (F[..., 0] + 1j * F[..., 1]).reshape(-1, 3, 3)
    return np.real(np.einsum("aij,lji->la", GELL_MANN, 1j * F))


class SmearedCharge(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, kernel):
        saved = _perturb(kernel, x.detach().cpu().numpy())
        try:
            q = kernel.MetaCharge()
        finally:
            _restore(kernel, saved)
        ctx.kernel = kernel
        ctx.save_for_backward(x)
        return x.new_tensor(q)

    @staticmethod
    def backward(ctx, grad_q):
        (x,) = ctx.saved_tensors
        kernel = ctx.kernel
        saved = _perturb(kernel, x.detach().cpu().numpy())
        try:
            F, _ = kernel.CalculateTopologicalForce(dvdq=1.0)
        finally:
            _restore(kernel, saved)
        return grad_q * x.new_tensor(force_components(F)), None
