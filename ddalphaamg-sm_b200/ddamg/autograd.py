"""torch.autograd view of the adjoint gradient.

L(theta) = Re(eta^dagger D(theta)^-1 b), D the Wilson-Dirac operator on U_mu(x) = exp(i theta_mu(x))
(src/dirac_operator.cpp:24-54).  The forward pass loads the links, runs the adaptive setup and
computes L together with dL/dtheta through ddamg_gradient (adjoint solve by gamma_5-hermiticity
plus the link-derivative kernel); backward scales that gradient by the incoming grad.  It exists
so that the gradient can be checked with torch's own machinery (finite differences, gradcheck
style comparisons); the solves themselves run in the CUDA library.
"""
import numpy as np
import torch


class SolveObservable(torch.autograd.Function):
    """apply(theta, solver, eta, b, seed) -> L.

    theta: float64 tensor of shape (Nx*Nt*2,) laid out [site][mu], site = x*Nt + t;
    solver: a ddamg.Solver of the same lattice; eta, b: complex128 numpy arrays of the fine size;
    seed: the setup seed (the hierarchy is rebuilt for every theta)."""

    @staticmethod
    def forward(ctx, theta, solver, eta, b, seed):
        th = theta.detach().cpu().numpy().astype(np.float64)
        solver.load_gauge(np.exp(1j * th))
        solver.setUpPhase(seed=seed)
        g, infos = solver.gradient(eta, b)
        x, _ = solver.solve(b)
        ctx.save_for_backward(torch.from_numpy(g).to(theta.device))
        ctx.infos = infos
        return theta.new_tensor(float(np.real(np.vdot(eta, x))))

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None, None


def observable(theta, solver, eta, b, seed=0):
    return SolveObservable.apply(theta, solver, eta, b, seed)
