"""Adjoint gradient on a 128x128 lattice (beta=2, m0=-0.15, 2 levels, Nv=10): dL/dtheta_mu(x) for
L = Re(eta^dagger D^-1 b) through the torch.autograd wrapper, against

  * the oracle's FP64 gradient (both solves at 1e-13 on the CPU, then the link derivative):
    relative 2-norm 1e-8;
  * central finite differences of L with step 1e-5 at 64 random links, each L from an FP64 GPU
    solve at relative residual 1e-13: |fd - g| <= 1e-6 * max(1, |fd|).

in FP64 and in mixed precision (FP32 smoother and intermediate levels, FP64 outer solve).
"""
import numpy as np
import pytest
import torch

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")
from ddamg.autograd import observable  # noqa: E402

N, BETA, M0, SWEEPS = 128, 2.0, -0.15, 500
ROWS = [[0, 32, 32, 10, 32, 32]]


@pytest.fixture(scope="module")
def field():
    th, acc = ddamg.gauge_metropolis(N, N, BETA, SWEEPS, 2024)
    n = 2 * N * N
    eta, b = po.gaussian(n, 71), po.gaussian(n, 72)
    # FP64 oracle gradient
    o = po.Oracle(N, N, 2, M0, ROWS, po.links_from_theta(th))
    o.setup(po.uniform(o.setup_random_count(), 9))
    psi, _ = o.solve(b, m=30, tol=1e-13)
    s3 = np.tile([1.0, -1.0], n // 2)
    lam_, _ = o.solve(s3 * eta, m=30, tol=1e-13)
    g_ref = o.link_gradient(psi, s3 * lam_)
    return th, eta, b, g_ref


def solver(precision, tol, max_rhs=2):
    p = ddamg.default_params(N, N, 2, M0, ROWS, precision=precision, max_rhs=max_rhs, fgmres_restart_length=30,
                             fgmres_tolerance=tol)
    return ddamg.Solver(p)


@pytest.mark.parametrize("precision", [ddamg.PREC_DOUBLE, ddamg.PREC_MIXED])
def test_gradient_128_autograd(field, precision):
    th, eta, b, g_ref = field
    s = solver(precision, 1e-12)
    theta = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    L = observable(theta, s, eta, b, seed=3)
    L.backward()
    g = theta.grad.numpy()
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) < 1e-8
    # finite differences of L(theta) with FP64 GPU solves
    fd_solver = solver(ddamg.PREC_DOUBLE, 1e-13, max_rhs=1)
    rng = np.random.default_rng(5)
    h = 1e-5
    for k in rng.choice(2 * N * N, size=64, replace=False):
        vals = []
        for sgn in (1.0, -1.0):
            t2 = th.copy()
            t2[k] += sgn * h
            fd_solver.load_gauge(np.exp(1j * t2))
            fd_solver.setUpPhase(seed=3)
            x, info = fd_solver.solve(b)
            assert info[0].rel_residual < 1e-13
            vals.append(np.real(np.vdot(eta, x)))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])
    fd_solver.close()
    s.close()


def test_gradient_batched_equals_sequential(field):
    """The two solves of the gradient in one lockstep batch give the same result as one by one."""
    th, eta, b, _ = field
    U = np.exp(1j * th)
    out = []
    for R in (1, 2):
        s = solver(ddamg.PREC_DOUBLE, 1e-10, max_rhs=R)
        s.load_gauge(U)
        s.setUpPhase(seed=3)
        g, infos = s.gradient(eta, b)
        out.append((g, [i.iterations for i in infos]))
        s.close()
    assert out[0][1] == out[1][1]
    assert np.linalg.norm(out[0][0] - out[1][0]) / np.linalg.norm(out[0][0]) < 1e-12
