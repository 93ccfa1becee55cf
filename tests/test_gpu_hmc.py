"""HMC for the two-flavour Schwinger model (ddamg_hmc_trajectory, ddamg_hmc_force): the forces against
central finite differences of the action computed on the CPU (numpy for the gauge part, the oracle's
CG on D^dagger D for the fermion part), the O(eps^2) scaling of the energy violation of the leapfrog
integrator, and a short Markov chain."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")

ROWS8 = [[0, 2, 2, 2, 2, 2]]


def gauge_action(th, Nx, Nt, beta):
    t0 = th[0::2].reshape(Nx, Nt)
    t1 = th[1::2].reshape(Nx, Nt)
    P = t0 + np.roll(t1, -1, axis=1) - np.roll(t0, -1, axis=0) - t1
    return beta * np.sum(1.0 - np.cos(P))


def make(Nx, Nt, m0, th, rows):
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, 2, m0, rows))
    s.load_gauge(np.exp(1j * th))
    return s


def test_gauge_force_matches_finite_differences():
    Nx, Nt, beta = 8, 8, 2.0
    th, _ = po.metropolis(Nx, Nt, beta, 20, 5)
    s = make(Nx, Nt, 0.2, th, ROWS8)
    F = s.hmc_force(th, np.zeros(2 * Nx * Nt, dtype=np.complex128), beta)  # phi = 0: gauge force only
    h = 1e-6
    for l in range(0, 2 * Nx * Nt, 7):
        tp, tm = th.copy(), th.copy()
        tp[l] += h
        tm[l] -= h
        fd = (gauge_action(tp, Nx, Nt, beta) - gauge_action(tm, Nx, Nt, beta)) / (2 * h)
        assert abs(F[l] - fd) < 1e-6 * max(1.0, abs(fd)), (l, F[l], fd)
    s.close()


def test_fermion_force_matches_finite_differences():
    Nx, Nt, beta, m0 = 8, 8, 2.0, 0.2
    th, _ = po.metropolis(Nx, Nt, beta, 20, 6)
    phi = po.gaussian(2 * Nx * Nt, 17)
    s = make(Nx, Nt, m0, th, ROWS8)
    F = s.hmc_force(th, phi, beta, cg_tol=1e-13)

    def action(t):
        o = po.Oracle(Nx, Nt, 2, m0, ROWS8, po.links_from_theta(t))
        X, it = o.cg_normal(phi, max_iter=20000, tol=1e-14)
        assert it > 0
        return gauge_action(t, Nx, Nt, beta) + float(np.real(np.vdot(phi, X)))

    rng = np.random.default_rng(2)
    h = 1e-5
    for l in rng.choice(2 * Nx * Nt, size=6, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[l] += h
        tm[l] -= h
        fd = (action(tp) - action(tm)) / (2 * h)
        assert abs(F[l] - fd) < 1e-5 * max(1.0, abs(fd)), (l, F[l], fd)
    s.close()


def test_leapfrog_energy_violation_scales_as_eps_squared():
    Nx, Nt, beta, m0 = 16, 16, 2.0, 0.1
    th, _ = po.metropolis(Nx, Nt, beta, 50, 7)
    rows = [[0, 4, 4, 4, 4, 4]]
    s = make(Nx, Nt, m0, th, rows)
    dh = []
    for steps in (10, 20):
        t = th.copy()
        info = s.hmc_trajectory(t, beta, md_steps=steps, tau=0.5, seed=11)  # same momenta and eta
        dh.append(abs(info.dH))
    s.close()
    ratio = dh[0] / dh[1]
    assert 2.5 < ratio < 6.5, (dh, ratio)


def test_short_chain_then_solve():
    Nx, Nt, beta, m0 = 16, 16, 2.0, 0.1
    th, _ = po.metropolis(Nx, Nt, beta, 50, 8)
    rows = [[0, 4, 4, 4, 4, 4]]
    s = make(Nx, Nt, m0, th, rows)
    acc = 0
    for k in range(5):
        info = s.hmc_trajectory(th, beta, md_steps=20, tau=1.0, seed=100 + k)
        acc += info.accepted
        assert info.cg_iterations > 0 and np.isfinite(info.dH)
        assert 0.3 < info.plaquette < 0.95
    assert acc >= 3
    assert np.all(th >= -np.pi) and np.all(th < np.pi)
    # the handle now holds the chain's field: a fresh setup and multigrid solve on it converge
    s.setUpPhase(seed=3)
    b = po.gaussian(2 * Nx * Nt, 9)
    x, info = s.solve(b)
    assert info[0].converged
    o = po.Oracle(Nx, Nt, 2, m0, rows, po.links_from_theta(th))
    assert np.linalg.norm(o.dirac(x) - b) / np.linalg.norm(b) < 1e-9
    s.close()
