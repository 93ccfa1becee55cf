"""GPU parity: the CUDA library (through the C ABI) against the CPU oracle on the golden
cases.  The oracle itself is pinned to the reference in test_oracle_golden.py.

Tolerances (relative 2-norm of the difference):
  * single operator applications (D_W, D_W^dagger, level operators, P, P^dagger): 1e-13 —
    same arithmetic, different summation order;
  * setup products (test vectors, coarse links), SAP, cycles: 1e-9 — the same algorithm, with
    rounding differences amplified through 4 smoothing iterations and Krylov solves;
  * solutions: 1e-9 against the reference's FP64 solution (the gate the solver is built to), with
    the true residual below 1e-10 under the oracle's operator and the iteration count within 10 %.
"""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")

OPS = ["ops_16x32_l3", "ops_32x32_l2", "ops_32x16_l3"]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make_pair(z, precision=ddamg.PREC_DOUBLE, cycle=ddamg.CYCLE_V, max_rhs=1):
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    o = po.Oracle(Nx, Nt, L, float(z["m0"]), z["rows"], U)
    rnd = po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1)
    o.setup(rnd)
    p = ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], precision=precision, cycle=cycle,
                             max_rhs=max_rhs, fgmres_restart_length=int(z["fgmres_m"]))
    s = ddamg.Solver(p)
    s.load_gauge(U)
    assert s.setup_random_count() == int(z["rnd_count"])
    s.setUpPhase(vectors=rnd)
    return s, o


@pytest.fixture(scope="module", params=OPS)
def pair(request, golden):
    z = golden(request.param)
    s, o = make_pair(z)
    yield z, s, o
    s.close()


def test_dirac(pair):
    z, s, o = pair
    assert rel(s.D_phi(z["probe_0"]), o.dirac(z["probe_0"])) < 1e-14
    assert rel(s.D_dagger_phi(z["probe_0"]), o.dirac(z["probe_0"], True)) < 1e-14
    # against the reference's own output
    assert rel(s.D_phi(z["probe_0"]), z["ref_Dphi"]) < 1e-14


def test_dirac_batched(pair):
    z, s, o = pair
    n = z["probe_0"].size
    if s.params.max_rhs < 1:
        pytest.skip()
    # nrhs fields back to back (within the handle's batch width)
    ntest = int(z["rows"][0][3])
    k = min(3, ntest)
    vs = np.concatenate([po.gaussian(n, 900 + i) for i in range(k)])
    out = s.D_phi(vs, nrhs=k)
    for i in range(k):
        assert rel(out[i * n:(i + 1) * n], o.dirac(vs[i * n:(i + 1) * n])) < 1e-14


def test_test_vectors_and_links(pair):
    z, s, o = pair
    L = int(z["levels"])
    for l in range(L - 1):
        assert rel(s.test_vectors(l), o.get_tvec(l)) < 1e-9, l
    for l in range(1, L):
        for w in (1, 2, 3):
            assert rel(s.coarse_links(l, w), o.get_links(l, w)) < 1e-9, (l, w)


def test_level_ops_and_transfers(pair):
    z, s, o = pair
    L = int(z["levels"])
    for l in range(L):
        v = z[f"probe_{l}"]
        tol = 1e-13 if l == 0 else 1e-9
        assert rel(s.D_operator(l, v), o.level_op(l, v)) < tol, l
    for l in range(L - 1):
        assert rel(s.Pdagg_v(l, z[f"probe_{l}"]), o.restrict(l, z[f"probe_{l}"])) < 1e-9
        assert rel(s.P_vc(l, z[f"probe_{l + 1}"]), o.prolong(l, z[f"probe_{l + 1}"])) < 1e-9


def test_transfers_exact_with_injected_vectors(pair):
    """With identical test vectors P and P^dagger agree to rounding."""
    z, s, o = pair
    L = int(z["levels"])
    for l in range(L - 1):
        s.set_test_vectors(l, o.get_tvec(l))
        assert rel(s.Pdagg_v(l, z[f"probe_{l}"]), o.restrict(l, z[f"probe_{l}"])) < 1e-13
        assert rel(s.P_vc(l, z[f"probe_{l + 1}"]), o.prolong(l, z[f"probe_{l + 1}"])) < 1e-13


def test_sap(pair):
    z, s, o = pair
    L = int(z["levels"])
    for l in range(L - 1):
        xg, itg = s.SAP(l, z[f"probe_{l}"], nu=3)
        xo, ito = o.sap(l, z[f"probe_{l}"], nu=3)
        assert itg == ito
        assert rel(xg, xo) < 1e-9, l


def test_sap_converges_standalone(golden):
    """SAP as a solver reaches tol and returns early (testSAP, src/amg.cpp:300-349)."""
    z = golden("ops_16x32_l3")
    s, o = make_pair(z)
    b = z["probe_0"]
    x, it = s.SAP(0, b, nu=500, tol=1e-12)
    assert it < 500
    assert rel(s.D_phi(x), b) < 1e-12
    xo, ito = o.sap(0, b, nu=500, tol=1e-12)
    assert abs(it - ito) <= 1
    s.close()


def test_coarse_gmres(pair):
    z, s, o = pair
    L = int(z["levels"])
    b = z[f"probe_{L - 1}"]
    xg, itg = s.coarse_gmres(b)
    xo, ito = o.coarse_gmres(b)
    assert itg == ito
    assert rel(xg, xo) < 1e-9


def test_cycles(golden):
    for name in OPS:
        z = golden(name)
        s, o = make_pair(z)
        ev = rel(s.v_cycle(z["probe_0"]), o.vcycle(z["probe_0"]))
        s.close()
        s, o = make_pair(z, cycle=ddamg.CYCLE_K)
        ek = rel(s.k_cycle(z["probe_0"]), o.kcycle(z["probe_0"]))
        print(f"{name}: V-cycle rel diff {ev:.2e}, K-cycle {ek:.2e}")
        assert ev < 1e-9 and ek < 1e-9, name
        s.close()


@pytest.mark.parametrize("name", ["ops_16x32_l3", "ops_32x32_l2", "solve_64x64_l2"])
@pytest.mark.parametrize("cycle,tag", [(ddamg.CYCLE_V, "V"), (ddamg.CYCLE_K, "K")])
def test_solve_fp64(golden, name, cycle, tag):
    z = golden(name)
    s, o = make_pair(z, cycle=cycle)
    x, info = s.solve(z["rhs"])
    ref_it = int(z[f"ref_iters_{tag}"])
    assert info[0].converged == 1
    assert info[0].rel_residual < 1e-10
    # true residual with the oracle's operator
    assert rel(o.dirac(x), z["rhs"]) < 1e-10
    # iteration count within +-10% of the reference's (at least +-1)
    assert abs(info[0].iterations - ref_it) <= max(1, int(0.1 * ref_it)), (info[0].iterations, ref_it)
    # the reference's FP64 solution to 1e-9
    e = rel(x, z[f"ref_x_{tag}"])
    print(f"{name} {tag}: iterations {info[0].iterations} (reference {ref_it}), rel diff to the reference {e:.2e}")
    assert e < 1e-9
    s.close()


@pytest.mark.parametrize("name", ["ops_16x32_l3", "solve_64x64_l2"])
def test_solve_mixed(golden, name):
    z = golden(name)
    s, o = make_pair(z, precision=ddamg.PREC_MIXED)
    x, info = s.solve(z["rhs"])
    assert info[0].converged == 1 and info[0].rel_residual < 1e-10
    assert rel(o.dirac(x), z["rhs"]) < 1e-10
    e = rel(x, z["ref_x_V"])
    print(f"{name} mixed: rel diff to the reference's FP64 solution {e:.2e}")
    assert e < 1e-9
    s.close()


def test_link_derivative(golden):
    z = golden("ops_16x32_l3")
    s, o = make_pair(z)
    n = z["probe_0"].size
    psi, lam = po.gaussian(n, 31), po.gaussian(n, 32)
    assert rel(s.link_derivative(psi, lam), o.link_gradient(psi, lam)) < 1e-13
    s.close()


def test_gradient_matches_oracle_and_fd(golden):
    """dL/dtheta for L = Re(eta^+ D^-1 b): adjoint solve + link derivative vs the oracle's FP64
    gradient (1e-8) and central finite differences of oracle solves (h = 1e-5, rel 1e-6)."""
    z = golden("ops_16x32_l3")
    s, o = make_pair(z)
    Nx, Nt = int(z["Nx"]), int(z["Nt"])
    n = z["probe_0"].size
    eta, b = po.gaussian(n, 41), po.gaussian(n, 42)
    g, infos = s.gradient(eta, b)
    psi, _ = o.solve(b, m=20, tol=1e-13)
    s3 = np.tile([1.0, -1.0], n // 2)
    lam_, _ = o.solve(s3 * eta, m=20, tol=1e-13)
    lam = s3 * lam_
    g_ref = o.link_gradient(psi, lam)
    assert rel(g, g_ref) < 1e-8
    rng = np.random.default_rng(0)
    th = z["theta"].copy()
    rows, m0, L = z["rows"], float(z["m0"]), int(z["levels"])
    rnd = po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1)
    for li in rng.choice(2 * Nx * Nt, size=8, replace=False):
        vals = []
        for sgn in (+1, -1):
            t2 = th.copy()
            t2[li] += sgn * 1e-5
            oo = po.Oracle(Nx, Nt, L, m0, rows, po.links_from_theta(t2))
            oo.setup(rnd)
            x, _ = oo.solve(b, m=20, tol=1e-14)
            vals.append(np.real(np.vdot(eta, x)))
        fd = (vals[0] - vals[1]) / 2e-5
        assert abs(fd - g[li]) <= 1e-6 * max(1.0, abs(fd)) + 1e-6, (li, fd, g[li])
    s.close()


def test_metropolis_matches_oracle():
    th_g, acc_g = ddamg.gauge_metropolis(16, 32, 2.0, 3, 99)
    th_o, acc_o = po.metropolis(16, 32, 2.0, 3, 99)
    # same chain: identical proposals and acceptance draws; cos/exp may differ by an ulp
    assert np.max(np.abs(th_g - th_o)) < 1e-12
    assert abs(acc_g - acc_o) < 1e-12


@pytest.mark.parametrize("cycle", [ddamg.CYCLE_V, ddamg.CYCLE_K])
@pytest.mark.parametrize("precision", [ddamg.PREC_DOUBLE, ddamg.PREC_MIXED])
def test_solve_batched_matches_single(golden, cycle, precision):
    """R right-hand sides in one lockstep solve follow exactly the single-RHS algorithm each."""
    z = golden("ops_16x32_l3")
    R = 3
    s1, o = make_pair(z, precision=precision, cycle=cycle)
    sb, _ = make_pair(z, precision=precision, cycle=cycle, max_rhs=R)
    n = z["rhs"].size
    bs = [po.gaussian(n, 300 + r) for r in range(R)]
    xb, infob = sb.solve(np.concatenate(bs), nrhs=R)
    for r in range(R):
        x1, info1 = s1.solve(bs[r])
        assert infob[r].iterations == info1[0].iterations
        assert infob[r].converged == 1
        assert rel(xb[r * n:(r + 1) * n], x1) < 1e-12
        assert rel(o.dirac(xb[r * n:(r + 1) * n]), bs[r]) < 1e-10
    s1.close()
    sb.close()


def test_solve_batched_with_zero_rhs(golden):
    z = golden("ops_16x32_l3")
    s, o = make_pair(z, max_rhs=2)
    n = z["rhs"].size
    b = np.concatenate([np.zeros(n, dtype=np.complex128), z["rhs"]])
    x, info = s.solve(b, nrhs=2)
    assert np.all(x[:n] == 0) and info[0].iterations == 0
    assert info[1].converged == 1 and rel(o.dirac(x[n:]), z["rhs"]) < 1e-10
    s.close()


def test_solve_bench_workload_matches_reference(golden):
    """The bench workload (256x256 FP64, 3 levels, FGMRES(30) V-cycle): with the reference's setup stream
    injected, the GPU solve takes the reference's iteration count and lands within 1e-9 of its solution."""
    z = golden("solve_256x256_l3")
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    theta, _ = po.metropolis(Nx, Nt, float(z["beta"]), int(z["sweeps"]), int(z["seed"]))
    U = po.links_from_theta(theta)
    b = po.gaussian(2 * Nx * Nt, int(z["rhs_seed"]))
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], fgmres_restart_length=int(z["fgmres_m"])))
    s.load_gauge(U)
    s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    x, info = s.solve(b)
    s.close()
    ref_it = int(z["ref_iters_V"])
    res = rel(po.dirac(Nx, Nt, float(z["m0"]), U, x), b)
    e = rel(x, z["ref_x_V"])
    print(f"256x256: iterations {info[0].iterations} (reference {ref_it}), residual {res:.2e}, rel diff {e:.2e}")
    assert info[0].converged == 1 and res < 1e-10
    assert abs(info[0].iterations - ref_it) <= max(1, ref_it // 10)
    assert e < 1e-9


@pytest.mark.parametrize("cycle", [ddamg.CYCLE_V, ddamg.CYCLE_K])
def test_solve_batched_tensor_cores_vs_oracle(golden, cycle):
    """The batched mixed solve whose coarse SAP runs on the tensor cores (8 right-hand sides, TF32 block
    operator): every solution within 1e-9 of the oracle's FP64 solve of the same system (solved to 1e-13),
    true residual below 1e-10 under the oracle's operator."""
    z = golden("ops_16x32_l3")
    R = 8
    s, o = make_pair(z, precision=ddamg.PREC_MIXED, cycle=cycle, max_rhs=R)
    n = z["rhs"].size
    bs = [po.gaussian(n, 600 + r) for r in range(R)]
    x, infos = s.solve(np.concatenate(bs), nrhs=R)
    assert "level 1 rhs 8:" in s.autotune_report()  # the tensor-core sweep ran (the autotuner timed it)
    s.close()
    worst = 0.0
    for r in range(R):
        xr = x[r * n:(r + 1) * n]
        xo, _ = o.solve(bs[r], cycle=int(cycle), m=20, tol=1e-13)
        assert infos[r].converged == 1
        assert rel(o.dirac(xr), bs[r]) < 1e-10
        worst = max(worst, rel(xr, xo))
    print(f"tensor-core batched mixed solve, cycle {int(cycle)}: max rel diff to the FP64 oracle {worst:.2e}")
    assert worst < 1e-9


def test_sap_level0_small_blocks(golden):
    """Level-0 SAP with 4 x 4-site blocks (configs[0]'s layout; the kernel that runs two block solves per
    warp) against the oracle, and a 3-vector batch (an odd number of block tasks, so one half-warp has no
    task) equal bit for bit to three single-vector sweeps."""
    z = golden("solve_64x64_l2")
    s, o = make_pair(z)
    v = z["probe_0"]
    xg, itg = s.SAP(0, v, nu=3)
    xo, ito = o.sap(0, v, nu=3)
    assert itg == ito
    assert rel(xg, xo) < 1e-9
    n = v.size
    vs = [po.gaussian(n, 700 + r) for r in range(3)]
    xb = s.SAP_batched(0, np.concatenate(vs), 3, nu=2, tol=0)
    for r in range(3):
        x1 = s.SAP_batched(0, vs[r], 1, nu=2, tol=0)
        assert np.array_equal(xb[r * n:(r + 1) * n], x1), r
    s.close()
