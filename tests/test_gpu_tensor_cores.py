"""The tensor-core block operator of batched FP32 coarse-level SAP sweeps (tcgen05, TF32 inputs,
FP32 accumulation) against the CUDA-core FP32 sweep and the oracle's FP64 SAP.

Tolerances (relative 2-norm):
  * CUDA-core FP32 SAP vs the FP64 oracle: 1e-4 (FP32 rounding through a GMRES(5)x5 block solve);
  * tensor-core SAP vs the FP64 oracle: 2e-2 -- TF32 keeps 10 mantissa bits (relative rounding
    about 5e-4 per operand) and the block solves stop at 1e-3;
  * full solves: the FP64 outer FGMRES reaches 1e-10 either way; iteration counts may differ by
    one from the CUDA-core path, the solution agrees with the FP64 solve to 1e-8.
"""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(z, R, tensor_cores, precision=None):
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    p = ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"],
                             precision=ddamg.PREC_MIXED if precision is None else precision, max_rhs=R,
                             fgmres_restart_length=int(z["fgmres_m"]), tensor_cores=tensor_cores)
    s = ddamg.Solver(p)
    s.load_gauge(U)
    rnd = po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1)
    s.setUpPhase(vectors=rnd)
    return s, U, rnd


@pytest.mark.parametrize("name", ["ops_16x32_l3", "ops_32x16_l3"])
def test_sap_batched_tensor_cores_vs_oracle(golden, name):
    z = golden(name)
    R = 8
    s_tc, U, rnd = make(z, R, 1)
    s_cc, _, _ = make(z, R, 0)
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"]), z["rows"], U)
    o.setup(rnd)
    n = o.size(1)
    vs = np.concatenate([po.gaussian(n, 500 + r) for r in range(R)])
    x_tc = s_tc.SAP_batched(1, vs, R, nu=1)
    x_cc = s_cc.SAP_batched(1, vs, R, nu=1)
    assert not np.array_equal(x_tc, x_cc)  # the tensor-core path ran
    e_tc, e_cc = [], []
    for r in range(R):
        xo, _ = o.sap(1, vs[r * n:(r + 1) * n], nu=1)
        e_cc.append(rel(x_cc[r * n:(r + 1) * n], xo))
        e_tc.append(rel(x_tc[r * n:(r + 1) * n], xo))
    print(name, "max rel err vs FP64 oracle: CUDA cores", max(e_cc), "tensor cores", max(e_tc))
    assert max(e_cc) < 1e-4
    assert max(e_tc) < 2e-2
    s_tc.close()
    s_cc.close()


def synthetic(N=128, nv=16, seed=7):
    """8x8-site aggregates and 4x4-site SAP blocks at level 0; level 1 (N/8)^2 sites with dof 2 nv,
    4x4-site aggregates and SAP blocks."""
    th, _ = ddamg.gauge_metropolis(N, N, 3.0, 200, seed)
    rows = [[0, N // 8, N // 8, nv, N // 4, N // 4], [1, N // 32, N // 32, nv, N // 32, N // 32]]
    return np.exp(1j * th), rows


@pytest.mark.parametrize("R", [16, 64])
def test_sap_batched_tensor_cores_dof32(R):
    """The production shape: dof 32 (Nv = 16), 4x4-site SAP blocks at level 1."""
    N = 128
    U, rows = synthetic(N, 16)
    out = []
    for tcf in (1, 0):
        p = ddamg.default_params(N, N, 3, -0.10, rows, precision=ddamg.PREC_MIXED, max_rhs=R, tensor_cores=tcf)
        s = ddamg.Solver(p)
        s.load_gauge(U)
        s.setUpPhase(seed=3)
        n = s.size(1)
        vs = ddamg.gaussian_field(n * R, 91)
        out.append(s.SAP_batched(1, vs, R, nu=2))
        s.close()
    errs = [rel(out[0][r * n:(r + 1) * n], out[1][r * n:(r + 1) * n]) for r in range(R)]
    print("R", R, "tensor vs CUDA cores, max rel diff", max(errs))
    assert 0 < max(errs) < 2e-2


@pytest.mark.parametrize("cycle", [ddamg.CYCLE_V, ddamg.CYCLE_K])
def test_solve_batched_tensor_cores(cycle):
    """Batched mixed solve with the tensor-core smoother: every rhs converges to 1e-10 and matches
    the FP64 solve; iterations within one of the CUDA-core mixed solve."""
    N, R = 128, 16
    U, rows = synthetic(N, 16)
    n = 2 * N * N
    b = ddamg.gaussian_field(n * R, 17)
    res = {}
    for key, prec, tcf in (("fp64", ddamg.PREC_DOUBLE, 0), ("cc", ddamg.PREC_MIXED, 0), ("tc", ddamg.PREC_MIXED, 1)):
        p = ddamg.default_params(N, N, 3, -0.10, rows, precision=prec, max_rhs=R, tensor_cores=tcf, cycle=cycle,
                                 fgmres_restart_length=30)
        s = ddamg.Solver(p)
        s.load_gauge(U)
        s.setUpPhase(seed=3)
        res[key] = s.solve(b, nrhs=R)
        s.close()
    x64, _ = res["fp64"]
    xtc, itc = res["tc"]
    _, icc = res["cc"]
    for r in range(R):
        assert itc[r].converged == 1 and itc[r].rel_residual < 1e-10
        assert abs(itc[r].iterations - icc[r].iterations) <= 1, (r, itc[r].iterations, icc[r].iterations)
        assert rel(xtc[r * n:(r + 1) * n], x64[r * n:(r + 1) * n]) < 1e-8


@pytest.mark.parametrize("R,precision", [(1, ddamg.PREC_DOUBLE), (3, ddamg.PREC_MIXED), (16, ddamg.PREC_MIXED)])
def test_cycle_graph_replay_matches_direct(R, precision):
    """The V-cycle captured into a CUDA graph (from the second preconditioner application of a
    batch width on) gives the same solves as launching the kernels one by one: bit-identical on
    the CUDA-core paths in the first solve (host-driven FGMRES around the replayed cycle); the second
    solve runs as one device-driven graph whose Givens arithmetic is compiled for the device, so it
    agrees to 1e-12 with the same iterations.  With the tensor-core smoother (R >= 8, mixed) each
    handle's autotuner may pick another tile shape (another TF32 accumulation order), so there the
    iterations agree and the solutions to 1e-9."""
    N = 128
    U, rows = synthetic(N, 16)
    n = 2 * N * N
    b = ddamg.gaussian_field(n * R, 23)
    out = []
    for graphs in (1, 0):
        p = ddamg.default_params(N, N, 3, -0.10, rows, precision=precision, max_rhs=R, cuda_graphs=graphs,
                                 fgmres_restart_length=30)
        s = ddamg.Solver(p)
        s.load_gauge(U)
        s.setUpPhase(seed=3)
        res = [s.solve(b, nrhs=R) for _ in range(2)]  # the second solve replays the captured cycle
        report = s.autotune_report()
        s.close()
        out.append((res, report))
    (g_res, g_rep), (d_res, _) = out
    assert f"cycle graph rhs {R}:" in g_rep, g_rep
    assert f"solve graph rhs {R}:" in g_rep, g_rep
    for k, ((xg, ig), (xd, idd)) in enumerate(zip(g_res, d_res)):
        assert [i.iterations for i in ig] == [i.iterations for i in idd]
        if R >= 8 and precision == ddamg.PREC_MIXED:
            assert np.linalg.norm(xg - xd) / np.linalg.norm(xd) < 1e-9
        elif k == 0:
            assert np.array_equal(xg, xd)
        else:
            assert np.linalg.norm(xg - xd) / np.linalg.norm(xd) < 1e-12
