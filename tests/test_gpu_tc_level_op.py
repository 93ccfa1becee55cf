"""The batched level operator D_c (Level::D_operator, src/level.cpp:394-426) on tcgen05 tensor cores:
per site and hop one M = 64, N = right-hand sides, K = 64 TF32 contraction of the packed operator tile
with the neighbour's vector tile, five hops accumulating in tensor memory, the mass term in FP32.
Against the FP32 CUDA-core kernel on the same handle (5e-3 relative: TF32 inputs keep 10 mantissa bits)
and the oracle's FP64 operator (1e-3 for the CUDA-core kernel: the mixed setup smooths the test vectors in
FP32, so the handle's coarse links differ from the oracle's at about 1e-4); and a batched mixed solve with
the tensor-core operator forced reaches the FP64 tolerance under the oracle's D_phi."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")
torch = pytest.importorskip("torch")

N, M0 = 64, -0.12
ROWS = [[0, 16, 16, 16, 16, 16], [1, 4, 4, 8, 4, 4]]  # level 1: 16 x 16 sites of dof 32 (Nv = 16), 4 x 4-site SAP blocks


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def field():
    th, _ = po.metropolis(N, N, 2.0, 20, 31)
    U = po.links_from_theta(th)
    o = po.Oracle(N, N, 3, M0, ROWS, U)
    rnd = po.uniform(o.setup_random_count(), 7)
    o.setup(rnd)
    return U, o, rnd


def handle(U, rnd, tc, R):
    s = ddamg.Solver(ddamg.default_params(N, N, 3, M0, ROWS, precision=ddamg.PREC_MIXED, max_rhs=R,
                                          tensor_cores=tc))
    s.load_gauge(U)
    s.setUpPhase(vectors=rnd)
    return s


@pytest.mark.parametrize("R", [8, 16, 64])
def test_tc_level_operator(field, R):
    U, o, rnd = field
    n = o.size(1)
    v = np.concatenate([po.gaussian(n, 50 + r) for r in range(R)])
    out = {}
    for tc in (0, 2):
        s = handle(U, rnd, tc, R)
        x = torch.tensor(v.view(np.float64).astype(np.float32), device="cuda")
        y = torch.zeros_like(x)
        ddamg.check(s.L.ddamg_apply_level_op_device(s.h, 1, 1, x.data_ptr(), y.data_ptr(), R))
        torch.cuda.synchronize()
        out[tc] = y.cpu().numpy().astype(np.float64).view(np.complex128)
        rep = s.autotune_report()
        s.close()
        if tc == 2:
            assert f"level 1 rhs {R} level operator:" in rep and "-> tensor cores" in rep, rep
    ref = np.concatenate([o.level_op(1, v[r * n:(r + 1) * n]) for r in range(R)])
    e_cc, e_tc, e_tt = rel(out[0], ref), rel(out[2], ref), rel(out[2], out[0])
    print(f"R {R}: CUDA cores vs FP64 oracle {e_cc:.1e}, tensor cores vs oracle {e_tc:.1e}, vs CUDA cores {e_tt:.1e}")
    assert e_cc < 1e-3
    assert e_tt < 5e-3 and e_tc < 5e-3
    for r in range(R):
        assert rel(out[2][r * n:(r + 1) * n], ref[r * n:(r + 1) * n]) < 5e-3


def test_batched_solve_with_tc_level_operator(field):
    U, o, rnd = field
    R = 16
    n = 2 * N * N
    b = np.concatenate([po.gaussian(n, 70 + r) for r in range(R)])
    s = handle(U, rnd, 2, R)
    x, info = s.solve(b, nrhs=R)
    x, info = s.solve(b, nrhs=R)  # the device-driven graph
    rep = s.autotune_report()
    s.close()
    assert "level operator:" in rep and "-> tensor cores" in rep, rep
    for r in range(R):
        assert info[r].converged == 1
        assert rel(po.dirac(N, N, M0, U, x[r * n:(r + 1) * n]), b[r * n:(r + 1) * n]) < 1e-10
