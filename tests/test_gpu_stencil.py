"""The two D_W kernel families against each other and against the oracle: the register kernels
(wilson_kernel, wilson_pair_kernel) and the staged-tile kernel (wilson_stage_kernel: bulk asynchronous
copies of 8 x 64-site tiles with their halo into shared memory).  Same arithmetic, so they agree to
rounding (1e-15 relative; 1e-6 in FP32), and both match the oracle's D_phi / D_dagger_phi (1e-13)."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")
torch = pytest.importorskip("torch")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(autouse=True)
def restore_variant():
    yield
    ddamg.set_stencil_kernel(0)


@pytest.mark.parametrize("Nx,Nt", [(64, 64), (16, 128), (8, 64), (32, 32)])
def test_staged_matches_register_and_oracle(Nx, Nt):
    th, _ = ddamg.gauge_metropolis(Nx, Nt, 2.0, 3, 5)
    U = np.exp(1j * th)
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, 2, -0.12, [[0, Nx // 4, Nt // 4, 4, Nx // 4, Nt // 4]], max_rhs=3))
    s.load_gauge(U)
    R = 3
    phi = np.concatenate([po.gaussian(Nx * Nt * 2, 20 + r) for r in range(R)])
    out = {}
    for kind in (1, 2):
        ddamg.set_stencil_kernel(kind)
        for dag in (0, 1):
            # FP64 through the host entry point, FP32 through the device one
            y = s.D_dagger_phi(phi, nrhs=R) if dag else s.D_phi(phi, nrhs=R)
            x32 = torch.tensor(phi.view(np.float64).astype(np.float32), device="cuda")
            y32 = torch.empty_like(x32)
            ddamg.check(s.L.ddamg_apply_dirac_f32_device(s.h, dag, x32.data_ptr(), y32.data_ptr(), R))
            torch.cuda.synchronize()
            out[kind, dag] = (y, y32.cpu().numpy().astype(np.float64).view(np.complex128))
    s.close()
    n = Nx * Nt * 2
    for dag in (0, 1):
        for r in range(R):
            ref = po.dirac(Nx, Nt, -0.12, U, phi[r * n:(r + 1) * n], dagger=bool(dag))
            for kind in (1, 2):
                assert rel(out[kind, dag][0][r * n:(r + 1) * n], ref) < 1e-13, (kind, dag, r)
                assert rel(out[kind, dag][1][r * n:(r + 1) * n], ref) < 1e-6, (kind, dag, r)
        assert rel(out[2, dag][0], out[1, dag][0]) < 1e-15
        assert rel(out[2, dag][1], out[1, dag][1]) < 1e-6


@pytest.mark.parametrize("precision", [ddamg.PREC_DOUBLE, ddamg.PREC_MIXED])
def test_solve_with_staged_stencil(golden, precision):
    """The solve's residuals (fused b - D x) and outer operator through the staged kernel."""
    z = golden("solve_64x64_l2")
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    res = {}
    for kind in (1, 2):
        ddamg.set_stencil_kernel(kind)
        s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], precision=precision,
                                              fgmres_restart_length=int(z["fgmres_m"])))
        s.load_gauge(U)
        s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
        x, info = s.solve(z["rhs"])
        s.close()
        res[kind] = (x, info[0].iterations)
    assert res[1][1] == res[2][1] == int(z["ref_iters_V"])
    assert rel(res[2][0], z["ref_x_V"]) < 1e-9
    assert rel(res[2][0], res[1][0]) < 1e-12
