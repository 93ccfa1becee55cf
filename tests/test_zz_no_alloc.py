"""The allocation-free coarsest solve (ddamg_coarse_gmres_noalloc) against the handle-based one.

It exists for callers that cannot allocate device memory while they solve; its scratch is one
fixed array compiled into the library, shared by every call.  This file is collected last so a
run that stops at the first failure has already run every other test.  Two calls in a row check
that the contents the first call leaves in the shared array do not leak into the second.
"""
import ctypes

import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")
torch = pytest.importorskip("torch")

# both paths run the same kernel with the same grid, so they agree to rounding of identical work
TOL = 1e-12


def device_links(s, level, C):
    """Reference-layout coarse links (G1/G2/G3) -> the library's [site][d][j][i] layout."""
    G1, G2, G3 = (s.coarse_links(level, w) for w in (1, 2, 3))
    S, dof = G1.size // (4 * C * C), 2 * C
    g1 = G1.reshape(S, 2, 2, C, C)
    g2 = G2.reshape(S, 2, 2, C, C, 2)
    g3 = G3.reshape(S, 2, 2, C, C, 2)
    M = np.zeros((S, 5, dof, dof), dtype=np.complex128)
    for d, A in enumerate((g1, g2[..., 0], g2[..., 1], g3[..., 0], g3[..., 1])):
        # [s][alf][bet][c][b] -> [s][j = b*2+bet][i = c*2+alf]
        M[:, d] = A.transpose(0, 4, 2, 3, 1).reshape(S, dof, dof)
    return M


def test_noalloc_coarse_gmres_matches_handle(golden):
    z = golden("ops_16x32_l3")
    Nx, Nt, L, m0 = int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"])
    rows = z["rows"]
    p = ddamg.default_params(Nx, Nt, L, m0, rows)
    s = ddamg.Solver(p)
    s.load_gauge(po.links_from_theta(z["theta"]))
    s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    C = int(rows[L - 2][3])
    cx, ct = int(rows[L - 2][1]), int(rows[L - 2][2])
    dev = torch.device("cuda:0")
    links = torch.from_numpy(device_links(s, L - 1, C).view(np.float64).copy()).to(dev)
    lib = ddamg._lib.load()
    n = cx * ct * 2 * C
    for call, seed in enumerate((501, 502)):
        b = po.gaussian(n, seed)
        x_ref, it_ref = s.coarse_gmres(b)
        bd = torch.from_numpy(b.view(np.float64).copy()).to(dev)
        xd = torch.full_like(bd, float("nan"))  # the output must be fully written
        it = ctypes.c_int(-1)
        torch.cuda.synchronize()
        st = lib.ddamg_coarse_gmres_noalloc(links.data_ptr(), bd.data_ptr(), xd.data_ptr(), cx, ct, 2 * C, m0,
                                            p.coarse_gmres_restart_length, p.coarse_gmres_restarts,
                                            p.coarse_gmres_tolerance, None, ctypes.byref(it))
        assert st == ddamg._lib.OK, lib.ddamg_last_error()
        x = xd.cpu().numpy().view(np.complex128)
        assert it.value == it_ref, (call, it.value, it_ref)
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < TOL, call
    s.close()


def test_noalloc_rejects_oversized_requests():
    lib = ddamg._lib.load()
    dev = torch.device("cuda:0")
    buf = torch.zeros(2, dtype=torch.float64, device=dev)
    # 64x64 sites x 64 dof with m = 400 needs far more than the fixed scratch
    st = lib.ddamg_coarse_gmres_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 64, 64, 64, -0.1, 400, 1,
                                        0.1, None, None)
    assert st == ddamg._lib.ERR_BAD_PARAM
    assert b"scratch" in lib.ddamg_last_error()
