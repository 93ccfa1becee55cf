"""The two coarsest-level GMRES kernels (Level::GMRES_level_l, include/level.h:70-140): the cooperative-grid
kernel and the thread-block-cluster kernel (one cluster of up to 16 CTAs per right-hand side, hardware
cluster barriers, neighbours and partial sums through distributed shared memory).  The same arithmetic per
element with other reduction trees: the same iteration counts, solutions within 1e-12 of each other and
1e-9 of the oracle; the multigrid solves built on either agree to 1e-12."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(z, kernel, **kw):
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], coarse_kernel=kernel,
                                          fgmres_restart_length=int(z["fgmres_m"]), **kw))
    s.load_gauge(U)
    s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    return s, U


@pytest.mark.parametrize("name", ["ops_16x32_l3", "ops_32x32_l2", "ops_32x16_l3"])
def test_cluster_coarse_gmres_matches_cooperative_and_oracle(golden, name):
    z = golden(name)
    L = int(z["levels"])
    b = z[f"probe_{L - 1}"]
    res = {}
    for kernel in (1, 2):
        s, U = make(z, kernel)
        rep = s.autotune_report()
        res[kernel] = s.coarse_gmres(b)
        s.close()
        assert ("cluster" if kernel == 2 else "cooperative grid") in rep, rep
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), L, float(z["m0"]), z["rows"], U)
    o.setup(po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    xo, ito = o.coarse_gmres(b)
    (x1, it1), (x2, it2) = res[1], res[2]
    print(f"{name}: iterations cooperative {it1}, cluster {it2}, oracle {ito}; cluster vs cooperative "
          f"{rel(x2, x1):.1e}, vs oracle {rel(x2, xo):.1e}")
    assert it1 == it2 == ito
    assert rel(x2, x1) < 1e-12 and rel(x2, xo) < 1e-9


@pytest.mark.parametrize("precision", [ddamg.PREC_DOUBLE, ddamg.PREC_MIXED])
def test_solves_on_cluster_coarse_kernel(golden, precision):
    """Single and batched (one launch, clusters looping over the right-hand sides) solves."""
    z = golden("solve_64x64_l2")
    n = z["rhs"].size
    R = 3
    bs = np.concatenate([z["rhs"]] + [po.gaussian(n, 900 + r) for r in range(R - 1)])
    out = {}
    for kernel in (1, 2):
        s, U = make(z, kernel, precision=precision, max_rhs=R)
        x1, i1 = s.solve(z["rhs"])
        xb, ib = s.solve(bs, nrhs=R)
        s.close()
        out[kernel] = (x1, i1[0].iterations, xb, [i.iterations for i in ib])
    assert out[1][1] == out[2][1] == int(z["ref_iters_V"])
    assert out[1][3] == out[2][3]
    assert rel(out[2][0], out[1][0]) < 1e-12 and rel(out[2][2], out[1][2]) < 1e-12
    assert rel(out[2][0], z["ref_x_V"]) < 1e-9
    for r in range(R):
        assert rel(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, out[2][2][r * n:(r + 1) * n]),
                   bs[r * n:(r + 1) * n]) < 1e-10


def test_coarse_kernel_chosen_by_timing(golden):
    z = golden("solve_64x64_l2")
    s, _ = make(z, 0)
    rep = s.autotune_report()
    s.close()
    assert "coarsest solve, 1 rhs:" in rep and " -> " in rep, rep
