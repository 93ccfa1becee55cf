"""The device-driven FGMRES: from the second solve of a batch width on, a solve runs as one CUDA graph
whose conditional nodes carry the FGMRES loops (the outer one and, for K-cycles, the inner FGMRES of
every coarse level), with the Hessenberg, Givens and restart work in device kernels.  It must give the
host-driven loop's iterations and solution (1e-12: the same arithmetic, the small dense work compiled
for the device instead of the host) and the reference's solution (1e-9)."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(z, precision, cycle, max_rhs=1, graphs=1):
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    p = ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], precision=precision, cycle=cycle,
                             max_rhs=max_rhs, fgmres_restart_length=int(z["fgmres_m"]), cuda_graphs=graphs)
    s = ddamg.Solver(p)
    s.load_gauge(U)
    s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    return s, U


@pytest.mark.parametrize("name", ["ops_16x32_l3", "solve_64x64_l2"])
@pytest.mark.parametrize("cycle,tag", [(ddamg.CYCLE_V, "V"), (ddamg.CYCLE_K, "K")])
@pytest.mark.parametrize("precision", [ddamg.PREC_DOUBLE, ddamg.PREC_MIXED])
def test_device_driven_solve_matches_host_driven(golden, name, cycle, tag, precision):
    z = golden(name)
    s, U = make(z, precision, cycle)
    c0 = ddamg.Solver.launch_count()
    x1, i1 = s.solve(z["rhs"])  # first solve of this width: host driven (tunes, captures the V-cycle)
    c1 = ddamg.Solver.launch_count()
    x2, i2 = s.solve(z["rhs"])  # device driven
    c2 = ddamg.Solver.launch_count()
    rep = s.autotune_report()
    s.close()
    assert "solve graph rhs 1:" in rep, rep
    assert i2[0].iterations == i1[0].iterations and i2[0].converged == 1
    assert abs(i2[0].rel_residual - i1[0].rel_residual) <= 1e-3 * i1[0].rel_residual
    e12 = rel(x2, x1)
    res = rel(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, x2), z["rhs"])
    eref = rel(x2, z[f"ref_x_{tag}"])
    print(f"{name} {tag} prec {precision}: iterations {i2[0].iterations}, host vs device {e12:.1e}, "
          f"residual {res:.1e}, vs reference {eref:.1e}, launches host {c1 - c0} device {c2 - c1}")
    assert e12 < 1e-12
    assert res < 1e-10 and eref < 1e-9
    # the launches of the device-driven solve are counted from its bodies' run counters: the same order
    # of magnitude as the host-driven loop's
    assert 0.5 * (c1 - c0) < c2 - c1 < 2.0 * (c1 - c0)


@pytest.mark.parametrize("cycle", [ddamg.CYCLE_V, ddamg.CYCLE_K])
def test_device_driven_batched_with_zero_rhs(golden, cycle):
    """Lockstep right-hand sides finish at different steps; a zero one takes 0 iterations."""
    z = golden("ops_16x32_l3")
    R = 3
    s, U = make(z, ddamg.PREC_MIXED, cycle, max_rhs=R)
    n = z["rhs"].size
    b = np.concatenate([po.gaussian(n, 401), np.zeros(n, dtype=np.complex128), z["rhs"]])
    x1, i1 = s.solve(b, nrhs=R)
    x2, i2 = s.solve(b, nrhs=R)
    rep = s.autotune_report()
    s.close()
    assert f"solve graph rhs {R}:" in rep
    for r in range(R):
        assert i2[r].iterations == i1[r].iterations
    for r in (0, 2):
        assert rel(x2[r * n:(r + 1) * n], x1[r * n:(r + 1) * n]) < 1e-12
    assert np.all(x2[n:2 * n] == 0) and i2[1].iterations == 0
    for r in (0, 2):
        assert rel(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, x2[r * n:(r + 1) * n]),
                   b[r * n:(r + 1) * n]) < 1e-10


def test_graphs_off_stays_host_driven(golden):
    z = golden("ops_16x32_l3")
    s, _ = make(z, ddamg.PREC_DOUBLE, ddamg.CYCLE_V, graphs=0)
    s.solve(z["rhs"])
    s.solve(z["rhs"])
    assert "solve graph" not in s.autotune_report()
    s.close()
