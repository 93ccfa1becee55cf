"""Iteration counts over several setups.  The reference's setup draws its test vectors from mt19937
(src/amg.cpp:6-17), which is not portable, so both codes are given the same injected random vectors
for each seed (pyoracle.uniform(rnd_count, seed)); the reference's V-cycle FGMRES iteration count for
every seed is in the golden file (tests/golden/make_golden.py, mode "seeds").  Cases: configs[0]
(64x64, 2 levels) and the bench's 256x256 3-level workload."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")


@pytest.mark.parametrize("name", ["seeds_64x64_l2", "seeds_256x256_l3"])
def test_iterations_match_reference_per_setup_seed(golden, name):
    z = golden(name)
    Nx, Nt, L, m0 = int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"])
    if "theta" in z:
        theta = z["theta"]
    else:  # regenerated: the Metropolis chain is seeded
        theta, _ = po.metropolis(Nx, Nt, float(z["beta"]), int(z["sweeps"]), int(z["seed"]))
    U = po.links_from_theta(theta)
    b = po.gaussian(2 * Nx * Nt, int(z["rhs_seed"]))
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, m0, z["rows"], fgmres_restart_length=int(z["fgmres_m"])))
    s.load_gauge(U)
    ours = []
    for sd in z["setup_seeds"]:
        s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(sd)))
        x, info = s.solve(b)
        assert info[0].converged and info[0].rel_residual < 1e-10
        ours.append(info[0].iterations)
    s.close()
    ref = [int(v) for v in z["ref_iters_V_seeds"]]
    for o, r in zip(ours, ref):
        assert abs(o - r) <= max(1, r // 10), (ours, ref)
    print(f"{name}: iterations per setup seed, GPU {ours}, reference {ref}")
