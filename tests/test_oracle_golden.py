"""Pins the CPU restatement (oracle/ddamg_oracle.c) against outputs of the
reference's own code (tests/golden/*.npz, made by tests/golden/make_golden.py
from oracle/_ref).  Everything here runs on the CPU."""
import numpy as np
import pytest

import pyoracle as po

OPS = ["ops_16x32_l3", "ops_32x32_l2", "ops_32x16_l3"]
# the restatement follows the reference's arithmetic order, so agreement is to a few ulps
TOL = 1e-13


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make_oracle(z):
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    o = po.Oracle(Nx, Nt, L, float(z["m0"]), z["rows"], po.links_from_theta(z["theta"]))
    o.setup(po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    return o


@pytest.fixture(scope="module", params=OPS)
def case(request, golden):
    z = golden(request.param)
    return z, make_oracle(z)


def test_inputs_regenerate(golden):
    for name in OPS + ["solve_64x64_l2"]:
        z = golden(name)
        th, _ = po.metropolis(int(z["Nx"]), int(z["Nt"]), float(z["beta"]), int(z["sweeps"]), int(z["seed"]))
        assert np.array_equal(th, z["theta"])
        rhs = po.gaussian(int(z["Nx"]) * int(z["Nt"]) * 2, int(z["seed"]) + 7)
        assert np.array_equal(rhs, z["rhs"])


def test_dirac(case):
    z, o = case
    assert rel(o.dirac(z["probe_0"]), z["ref_Dphi"]) < TOL
    assert rel(o.dirac(z["probe_0"], True), z["ref_Ddagphi"]) < TOL


def test_level_ops_and_links(case):
    z, o = case
    L = int(z["levels"])
    for l in range(L):
        assert rel(o.level_op(l, z[f"probe_{l}"]), z[f"ref_Dop_{l}"]) < TOL
        if l >= 1:
            for w in (1, 2, 3):
                assert rel(o.get_links(l, w), z[f"ref_G{w}_{l}"]) < TOL, (l, w)


def test_transfers_and_tvec(case):
    z, o = case
    L = int(z["levels"])
    for l in range(L - 1):
        assert rel(o.get_tvec(l), z[f"ref_tvec_{l}"]) < TOL
        assert rel(o.restrict(l, z[f"probe_{l}"]), z[f"ref_Pdagg_{l}"]) < TOL
        assert rel(o.prolong(l, z[f"probe_{l + 1}"]), z[f"ref_P_{l}"]) < TOL


def test_sap_and_coarse(case):
    z, o = case
    L = int(z["levels"])
    for l in range(L - 1):
        x, it = o.sap(l, z[f"probe_{l}"], nu=3)
        assert it == int(z[f"ref_SAP_{l}_iters"])
        assert rel(x, z[f"ref_SAP_{l}"]) < TOL
    x, it = o.coarse_gmres(z[f"probe_{L - 1}"])
    assert it == int(z["ref_coarse_gmres_iters"])
    assert rel(x, z["ref_coarse_gmres"]) < 1e-12


def test_cycles(case):
    z, o = case
    assert rel(o.vcycle(z["probe_0"]), z["ref_vcycle"]) < 1e-12
    assert rel(o.kcycle(z["probe_0"]), z["ref_kcycle"]) < 1e-12


@pytest.mark.parametrize("name", ["ops_16x32_l3", "ops_32x32_l2", "solve_64x64_l2"])
@pytest.mark.parametrize("cycle,tag", [(0, "V"), (1, "K")])
def test_solve(golden, name, cycle, tag):
    z = golden(name)
    o = make_oracle(z)
    x, it = o.solve(z["rhs"], cycle=cycle, m=int(z["fgmres_m"]))
    assert it == int(z[f"ref_iters_{tag}"])
    assert rel(x, z[f"ref_x_{tag}"]) < 1e-12
    # the solve meets the reference's convergence test D x = b (src/methods.cpp:173-190)
    r = o.dirac(x) - z["rhs"]
    assert np.linalg.norm(r) / np.linalg.norm(z["rhs"]) < 1e-10


def test_gamma5_hermiticity(golden):
    """D^dagger = sigma_3 D sigma_3, the identity the adjoint solve relies on."""
    z = golden("ops_16x32_l3")
    o = make_oracle(z)
    v = z["probe_0"].reshape(-1, 2)
    s3 = np.array([1.0, -1.0])
    lhs = o.dirac(v.reshape(-1), True)
    rhs = (o.dirac((v * s3).reshape(-1)).reshape(-1, 2) * s3).reshape(-1)
    assert rel(lhs, rhs) < 1e-14


def test_galerkin_identity(golden):
    """D_c = P^dagger D P at every level (amg.cpp:249-298)."""
    z = golden("ops_16x32_l3")
    o = make_oracle(z)
    for l in range(int(z["levels"]) - 1):
        vc = z[f"probe_{l + 1}"]
        lhs = o.level_op(l + 1, vc)
        rhs = o.restrict(l, o.level_op(l, o.prolong(l, vc)))
        assert rel(lhs, rhs) < 1e-12


def test_krylov_comparison_solvers(golden):
    """bi_cgstab and conjugate_gradient on D^dagger D (src/conjugate_gradient.cpp) against the
    reference's own run: same iteration counts, same iterates to rounding."""
    z = golden("krylov_32x32")
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"]), z["rows"],
                  po.links_from_theta(z["theta"]))
    xb, itb = o.bicgstab(z["rhs"])
    assert itb == int(z["ref_iters_bicg"])
    assert rel(xb, z["ref_x_bicg"]) < 1e-12
    xc, itc = o.cg_normal(o.dirac(z["rhs"], True))  # Methods::CG solves with D^dagger rhs
    assert itc == int(z["ref_iters_cg"])
    assert rel(xc, z["ref_x_cg"]) < 1e-12
    for x in (xb, xc):
        assert np.linalg.norm(o.dirac(x) - z["rhs"]) / np.linalg.norm(z["rhs"]) < 1e-9


def test_iterations_per_setup_seed_64(golden):
    """The oracle, given the same injected setup vectors, takes the reference's V-cycle iteration count
    for every seed of configs[0] (64x64, 2 levels)."""
    z = golden("seeds_64x64_l2")
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"]), z["rows"],
                  po.links_from_theta(z["theta"]))
    its = []
    for sd in z["setup_seeds"][:4]:
        o.setup(po.uniform(int(z["rnd_count"]), int(sd)))
        _, it = o.solve(z["rhs"], cycle=0, m=int(z["fgmres_m"]))
        its.append(it)
    assert its == [int(v) for v in z["ref_iters_V_seeds"][:4]]


@pytest.mark.parametrize("name", ["multilevel_32x32_l2", "multilevel_16x32_l3"])
@pytest.mark.parametrize("cycle,tag", [(0, "V"), (1, "K")])
def test_apply_multilevel(golden, name, cycle, tag):
    """AlgebraicMG::applyMultilevel (src/amg.cpp:177-243): same cycle count, same iterate bit for bit."""
    z = golden(name)
    o = make_oracle(z)
    x, n, relres = o.apply_multilevel(z["rhs"], cycle=cycle, it=100, tol=1e-10)
    assert n == int(z[f"ref_cycles_ml_{tag}"])
    assert relres < 1e-10
    assert rel(x, z[f"ref_x_ml_{tag}"]) < TOL


@pytest.mark.parametrize("name", ["multilevel_32x32_l2", "fgmres_sap_64x64"])
def test_fgmres_sap(golden, name):
    """FGMRES_SAP (include/sap.h:236-333) with the reference's 4 x 4 SAP blocks."""
    z = golden(name)
    Nx, Nt = int(z["Nx"]), int(z["Nt"])
    o = po.Oracle(Nx, Nt, int(z["levels"]), float(z["m0"]), z["rows"], po.links_from_theta(z["theta"]))
    x, it = o.fgmres_sap(z["rhs"], 4, 4, m=int(z["fgmres_m"]), restarts=50, tol=1e-10)
    assert it == int(z["ref_iters_fsap"])
    assert rel(x, z["ref_x_fsap"]) < TOL
    assert rel(po.dirac(Nx, Nt, float(z["m0"]), po.links_from_theta(z["theta"]), x), z["rhs"]) < 1e-10


def test_sap_fine(golden):
    """SAP_C::SAP of SAP_fine_level (Methods::SAP) over 4 x 8 blocks, 3 iterations from zero."""
    z = golden("multilevel_32x32_l2")
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"]), z["rows"],
                  po.links_from_theta(z["theta"]))
    x, it = o.sap_fine(z["rhs"], 4, 8, nu=3)
    assert it == int(z["ref_iters_sapfine_4x8"])
    assert rel(x, z["ref_x_sapfine_4x8"]) < TOL


def test_dirac_plain_matches_hierarchy(golden):
    z = golden("ops_16x32_l3")
    U = po.links_from_theta(z["theta"])
    o = make_oracle(z)
    for dag in (False, True):
        assert np.array_equal(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, z["probe_0"], dag),
                              o.dirac(z["probe_0"], dag))


def test_solve_256_fixture_regenerates(golden):
    """The bench workload's fixture stores only the reference's solution: its field and right-hand side come
    back from their seeds, and the reference's solution has the residual the reference reported."""
    z = golden("solve_256x256_l3")
    Nx, Nt = int(z["Nx"]), int(z["Nt"])
    th, _ = po.metropolis(Nx, Nt, float(z["beta"]), int(z["sweeps"]), int(z["seed"]))
    U = po.links_from_theta(th)
    b = po.gaussian(2 * Nx * Nt, int(z["rhs_seed"]))
    r = rel(po.dirac(Nx, Nt, float(z["m0"]), U, z["ref_x_V"]), b)
    assert r < 1e-10
    assert abs(r - float(z["ref_relres_V"])) < 1e-3 * r
