"""The reference's other solver entry points on the GPU, through the C ABI, against the reference's own
outputs (tests/golden/multilevel_*.npz, fgmres_sap_64x64.npz, made by tests/golden/make_golden.py) and
the oracle:

  * AlgebraicMG::applyMultilevel (src/amg.cpp:177-243), the stand-alone V/K-cycle iteration;
  * FGMRES_SAP (include/sap.h:236-333), FGMRES preconditioned by one fine-level SAP iteration;
  * SAP_C::SAP of SAP_fine_level (Methods::SAP, src/methods.cpp:60-80) over its own block counts;
  * the bounded grid barrier of the coarsest-level GMRES: a poll limit of 1 makes it give up, the call
    reports DDAMG_ERR_DEVICE_TIMEOUT, and the same handle solves normally once the limit is back.

Tolerances (relative 2-norm): solutions 1e-9 against the reference's FP64 solution, true residuals below
1e-10 under the oracle's operator; SAP iterates (no solver tolerance involved) 1e-9.
"""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solver(z, precision=ddamg.PREC_DOUBLE, cycle=ddamg.CYCLE_V, setup=True, **kw):
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], precision=precision, cycle=cycle,
                                          fgmres_restart_length=int(z["fgmres_m"]), **kw))
    s.load_gauge(U)
    if setup:
        s.setUpPhase(vectors=po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    return s, U


@pytest.mark.parametrize("name", ["multilevel_32x32_l2", "multilevel_16x32_l3"])
@pytest.mark.parametrize("cycle,tag", [(ddamg.CYCLE_V, "V"), (ddamg.CYCLE_K, "K")])
def test_apply_multilevel_matches_reference(golden, name, cycle, tag):
    z = golden(name)
    s, U = solver(z, cycle=cycle)
    x, n, relres = s.applyMultilevel(z["rhs"], max_cycles=100, tol=1e-10)
    s.close()
    ref_n = int(z[f"ref_cycles_ml_{tag}"])
    res = rel(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, x), z["rhs"])
    e = rel(x, z[f"ref_x_ml_{tag}"])
    print(f"{name} {tag}: cycles {n} (reference {ref_n}), residual {res:.2e}, rel diff {e:.2e}")
    assert n == ref_n
    assert relres < 1e-10 and res < 1e-10
    assert e < 1e-9


@pytest.mark.parametrize("cycle", [ddamg.CYCLE_V, ddamg.CYCLE_K])
def test_apply_multilevel_mixed(golden, cycle):
    """Mixed precision: FP32 cycles on the FP64 residual reach the FP64 tolerance."""
    z = golden("multilevel_16x32_l3")
    tag = "V" if cycle == ddamg.CYCLE_V else "K"
    s, U = solver(z, precision=ddamg.PREC_MIXED, cycle=cycle)
    x, n, relres = s.applyMultilevel(z["rhs"], max_cycles=100, tol=1e-10)
    s.close()
    ref_n = int(z[f"ref_cycles_ml_{tag}"])
    assert relres < 1e-10
    assert rel(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, x), z["rhs"]) < 1e-10
    assert abs(n - ref_n) <= max(1, ref_n // 10), (n, ref_n)
    assert rel(x, z[f"ref_x_ml_{tag}"]) < 1e-9


def test_apply_multilevel_initial_guess_and_limits(golden):
    z = golden("multilevel_32x32_l2")
    s, U = solver(z)
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"]), z["rows"], U)
    o.setup(po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    # a non-zero initial guess: three cycles on it, as the oracle's applyMultilevel does
    x0 = po.gaussian(z["rhs"].size, 5)
    xg, ng, rg = s.applyMultilevel(z["rhs"], x0=x0, max_cycles=3, tol=1e-10, allow_not_converged=True)
    xo, no, ro = o.apply_multilevel(z["rhs"], it=3, tol=1e-10, x0=x0)
    assert ng == no == 3
    assert rel(xg, xo) < 1e-9 and abs(rg - ro) < 1e-6 * ro
    with pytest.raises(ddamg.DDAMGError) as e:
        s.applyMultilevel(z["rhs"], max_cycles=2, tol=1e-10)
    assert e.value.status == ddamg._lib.NOT_CONVERGED
    # the zero right-hand side: x = 0 after 0 cycles
    x, n, r = s.applyMultilevel(np.zeros_like(z["rhs"]), x0=x0)
    assert n == 0 and not np.any(x)
    s.close()


@pytest.mark.parametrize("name", ["multilevel_32x32_l2", "fgmres_sap_64x64"])
@pytest.mark.parametrize("precision", [ddamg.PREC_DOUBLE, ddamg.PREC_MIXED])
def test_fgmres_sap_matches_reference(golden, name, precision):
    z = golden(name)
    s, U = solver(z, precision=precision, setup=False)
    x, info = s.fgmres_sap(z["rhs"], 4, 4, m=int(z["fgmres_m"]), restarts=50, tol=1e-10)
    s.close()
    ref_it = int(z["ref_iters_fsap"])
    res = rel(po.dirac(int(z["Nx"]), int(z["Nt"]), float(z["m0"]), U, x), z["rhs"])
    e = rel(x, z["ref_x_fsap"])
    print(f"{name} prec {precision}: FGMRES_SAP iterations {info.iterations} (reference {ref_it}), residual "
          f"{res:.2e}, rel diff {e:.2e}")
    assert info.converged == 1 and res < 1e-10
    assert abs(info.iterations - ref_it) <= max(1, ref_it // 10)
    assert e < 1e-9


def test_sap_fine_matches_reference(golden):
    z = golden("multilevel_32x32_l2")
    s, U = solver(z, setup=False)
    x, it = s.SAP_fine(z["rhs"], 4, 8, nu=3)
    assert it == int(z["ref_iters_sapfine_4x8"])
    assert rel(x, z["ref_x_sapfine_4x8"]) < 1e-9
    # bad block counts are rejected on the host
    for bx, bt in ((3, 4), (5, 8), (1, 3)):
        with pytest.raises(ddamg.DDAMGError) as e:
            s.SAP_fine(z["rhs"], bx, bt, nu=1)
        assert e.value.status == ddamg._lib.ERR_BAD_PARAM
    s.close()


def test_counters_and_metadata(golden, tmp_path):
    """The handle's iteration counters follow each method's last run and land in the metadata file
    (writeMetadata, src/io.cpp:72-145)."""
    z = golden("multilevel_32x32_l2")
    s, U = solver(z)
    assert set(s.counters().values()) == {-1}
    _, it_sap = s.SAP_fine(z["rhs"], 4, 8, nu=3)
    _, info_f = s.fgmres_sap(z["rhs"], 4, 4, m=20, restarts=50, tol=1e-10)
    _, info_v = s.solve(z["rhs"])
    c = s.counters()
    assert (c["SAP"], c["FGMRES_SAP"], c["vCycle"]) == (it_sap, info_f.iterations, info_v[0].iterations)
    assert c["kCycle"] == -1 and c["CG"] == -1
    path = str(tmp_path / "meta.dat")
    s.writeMetadata(ddamg.CYCLE_V, 1e-10, path)
    s.close()
    lines = open(path).read().splitlines()
    i = lines.index("#V cycle fgmres iterations,  Setup phase FLOPS, Total FLOPS")
    assert int(lines[i + 1].split()[0]) == info_v[0].iterations
    i = lines.index("#SAP iterations,   FLOPS")
    assert int(lines[i + 1].split()[0]) == it_sap


def test_coarse_barrier_timeout_then_recovers(golden):
    """A poll limit of 1 makes the coarsest GMRES kernel's first barrier that has to wait give up: every CTA
    leaves at its next barrier, the call reports DEVICE_TIMEOUT, and after the limit is restored the same
    handle's coarsest solve and full solve agree with the oracle (the status word is cleared per launch)."""
    z = golden("ops_16x32_l3")
    s, U = solver(z, coarse_kernel=1)  # the cooperative-grid kernel, whose grid barriers poll
    o = po.Oracle(int(z["Nx"]), int(z["Nt"]), int(z["levels"]), float(z["m0"]), z["rows"], U)
    o.setup(po.uniform(int(z["rnd_count"]), int(z["seed"]) + 1))
    L = int(z["levels"])
    b = z[f"probe_{L - 1}"]
    s.set_coarse_barrier_polls(1)
    statuses = []
    for _ in range(5):  # a barrier whose CTAs all arrive within one poll does not wait: try a few solves
        try:
            s.coarse_gmres(b)
            statuses.append(ddamg._lib.OK)
        except ddamg.DDAMGError as e:
            statuses.append(e.status)
            if e.status == ddamg._lib.ERR_DEVICE_TIMEOUT:
                break
    assert statuses[-1] == ddamg._lib.ERR_DEVICE_TIMEOUT, statuses
    s.set_coarse_barrier_polls(1 << 24)
    xg, itg = s.coarse_gmres(b)
    xo, ito = o.coarse_gmres(b)
    assert itg == ito and rel(xg, xo) < 1e-9
    x, info = s.solve(z["rhs"])
    assert info[0].converged == 1 and rel(o.dirac(x), z["rhs"]) < 1e-10
    s.close()
