"""GPU parity of the comparison solvers (src/conjugate_gradient.cpp): BiCGstab on D_W and CG on the
normal equations D^dagger D, through the C ABI, against the reference's own run on the 32x32
golden case (tests/golden/krylov_32x32.npz) and the oracle restatement.

Tolerances: the GPU sums in a different order than the reference, so the iterates drift apart at
rounding level and the stopping iteration can move by a few: iteration counts within 10 %,
solutions within the solver tolerance times the conditioning (1e-7 for BiCGstab on D, 1e-6 for CG
on D^dagger D, whose condition number is the square)."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def case(golden):
    z = golden("krylov_32x32")
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"]))
    s.load_gauge(U)
    o = po.Oracle(Nx, Nt, L, float(z["m0"]), z["rows"], U)
    yield z, s, o
    s.close()


def test_bicgstab_matches_reference(case):
    z, s, o = case
    b = z["rhs"]
    x, info = s.bi_cgstab(b)
    ref_it = int(z["ref_iters_bicg"])
    assert info.converged
    assert abs(info.iterations - ref_it) <= max(2, ref_it // 10), (info.iterations, ref_it)
    assert info.rel_residual < 2e-10
    assert rel(o.dirac(x), b) < 2e-10
    assert rel(x, z["ref_x_bicg"]) < 1e-7


def test_cg_normal_matches_reference(case):
    z, s, o = case
    b = z["rhs"]
    phi = s.D_dagger_phi(b)
    assert rel(phi, o.dirac(b, True)) < 1e-14
    x, info = s.conjugate_gradient(phi)
    ref_it = int(z["ref_iters_cg"])
    assert info.converged
    assert abs(info.iterations - ref_it) <= max(2, ref_it // 10), (info.iterations, ref_it)
    assert info.rel_residual < 2e-10  # ||phi - D^dagger D x|| / ||phi||
    assert rel(x, z["ref_x_cg"]) < 1e-6
    # Methods::CG: the same solve from b
    x2, info2 = s.CG(b)
    assert info2.iterations == info.iterations and rel(x2, x) < 1e-14


def test_bicgstab_from_x0_and_iteration_cap(case):
    z, s, o = case
    b = z["rhs"]
    # starting at the oracle's converged solution the first ||s|| test passes: k+1 = 1
    xo, _ = o.bicgstab(b)
    x, info = s.bi_cgstab(b, x0=xo, tol=1e-8)
    assert info.converged and info.iterations == 1
    assert rel(x, xo) < 1e-8
    # a cap the solve cannot meet: DDAMG_NOT_CONVERGED with the reference's count (max_iter)
    x, info = s.bi_cgstab(b, max_iter=5)
    assert not info.converged and info.iterations == 5
    xo5, it5 = o.bicgstab(b, max_iter=5)
    assert it5 == 5 and rel(x, xo5) < 1e-10
    x, info = s.conjugate_gradient(s.D_dagger_phi(b), max_iter=7)
    assert not info.converged and info.iterations == 7


def test_repeated_solves_are_deterministic(case):
    z, s, _ = case
    b = z["rhs"]
    x1, i1 = s.bi_cgstab(b)
    x2, i2 = s.bi_cgstab(b)
    assert i1.iterations == i2.iterations and np.array_equal(x1, x2)
    # with cuda_graphs (the default) the iteration runs as a device-side graph loop
    assert "bicgstab: device loop" in s.autotune_report()


def test_host_batched_path_matches_device_loop(golden):
    z = golden("krylov_32x32")
    Nx, Nt, L = int(z["Nx"]), int(z["Nt"]), int(z["levels"])
    U = po.links_from_theta(z["theta"])
    out = []
    for graphs in (1, 0):
        s = ddamg.Solver(ddamg.default_params(Nx, Nt, L, float(z["m0"]), z["rows"], cuda_graphs=graphs))
        s.load_gauge(U)
        out.append((s.bi_cgstab(z["rhs"]), s.conjugate_gradient(z["rhs"], max_iter=50), s.autotune_report()))
        s.close()
    (xa, ia), (ca, ja), ra = out[0]
    (xb, ib), (cb, jb), rb = out[1]
    assert "device loop" in ra and "host-queued" in rb
    assert ia.iterations == ib.iterations and np.array_equal(xa, xb)
    assert ja.iterations == jb.iterations == 50 and np.array_equal(ca, cb)


def test_zero_rhs(case):
    z, s, _ = case
    b = np.zeros_like(z["rhs"])
    x, info = s.bi_cgstab(b)
    assert info.converged and info.iterations == 0 and not x.any()
    x, info = s.conjugate_gradient(b)
    assert info.converged and info.iterations == 0 and not x.any()
