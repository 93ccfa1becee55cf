"""C-ABI checks that need no GPU: the library loads, exports every entry point declared in
include/ddamg.h, and its host-only functions (parameters parser, binary I/O, RHS generator)
agree with the reference formats and the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyoracle as po
from ddamg import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(REPO, "include", "ddamg.h")).read()
    return sorted(set(re.findall(r"\b(ddamg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(L, s), s
    # the Python binding declares exactly the header's entry points
    assert sorted(_lib.SIGNATURES) == syms


def test_params_default_matches_reference_constants():
    import ddamg

    p = ddamg.default_params()
    # src/variables.cpp:100-134
    assert (p.sap_gmres_restart_length, p.sap_gmres_restarts, p.sap_gmres_tolerance) == (5, 5, 1e-3)
    assert p.sap_test_vectors_iterations == 4
    assert (p.coarse_gmres_restart_length, p.coarse_gmres_restarts, p.coarse_gmres_tolerance) == (400, 10, 0.1)
    assert (p.nu1, p.nu2) == (0, 2)
    assert (p.kcycle_restart_length, p.kcycle_restarts, p.kcycle_tolerance) == (5, 2, 0.1)
    assert (p.fgmres_restart_length, p.fgmres_restarts, p.fgmres_tolerance) == (20, 50, 1e-10)


def test_parse_params_file(tmp_path):
    import ddamg

    f = tmp_path / "parameters"
    f.write_text("0 64 64 12 64 64\n1 16 16 12 16 16\n")
    p = ddamg.read_parameters(str(f), 3)
    assert [list(p.rows[i]) for i in range(2)] == [[0, 64, 64, 12, 64, 64], [1, 16, 16, 12, 16, 16]]
    # row count must equal levels - 1 (include/params.h:101-104)
    with pytest.raises(ddamg.DDAMGError) as e:
        ddamg.read_parameters(str(f), 2)
    assert e.value.status == _lib.ERR_BAD_PARAM
    with pytest.raises(ddamg.DDAMGError) as e:
        ddamg.read_parameters(str(tmp_path / "missing"), 2)
    assert e.value.status == _lib.ERR_IO
    bad = tmp_path / "bad"
    bad.write_text("0 8 8 x 4 4\n")
    with pytest.raises(ddamg.DDAMGError):
        ddamg.read_parameters(str(bad), 2)


def test_binary_io_roundtrip_against_oracle(tmp_path):
    import ddamg

    Nx, Nt = 6, 10
    field = po.gaussian(2 * Nx * Nt, 5)
    a, b = str(tmp_path / "a.bin"), str(tmp_path / "b.bin")
    ddamg.write_binary(a, Nx, Nt, field)
    po.write_binary(b, Nx, Nt, field)
    assert open(a, "rb").read() == open(b, "rb").read()
    assert os.path.getsize(a) == 28 * 2 * Nx * Nt  # src/io.cpp:32-44 record size
    assert np.array_equal(ddamg.read_binary(a, Nx, Nt), field)
    with pytest.raises(ddamg.DDAMGError) as e:
        ddamg.read_binary(str(tmp_path / "none.bin"), Nx, Nt)
    assert e.value.status == _lib.ERR_IO
    with pytest.raises(ddamg.DDAMGError):
        ddamg.read_binary(a, Nx, Nt + 2)  # short file


def test_gaussian_field_matches_oracle():
    import ddamg

    g = ddamg.gaussian_field(1000, 42)
    assert np.array_equal(g, po.gaussian(1000, 42))
    assert abs(np.mean(np.abs(g) ** 2) - 1.0) < 0.1


def test_null_handle_and_bad_args_rejected():
    L = _lib.load()
    assert L.ddamg_load_gauge(None, None) == _lib.ERR_BAD_PARAM
    assert L.ddamg_params_default(None) == _lib.ERR_BAD_PARAM
    assert L.ddamg_gauge_metropolis(3, 4, 1.0, 1, 1, 1.0, None, None, 0) == _lib.ERR_BAD_PARAM


def test_halo_layout_round_trip():
    """ddamg_from_halo / ddamg_to_halo follow the reference's spinor indexing idx(x, t, mu) =
    (x*(Nt+2)+t)*DOF + mu for x, t >= 1 (include/utils.h:46-52)."""
    import ddamg

    Nx, Nt, dof = 5, 7, 4
    rng = np.random.default_rng(3)
    halo = rng.standard_normal((Nx + 2) * (Nt + 2) * dof) + 1j * rng.standard_normal((Nx + 2) * (Nt + 2) * dof)
    c = ddamg.from_halo(halo, Nx, Nt, dof)
    for x in range(1, Nx + 1):
        for t in range(1, Nt + 1):
            for d in range(dof):
                assert c[((x - 1) * Nt + (t - 1)) * dof + d] == halo[(x * (Nt + 2) + t) * dof + d]
    h2 = ddamg.to_halo(c, Nx, Nt, dof)
    inner = np.zeros((Nx + 2, Nt + 2), dtype=bool)
    inner[1:-1, 1:-1] = True
    mask = np.repeat(inner.reshape(-1), dof)
    assert np.array_equal(h2[mask], halo[mask]) and not h2[~mask].any()
    assert ddamg._lib.load().ddamg_from_halo(None, Nx, Nt, dof, None) == _lib.ERR_BAD_PARAM
