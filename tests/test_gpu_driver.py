"""The command-line driver (ddalphaamg-sm_b200/driver/ddamg_main.cpp), a C++ program that calls only the
C ABI and follows the reference's run sequence (src/main.cpp): the same seven answers on standard input,
then CG on the normal equations, FGMRES with the V-cycle and with the K-cycle, and the solution check.
Run on the 32x32 golden case against the reference's own results for it."""
import os
import re
import subprocess

import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu
ddamg = pytest.importorskip("ddamg")

DRIVER = os.path.join(os.path.dirname(ddamg.__file__), "ddamg_main")


def test_driver_follows_the_reference_main(golden, tmp_path):
    z = golden("krylov_32x32")
    zs = golden("ops_32x32_l2")  # the same lattice, field and right-hand side (seed 12)
    assert np.array_equal(z["theta"], zs["theta"]) and np.array_equal(z["rhs"], zs["rhs"])
    Nx, Nt = int(z["Nx"]), int(z["Nt"])
    conf, rhs, par, xout = (str(tmp_path / f) for f in ("conf.bin", "rhs.bin", "params", "x.bin"))
    po.write_binary(conf, Nx, Nt, po.links_from_theta(z["theta"]))
    po.write_binary(rhs, Nx, Nt, z["rhs"])
    with open(par, "w") as f:
        for r in z["rows"]:
            f.write(" ".join(str(int(v)) for v in r) + "\n")
    answers = f"1 1 {int(z['levels'])} {float(z['m0'])!r} {conf} {rhs} {par}\n"
    r = subprocess.run([DRIVER, str(Nx), str(Nt), xout], input=answers, capture_output=True, text=True, timeout=300,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    out = r.stdout
    cg = int(re.search(r"CG for D\^\+D converged in (\d+) iterations", out).group(1))
    ref_cg = int(z["ref_iters_cg"])
    assert abs(cg - ref_cg) <= max(2, ref_cg // 10), (cg, ref_cg)
    runs = re.findall(r"FGMRES converged in (\d+) iterations, relative residual ([0-9.e+-]+)", out)
    assert len(runs) == 2  # V-cycle, K-cycle
    for it, res in runs:
        assert float(res) < 1e-10
    # the reference's own stock-setup V-cycle solve of this system
    assert abs(int(runs[0][0]) - int(zs["ref_iters_V_stock"])) <= 2
    assert out.count("Solution verified") == 2 and "Solution differs" not in out
    # the two metadata files of src/main.cpp:92,97 (writeMetadata), in the working directory
    L = int(z["levels"])
    for tag, (it, _) in zip("VK", runs):
        lines = open(tmp_path / f"metadata_{Nx}x{Nt}_Levels{L}_{tag}cycle.dat").read().splitlines()
        i = lines.index(f"#{tag} cycle fgmres iterations,  Setup phase FLOPS, Total FLOPS")
        assert int(lines[i + 1].split()[0]) == int(it)
        i = lines.index("#CG iterations,   FLOPS")
        assert int(lines[i + 1].split()[0]) == cg
    x = po.read_binary(xout, Nx, Nt)
    assert np.linalg.norm(x - zs["ref_x_V"]) / np.linalg.norm(zs["ref_x_V"]) < 1e-7
