"""The run metadata file (writeMetadata, src/io.cpp:72-145) against the reference's own output
(tests/golden/metadata_16x32_l3.npz, made by tests/golden/make_golden.py): every line but the
date agrees byte for byte.  Host only: no device is touched."""
import os

import numpy as np

import ddamg

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    return np.load(os.path.join(HERE, "golden", "metadata_16x32_l3.npz"))


def _params(d):
    return ddamg.default_params(int(d["Nx"]), int(d["Nt"]), int(d["levels"]), float(d["m0"]),
                                [list(map(int, r)) for r in d["rows"]])


def _lines(text):
    return [ln for ln in text.splitlines() if not ln.startswith("Date: ")]


def test_metadata_matches_reference(tmp_path, monkeypatch):
    d = _golden()
    monkeypatch.setenv("HOSTNAME", "golden-host")
    for cyc in (0, 1):
        ref = bytes(d[f"ref_metadata_{cyc}"]).decode()
        path = str(tmp_path / f"meta{cyc}.dat")
        ddamg.write_metadata(_params(d), d[f"metadata_counts_{cyc}"], cyc, float(d[f"metadata_tol_{cyc}"]), path)
        ours = open(path).read()
        assert _lines(ours) == _lines(ref)
        assert ours.endswith("\n") and ref.endswith("\n")
        assert any(ln.startswith("Date: 20") for ln in ours.splitlines())


def test_metadata_default_name(tmp_path, monkeypatch):
    d = _golden()
    monkeypatch.chdir(tmp_path)
    ddamg.write_metadata(_params(d), [-1] * 7, 1, 1e-10)
    assert os.path.exists(tmp_path / "metadata_16x32_Levels3_Kcycle.dat")


def test_metadata_errors(tmp_path):
    d = _golden()
    p = _params(d)
    try:
        ddamg.write_metadata(p, [-1] * 7, 2, 1e-10, str(tmp_path / "x.dat"))
        raise AssertionError("cycle 2 accepted")
    except ddamg.DDAMGError as e:
        assert e.status == ddamg._lib.ERR_BAD_PARAM
    try:
        ddamg.write_metadata(p, [-1] * 7, 0, 1e-10, str(tmp_path / "no_such_dir" / "x.dat"))
        raise AssertionError("unwritable path accepted")
    except ddamg.DDAMGError as e:
        assert e.status == ddamg._lib.ERR_IO
