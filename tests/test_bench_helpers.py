"""Host-side arithmetic of bench.py that needs no GPU: the algorithmic byte counts the roofline figures
use, and the parsing of the autotuner report for the tensor-pipe figure."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_sap_sweep_bytes_256():
    g = bench.level_geoms()[1]  # 64x64 coarse sites, dof 24
    assert (g["sites"], g["dof"]) == (4096, 24)
    # links of the colour once (2048 sites x 5 x 24^2 x 16 B) + r, x read and x written per vector
    assert bench.sap_sweep_bytes(g, 8) == 2048 * 5 * 576 * 16 + 3 * 2048 * 24 * 16
    assert bench.sap_sweep_bytes(g, 8, 12) == 2048 * 5 * 576 * 16 + 12 * 3 * 2048 * 24 * 16


def test_sap_l2_bytes_256():
    # 128 blocks per colour x 31 applications x 64 in-block link matrices (4x4 block) x 24^2 x 16 B
    assert bench.sap_l2_bytes(1) == 128 * 31 * 64 * 576 * 16


def test_tensor_figure_parses_the_chosen_shape():
    rep = ("level 1 rhs 64 fp32 CUDA-core sweep: [rhs/cta 1: 900 us *]\n"
           "level 1 rhs 64: [rhs/cta 16 stages 3 chains 1: 223.1 us] [rhs/cta 64 stages 3 chains 2: 71.5 us *]\n")
    t = bench.tensor_figure(rep, 1, 64, 4.0e9)
    assert t["tile"] == {"rhs_per_cta": 64, "ring_stages": 3, "chains": 2}
    assert abs(t["achieved_tflops"] - 4.0e9 / 71.5e-6 / 1e12) < 1e-9
    assert 0 < t["frac"] < 1
    assert bench.tensor_figure("level 2 rhs 64: [rhs/cta 16 stages 3 chains 1: 1 us *]", 1, 64, 1.0) is None
