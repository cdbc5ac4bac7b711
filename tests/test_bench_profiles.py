"""The figures bench.py reads from the committed ncu summaries under profiles/ (CPU only).

The roofline entries of the bench lines divide live CUDA-event timings by figures measured once with ncu and
committed as text (instructions per move, DRAM bytes per launch, measured peaks). A summary rewritten without one
of its `key: value` lines would silently turn a roofline into null, so each figure is checked here: present,
parsed and in a plausible range.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402

FIGURES = [
    # (summary, key, low, high)
    ("k_descent_plain", "warp_inst_per_move_per_block", 500, 5000),
    ("k_descent_plain", "dram_bytes_per_launch", 1e5, 1e8),
    ("k_descent_neighborhood", "warp_inst_per_move_per_block", 1000, 20000),
    ("k_descent_neighborhood", "dram_bytes_per_launch", 1e5, 1e9),
    ("k_descent_wide2_sparse_n65536", "warp_inst_per_move_per_block", 1000, 100000),
    ("k_descent_large", "dram_bytes_per_launch", 1e6, 1e11),
    ("k_rebuild_tensor_n32768", "dram_bytes_per_launch", 1e7, 1e10),
    ("peaks_l2_hbm_int8", "l2_copy_gbs", 5000, 30000),
    ("peaks_l2_hbm_int8", "hbm_copy_gbs", 3000, 10000),
    ("peaks_l2_hbm_int8", "int8_tops", 1000, 10000),
]


@pytest.mark.parametrize("name,key,low,high", FIGURES, ids=[f"{n}:{k}" for n, k, _, _ in FIGURES])
def test_profile_figure_present(name, key, low, high):
    value = bench.profiled_value(name, key)
    assert value is not None, f"profiles/{name}.txt has no '{key}:' line"
    assert low <= value <= high, (name, key, value)


def test_hbm_peak_falls_back_to_the_committed_measurement():
    value, kind = bench.measured_peak_hbm()
    if os.path.exists(os.path.join(REPO, "MEASURED_PEAKS.json")):
        assert kind == "measured"
    else:
        assert kind.startswith("measured (profiles/") and value == bench.profiled_value("peaks_l2_hbm_int8",
                                                                                          "hbm_copy_gbs")
