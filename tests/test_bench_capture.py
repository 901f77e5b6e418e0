"""The bench's roofline `traffic` comes from committed ncu captures (profiles/*.csv): CPU checks of
the parser's units and of the rule that a capture is used only for a launch of the same shape."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.fixture(scope="module")
def bench():
    import bench as b
    return b


def test_capture_units_and_shape(bench):
    cap = bench.ncu_capture("k_lnl_full_mixed_cfg2")
    assert cap is not None and "k_lnl_full_mixed" in cap["kernel"]
    # 3.32 MB read + 35 KB written, in bytes; duration in seconds
    assert 1e6 < cap["dram_bytes"] < 1e8
    assert 50e-6 < cap["duration_s"] < 1e-3
    tr, info = bench.capture_traffic("k_lnl_full_mixed_cfg2", "k_lnl_full_mixed", cap["grid"].replace(" ", ""),
                                     cap["block"].replace(" ", ""), 0.17)
    assert tr == cap["dram_bytes"] and info["traffic_capture_matches_launch"]
    # another grid (a different batch size or tiling): no traffic figure
    tr, info = bench.capture_traffic("k_lnl_full_mixed_cfg2", "k_lnl_full_mixed", "(4096,1,1)", "(256,1,1)", 0.17)
    assert tr is None and not info["traffic_capture_matches_launch"]
    tr, info = bench.capture_traffic("no_such_capture", "k", None, None, 1.0)
    assert tr is None


def test_streaming_capture_in_bytes(bench):
    cap = bench.ncu_capture("k_lnl_multi_cfg4")
    assert cap is not None and "k_lnl_multi" in cap["kernel"]
    assert cap["dram_bytes"] > 1e10 and 1e-3 < cap["duration_s"] < 1.0
