"""The roofline block of bench.py's JSON line, on the CPU (no kernel runs).

achieved = 48 B x particles + 44 B x cells over the kernel's time; traffic and the
instruction counters come from the committed ncu capture of that kernel on that
workload, scaled to the launch, and are left out (null) for a workload without one.
"""
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_roofline_from_capture():
    import bench
    n, cells, ms = 536_870_912, 4096 * 1024, 11.5
    r = bench.roofline(n, cells, ms, "k_slot", "k_slot_traffic.json")
    alg = 48.0 * n + 44.0 * cells
    assert r["alg_bytes_per_launch"] == alg
    assert r["achieved"] == pytest.approx(alg / (ms / 1e3) / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    with open(os.path.join(ROOT, "profiles", "k_slot_traffic.json")) as f:
        t = json.load(f)
    assert r["traffic"] == pytest.approx(t["dram_bytes_per_particle"] * n)
    assert r["warp_inst_per_particle"] == t["warp_inst_per_particle"]
    assert r["counters_from"] == t["source"]


def test_roofline_without_capture_has_no_traffic():
    import bench
    r = bench.roofline(1_073_741_824, 8192 * 2048, 39.0, "k_slot", None)
    assert r["traffic"] is None and r["warp_inst_per_particle"] is None and r["counters_from"] is None
    assert r["frac"] > 0


@pytest.mark.parametrize("name", ["k_slot_traffic.json", "k_slot_batch_traffic.json"])
def test_traffic_files_name_their_capture(name):
    with open(os.path.join(ROOT, "profiles", name)) as f:
        t = json.load(f)
    assert os.path.exists(os.path.join(ROOT, t["source"]))
    # DRAM bytes per particle at least the 48 algorithmic bytes, lane efficiency a fraction
    assert t["dram_bytes_per_particle"] >= 48.0 and 0.0 < t["lane_efficiency"] <= 1.0
