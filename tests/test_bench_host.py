"""Host-side pieces of bench.py that need no GPU: the DRAM traffic the
roofline line reports, read from the ncu captures under profiles/."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_every_bench_workload_with_a_capture_reports_traffic():
    with open(os.path.join(ROOT, "profiles", "propagate_kernel_traffic.json")) as f:
        entries = json.load(f)
    names = {e["workload"] for e in entries}
    assert {"type_ia_1d", "cart3d", "batch64_1d"} <= names
    for e in entries:
        assert e["dram_bytes"] == e["dram_read_bytes"] + e["dram_write_bytes"]
        assert "--clock-control none" in e["command"]
        if e["scale"] == "segments":
            # the captured launch itself is reproduced, and twice the segments twice the bytes
            assert abs(bench.captured_traffic(e["workload"], e["segments"]) - e["dram_bytes"]) < 1
            assert abs(bench.captured_traffic(e["workload"], 2 * e["segments"]) - 2 * e["dram_bytes"]) < 2
        else:
            assert bench.captured_traffic(e["workload"], 123) == e["dram_bytes"]
    assert bench.captured_traffic("no_such_workload", 1) is None
