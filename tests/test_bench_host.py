"""Host-side pieces of bench.py that need no GPU: the DRAM traffic and the
issue rate the roofline line reports, read from the ncu captures under
profiles/."""
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
        elif e["scale"] == "packets":
            # the captured launch is reproduced; the part beyond the fixed
            # first touch grows with the packets
            assert abs(bench.captured_traffic(e["workload"], 123, e["packets"]) - e["dram_bytes"]) < 1
            per = (e["dram_bytes"] - e["fixed_bytes"]) / e["packets"]
            assert 0 < per < 1000
            twice = bench.captured_traffic(e["workload"], 123, 2 * e["packets"])
            assert abs(twice - (2 * e["dram_bytes"] - e["fixed_bytes"])) < 2
        else:
            assert bench.captured_traffic(e["workload"], 123) == e["dram_bytes"]
    assert bench.captured_traffic("no_such_workload", 1) is None


def test_issue_rate_from_the_captured_instruction_count():
    """The issue figure beside the roofline: warp instructions per segment
    from the capture x segments / kernel time, against 4 warp instructions
    per cycle per SM at the sampled clock."""
    with open(os.path.join(ROOT, "profiles", "propagate_kernel_traffic.json")) as f:
        entries = json.load(f)
    e = next(t for t in entries if "warp_inst_per_segment" in t)
    wps = e["warp_inst_per_segment"]
    r = bench.captured_issue(e["workload"], 1e10, 1000.0, 2000.0, 100)
    assert abs(r["achieved"] - wps * 1e10) < 1e-3 * wps * 1e10
    assert r["peak"] == 4 * 100 * 2000e6
    assert abs(r["frac"] - wps * 1e10 / 8e11) < 1e-12
    assert bench.captured_issue(e["workload"], 1e10, 1000.0, None, 100) is None
    assert bench.captured_issue("no_such_workload", 1e10, 1000.0, 2000.0, 100) is None


def test_chi2_summary_of_two_spectra():
    """The matched-chi^2 figure bench.py reports: two independent spectra of
    the same equal-energy packet process give chi^2 / dof near 1 and a p-value
    that is not small; a 5% distortion of one of them is rejected."""
    import numpy as np
    rng = np.random.default_rng(7)
    lam = 2000.0 * np.exp(-np.linspace(0, 3, 400))
    ca, cb = rng.poisson(lam).astype(float), rng.poisson(lam).astype(float)
    fa, fb = 3.0 * ca, 3.0 * cb
    same = bench.chi2_summary(fa, ca, fb, cb)
    assert same["dof"] == int(((ca >= 10) & (cb >= 10)).sum())
    assert 0.8 < same["chi2_per_dof"] < 1.2 and same["p_value"] > 0.01
    bent = bench.chi2_summary(fa * (1 + 0.05 * np.sin(np.arange(400))), ca, fb, cb)
    assert bent["p_value"] < 1e-6
    assert bench.chi2_summary(fa, 0 * ca, fb, cb) == {"chi2_per_dof": None, "dof": 0, "p_value": None}
