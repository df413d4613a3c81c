"""bench.py's host-side arithmetic on synthetic counters: per-kernel
algorithmic bytes (32-byte nodes for the range searches), the whole-iteration
roofline's record sizes, and the clock sampler's timed window."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from gpuupbp_b200.upbp import KERNELS, WORK_NAMES  # noqa: E402


def fake_stats():
    work = {k: {n: 0 for n in WORK_NAMES} for k in KERNELS}
    work["bb1d_query"].update(nodes=1000, beam_cand=100, beam_hit=10)
    work["light_pass"].update(nodes=500, tris=50, rays=5)
    return {"timed_iterations": 2, "ms_kernel_sum": {k: 2.0 for k in KERNELS}, "segment_queries": 7,
            "point_queries": 3, "nee_samples": 0, "bpt_pairs": 4, "work": work, "surface_vertices": 5,
            "medium_vertices": 6, "beam_chunks": 9, "light_vertices": 11, "light_beams": 2}


def test_kernel_rooflines_use_compressed_node_bytes():
    k = bench.kernel_rooflines(fake_stats(), pixels=100)
    bb = k["bb1d_query"]
    expect = 1000 * 32 + 100 * 48 + 10 * 128 + bench.SEG_RECORD * 7 + bench.HIT_RECORD * 2 * 10
    assert bb["bytes"] == expect and bb["ms"] == 1.0
    assert k["light_pass"]["bytes"] == 500 * 64 + 50 * 48 + 5 * 72


def test_iteration_bytes_follow_the_canonical_sizes():
    b = bench.iteration_bytes(fake_stats(), pixels=100)
    expect = (500 * 32 + 50 * 40) + 11 * 80 * 2 + 2 * 128 * 2 + 100 * 128 + 4 * 80 + (5 + 6 + 9) * 40 + 100 * 24
    assert b == expect


def test_clock_summary_counts_only_the_timed_window():
    c = bench.ClockSampler(0)
    t = 1_700_000_000.0

    def line(ts, mhz, cap):
        stamp = datetime.datetime.fromtimestamp(ts).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        return f"{stamp}, {mhz}, 1965, 500.0, Not Active, Not Active, Not Active, {'Active' if cap else 'Not Active'}"

    c.lines = [line(t - 10, 900, True), line(t + 0.1, 1965, False), line(t + 0.3, 1950, False), "garbage"]
    s = c.summary(t, t + 0.4)
    assert s == {"sm_mhz": 1957.5, "sm_max_mhz": 1965.0, "reasons": [], "samples": 2}
    assert c.summary()["samples"] == 3 and c.summary()["reasons"] == ["sw_power_cap"]


def test_relmse_and_reference_streams():
    """relMSE as defined, and the equal-time references render the same
    radius schedule on other random streams (-ioff shifts only those)."""
    import numpy as np

    from gpuupbp_b200 import quality
    ref = np.array([[[1.0, 0.0, 2.0]]])
    x = np.array([[[1.5, 0.1, 2.0]]])
    want = np.mean(np.array([0.25 / 1.01, 0.01 / 0.01, 0.0]))
    assert abs(quality.relmse(x, ref) - want) < 1e-12
    assert quality.relmse(ref, ref) == 0.0
    assert quality.REFERENCE_IOFF[0] == "-ioff" and int(quality.REFERENCE_IOFF[1]) > 100000
