"""Pins the oracle: the reference's render loop compiled for the CPU must
reproduce the committed golden images, the PCG32 restatement must match the
published PCG32 known-answer sequence, and the brute-force neighbour
predicates must agree with hand-computed cases."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import neighbors
from cases import CASES, command_line
from gpuupbp_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def frac_close(a, b, rel=1e-4):
    r = np.abs(a - b) / (np.abs(b) + 1e-3)
    return float(np.mean(np.all(r < rel, axis=-1)))


@pytest.mark.parametrize("case", ["box_tiny_all", "box_all_bp2d", "media_field_tiny", "dense_beams_tiny"])
def test_oracle_reproduces_golden(case, scene_dir, oracle_available):
    if not oracle_available:
        pytest.skip("oracle/_ref not built")
    import ref_cpu
    gold = np.load(os.path.join(GOLDEN, "oracle_images.npz"))
    counts = json.load(open(os.path.join(GOLDEN, "oracle_counts.json")))
    workload, tiny, _, iters = CASES[case]
    path = scenes.write_workload(workload, scene_dir, tiny=tiny)
    r = ref_cpu.RefRenderer(command_line(case, path), threads=0)
    for it in range(iters):
        img = r.run_iteration(it)
        st = r.stats()
        assert {k: st[k] for k in ("vertices", "surface", "medium", "beams")} == counts[case][it]
        # multithreaded float atomics change only the summation order
        assert frac_close(img, gold[f"{case}/{it}"]) > 0.999
    r.close()
    assert ref_cpu.RefRenderer.exception_counts()[0] == 0  # no failed GPU_ASSERT in the reference code


PCG_KAT = [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]


def test_pcg32_known_answer():
    src = r'''
#include <stdio.h>
#include "pcg32_ref.h"
int main(void) {
    upbp_oracle_pcg32 r; r.state = 0u; r.inc = (54u << 1u) | 1u;
    upbp_oracle_pcg32_next(&r); r.state += 42u; upbp_oracle_pcg32_next(&r);
    for (int i = 0; i < 6; i++) printf("%u\n", upbp_oracle_pcg32_next(&r));
    upbp_oracle_pcg32_init(&r, 7u, 5u, 1u);
    printf("%.9g\n", upbp_oracle_pcg32_uniform(&r));
    return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "kat.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "kat")
        subprocess.run(["gcc", "-O1", "-I", os.path.join(ROOT, "oracle"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert [int(x) for x in out[:6]] == PCG_KAT
    # Python restatement of the seeded stream used by both renderers
    u = float(out[6])
    assert u == pytest.approx(python_stream(7, 5, 1)[0], abs=0)


def python_stream(iteration, path, pass_, n=1):
    M = (1 << 64) - 1

    def splitmix(x):
        x = (x + 0x9E3779B97F4A7C15) & M
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
        return x ^ (x >> 31)

    state, inc = 0, ((((path << 1) | pass_) << 1) | 1) & M

    def nxt():
        nonlocal state
        old = state
        state = (old * 6364136223846793005 + inc) & M
        xs = (((old >> 18) ^ old) >> 27) & 0xffffffff
        rot = old >> 59
        return ((xs >> rot) | (xs << ((-rot) & 31))) & 0xffffffff

    nxt()
    state = (state + splitmix(iteration)) & M
    nxt()
    return [np.float32(nxt() >> 8) * np.float32(1.0 / 16777216.0) for _ in range(n)]


def test_neighbor_predicates_hand_cases():
    pts = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [0.5, 0.5, 0, 0], [3, 0, 0, 0]], np.float32)
    # inclusive radius: |x-p|^2 <= r^2
    assert list(neighbors.points_in_radius(pts, [0, 0, 0], 1.0)) == [0, 1, 2]
    assert list(neighbors.points_in_radius(pts, [0, 0, 0], 0.999)) == [0, 2]
    # disc crossing: t strictly inside (tmin, tmax), radius inclusive
    q = [-1, 0.5, 0, 1, 0, 0, 0.0, 2.0]  # point 1 projects to t = 2 = tmax: excluded
    assert list(neighbors.points_near_segment(pts, q, 0.25)) == [0, 2]
    q = [-1, 0.5, 0, 1, 0, 0, 1.0, 2.5]  # point 0 projects to t = 1 = tmin: excluded
    assert list(neighbors.points_near_segment(pts, q, 0.25)) == [1, 2]
    s = np.float32(0.70710677)
    beams = np.array([[-s, -s, 0, 2, s, s, 0, 0], [5 - s, -s, 0, 2, s, s, 0, 0], [-s, -s, 0.05, 2, s, s, 0, 0]],
                     np.float32)
    beams[:, 7] = np.array([0, 1, 7], np.uint32).view(np.float32)
    q = [-1, 0, 0, 1, 0, 0, 0.0, 3.0]
    assert list(neighbors.beams_near_segment(beams, q, 0.01)) == [0, 2]
    assert list(neighbors.beams_near_segment(beams, q, 0.01, path_limit=5)) == [0]
    parallel = np.array([[0, 0, 0, 1, 1, 0, 0, 0]], np.float32)
    assert list(neighbors.beams_near_segment(parallel, q, 1.0)) == []
    # the reference's closest-point formula divides by d1.d2: exactly
    # perpendicular beams are never reported (intersection.cuh:162)
    perpendicular = np.array([[0, -1, 0, 2, 0, 1, 0, 0]], np.float32)
    assert list(neighbors.beams_near_segment(perpendicular, q, 0.01)) == []
    assert list(neighbors.beams_near_point(beams, [0.1, 0.1, 0.01], 0.0004)) == [0]
