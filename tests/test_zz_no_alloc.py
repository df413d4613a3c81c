"""upbp_debug_query_static: the neighbour-set query for callers that cannot
allocate device memory on every call (an application that hands the renderer
a fixed device-memory budget, or one whose other streams must not wait on the
device-wide synchronisation that freeing device memory implies).  It stages
its data in one static device array instead of per-call allocations.

Checked through the C ABI against upbp_debug_query on the same queries, two
calls in a row (the static array keeps the previous call's contents, so the
second call shows that nothing stale leaks into its results).  Neighbour sets
are integer results: they must be equal exactly.  Neither query may change
the last iteration's work counters.  The file is named to be
collected last; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu

KINDS = {0: "SURF", 1: "PP3D", 2: "PB2D", 3: "BB1D", 4: "BP2D"}
CAP = 256  # ids per query, the static variant's maximum


def _queries(r, rng, kind, n):
    surf, med, beams = r.photons(0), r.photons(1), r.photons(2)
    q = np.zeros((n, 8), np.float32)
    if kind in (0, 1):
        pts = surf if kind == 0 else med
        q[:, :3] = pts[rng.integers(0, len(pts), n), :3] + rng.normal(size=(n, 3)).astype(np.float32) * 0.01
        return q
    if kind == 2:
        c = med[rng.integers(0, len(med), n), :3]
    else:
        b = beams[rng.integers(0, len(beams), n)]
        c = b[:, :3] + b[:, 4:7] * (rng.uniform(0, 1, n).astype(np.float32) * b[:, 3])[:, None]
    if kind == 4:
        q[:, :3] = c + rng.normal(size=(n, 3)).astype(np.float32) * 0.01
        return q
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q[:, :3] = c - d * 0.3
    q[:, 3:6] = d
    q[:, 6] = 0.0
    q[:, 7] = 0.6
    return q


def _call(fn, ctx, kind, q):
    n = len(q)
    counts = np.full(n, 0xDEADBEEF, np.uint32)
    ids = np.full((n, CAP), 0xDEADBEEF, np.uint32)
    rc = fn(ctx, kind, q.ctypes.data, n, counts.ctypes.data, ids.ctypes.data, CAP)
    assert rc == 0
    return counts, ids


def test_static_scratch_query_matches_allocating_query(tmp_path):
    from gpuupbp_b200 import upbp
    L = upbp.load_library()
    path = scenes.write_workload("box_medium", str(tmp_path))
    r = upbp.Renderer(["-s", "-1", path, "-a", "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d", "-l", "8", "-r", "64x64",
                       "-r_initial", "-0.02"])
    r.run_iteration(0)
    work_before = r.stats()["work"]
    rng = np.random.default_rng(5)
    for kind in KINDS:
        for call in range(2):
            q = _queries(r, rng, kind, 1000 + 300 * call)
            want_c, want_i = _call(L.upbp_debug_query, r._ctx, kind, q)
            got_c, got_i = _call(L.upbp_debug_query_static, r._ctx, kind, q)
            assert np.array_equal(got_c, want_c), KINDS[kind]
            assert want_c.max() <= CAP
            assert want_c.sum() > 0, KINDS[kind]
            for i, c in enumerate(want_c):
                assert np.array_equal(np.sort(got_i[i, :c]), np.sort(want_i[i, :c]))
                assert not got_i[i, c:].any()  # slots beyond the count are cleared
    # the queries count their work in a row of their own: the iteration's
    # work counters read the same after them
    assert r.stats()["work"] == work_before
    # sizes beyond the static array are refused, not truncated
    q = np.zeros((4097, 8), np.float32)
    counts = np.zeros(4097, np.uint32)
    ids = np.zeros((4097, 1), np.uint32)
    assert L.upbp_debug_query_static(r._ctx, 0, q.ctypes.data, 4097, counts.ctypes.data, ids.ctypes.data, 1) == -1
    q = np.zeros((4, 8), np.float32)
    assert L.upbp_debug_query_static(r._ctx, 0, q.ctypes.data, 4, counts.ctypes.data, ids.ctypes.data, 257) == -1
    r.close()
