"""The sequential statement of the device's scene BVH build
(oracle/sah_ref.cpp, the checker the GPU build is compared with bit for bit
in tests/test_scene_bvh_gpu.py), on random triangles: every primitive in
exactly one leaf, every stored child box containing the boxes of its
subtree, node slots as documented (a subtree of m primitives in m - 1
consecutive slots), depth within the device walks' stack."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


@pytest.fixture(scope="module")
def sah():
    import ref_cpu
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "sah", "-s"], check=True)
    return ref_cpu.sah_build


def triangles(centres, size, rng):
    """Triangle records (v0, e1, e2 as float4s) around the given centres."""
    n = len(centres)
    v = centres[:, None, :] + (rng.random((n, 3, 3)) - 0.5) * size
    tri = np.zeros((n, 12), np.float32)
    tri[:, 0:3] = v[:, 0]
    tri[:, 4:7] = (v[:, 1].astype(np.float32) - v[:, 0].astype(np.float32))
    tri[:, 8:11] = (v[:, 2].astype(np.float32) - v[:, 0].astype(np.float32))
    return tri


def run(sah, tri):
    nodes, order, boxes = sah(tri)
    links = nodes.view(np.int32)[:, 12:16] if len(nodes) else np.zeros((0, 4), np.int32)
    return nodes, links, order, boxes


def check_tree(boxes, nodes, links, order):
    n = len(boxes)
    assert sorted(order.tolist()) == list(range(n))
    seen = np.zeros(n, bool)
    max_depth = 0

    def subtree(link, slot_lo, depth):
        nonlocal max_depth
        max_depth = max(max_depth, depth)
        if link < 0:
            pos = ~link
            assert not seen[pos]
            seen[pos] = True
            b = boxes[order[pos]]
            return b[:3].copy(), b[3:].copy(), 1
        assert link == slot_lo, (link, slot_lo)
        lo_l, hi_l, m_l = subtree(links[link, 0], link + 1, depth + 1)
        lo_r, hi_r, m_r = subtree(links[link, 1], link + m_l, depth + 1)
        assert (links[link, 2], links[link, 3]) == (m_l, m_r)
        nd = nodes[link]
        assert np.all(nd[0:3] <= lo_l) and np.all(nd[3:6] >= hi_l)
        assert np.all(nd[6:9] <= lo_r) and np.all(nd[9:12] >= hi_r)
        return np.minimum(lo_l, lo_r), np.maximum(hi_l, hi_r), m_l + m_r

    _, _, m = subtree(0, 0, 0)
    assert m == n and seen.all()
    assert max_depth < 64
    return max_depth


@pytest.mark.parametrize("n,seed", [(2, 0), (3, 1), (17, 2), (1000, 3), (20000, 4)])
def test_sah_tree_is_valid(sah, n, seed):
    rng = np.random.default_rng(seed)
    tri = triangles(rng.random((n, 3)) * 10, 0.4, rng)
    nodes, links, order, boxes = run(sah, tri)
    check_tree(boxes, nodes, links, order)


def test_sah_tolerates_nan_triangles(sah):
    """A NaN vertex (a malformed triangle) still lands in exactly one leaf."""
    rng = np.random.default_rng(5)
    n = 200
    tri = triangles(rng.random((n, 3)) * 4, 0.1, rng)
    tri[[3, 77], 0] = np.nan
    nodes, links, order, boxes = run(sah, tri)
    assert sorted(order.tolist()) == list(range(n))


def test_sah_coincident_centroids(sah):
    """All centroids equal: the builder falls back to middle splits."""
    n = 300
    tri = np.tile(np.array([[0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0]], np.float32), (n, 1))
    nodes, links, order, boxes = run(sah, tri)
    assert check_tree(boxes, nodes, links, order) <= 10
    # the middle split of a stable order keeps the input order
    assert order.tolist() == list(range(n))
