"""Host binned-SAH build of the scene BVH (gpuupbp_b200/csrc/host/upbp_sah.cpp),
compiled on its own with g++ and checked on random boxes: every primitive in
exactly one leaf, every stored child box containing the boxes of its
subtree, node slots as documented (a subtree of m primitives in m - 1
consecutive slots), depth within the device walks' stack."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "gpuupbp_b200", "csrc", "host", "upbp_sah.cpp")

HARNESS = r"""
#include <cstdio>
#include <vector>
#include "upbp_sah.h"
int main(int argc, char** argv) {
    FILE* f = fopen(argv[1], "rb");
    unsigned n; if (fread(&n, 4, 1, f) != 1) return 2;
    std::vector<float> boxes(6 * (size_t)n);
    if (fread(boxes.data(), 4, boxes.size(), f) != boxes.size()) return 2;
    fclose(f);
    std::vector<float> nodes(16 * (size_t)(n - 1));
    std::vector<unsigned> order(n);
    upbp_host::sah_build(boxes.data(), n, nodes.data(), order.data(), 4);
    FILE* o = fopen(argv[2], "wb");
    fwrite(nodes.data(), 4, nodes.size(), o);
    fwrite(order.data(), 4, order.size(), o);
    fclose(o);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("sah")
    (d / "main.cpp").write_text(HARNESS)
    exe = d / "sah"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.dirname(SRC), str(d / "main.cpp"), SRC,
                    "-o", str(exe)], check=True)
    return d, exe


def run(harness, boxes):
    d, exe = harness
    n = len(boxes)
    with open(d / "in.bin", "wb") as f:
        f.write(np.uint32(n).tobytes())
        f.write(boxes.astype(np.float32).tobytes())
    subprocess.run([str(exe), str(d / "in.bin"), str(d / "out.bin")], check=True)
    raw = np.fromfile(d / "out.bin", dtype=np.uint8)
    nodes = raw[: 64 * (n - 1)].view(np.float32).reshape(n - 1, 16)
    links = raw[: 64 * (n - 1)].view(np.int32).reshape(n - 1, 16)[:, 12:16]
    order = raw[64 * (n - 1):].view(np.uint32)
    return nodes, links, order


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
def test_sah_tree_is_valid(harness, n, seed):
    rng = np.random.default_rng(seed)
    c = rng.random((n, 3)) * 10
    ext = rng.random((n, 3)) * 0.2
    boxes = np.concatenate([c - ext, c + ext], axis=1).astype(np.float32)
    nodes, links, order = run(harness, boxes)
    check_tree(boxes, nodes, links, order)


def test_sah_tolerates_nan_boxes(harness):
    """A NaN box (a malformed vertex) still lands in exactly one leaf."""
    rng = np.random.default_rng(5)
    n = 200
    c = rng.random((n, 3)) * 4
    boxes = np.concatenate([c - 0.05, c + 0.05], axis=1).astype(np.float32)
    boxes[[3, 77]] = np.nan
    nodes, links, order = run(harness, boxes)
    assert sorted(order.tolist()) == list(range(n))


def test_sah_coincident_centroids(harness):
    """All centroids equal: the builder falls back to middle splits."""
    n = 300
    boxes = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (n, 1))
    nodes, links, order = run(harness, boxes)
    assert check_tree(boxes, nodes, links, order) <= 10
