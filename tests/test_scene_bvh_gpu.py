"""The static scene's BVH built on the device (upbp_scene_bvh.cuh) against
the sequential statement of the same build (oracle/sah_ref.cpp) on the same
triangles: every node's boxes, links and counts and the leaf order equal,
bit for bit (a zero's sign aside: the device's min/max atomics store +0
where the sequential min keeps -0, the same value).  Both classes of
triangles, on the box, the full 1.64M-triangle media field, the dense-beam
enclosure and a predefined scene with spheres."""
import os
import sys

import numpy as np
import pytest

from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

CASES = {
    "box_medium": ["-s", "-1", None, "-a", "upbp_all", "-l", "8", "-r", "16x16"],
    "media_field": ["-s", "-1", None, "-a", "upbp_all", "-l", "12", "-r", "16x9"],
    "dense_beams": ["-s", "-1", None, "-a", "upbp_all", "-l", "16", "-r", "16x9"],
    "predef_2": ["-s", "2", "-a", "upbp_all", "-l", "8", "-r", "16x16"],
}


@pytest.mark.parametrize("case", list(CASES))
def test_device_scene_bvh_equals_sequential_build(case, scene_dir):
    import ref_cpu
    from gpuupbp_b200 import upbp
    args = list(CASES[case])
    if None in args:
        args[args.index(None)] = scenes.write_workload(case, scene_dir)
    r = upbp.Renderer(args)
    compared = 0
    for real in (True, False):
        nodes, tris = r.scene_bvh(real)
        n = len(tris)
        if n == 0:
            continue
        orig = tris[:, 3].view(np.int32).copy()
        assert sorted(orig.tolist()) == list(range(n))
        by_orig = np.zeros_like(tris)
        by_orig[orig] = tris
        ref_nodes, ref_order, _ = ref_cpu.sah_build(by_orig)
        assert np.array_equal(orig, ref_order.astype(np.int32)), (case, real)
        if n > 1:
            assert np.array_equal(nodes[:, 12:16].view(np.int32), ref_nodes[:, 12:16].view(np.int32)), (case, real)
            assert np.array_equal(nodes[:, :12], ref_nodes[:, :12]), (case, real)  # as floats: -0 == +0
        compared += n
    st = r.stats()
    print(f"{case}: {compared} triangles, device build {st['ms_scene_bvh']:.1f} ms")
    r.close()
    assert compared > 0
