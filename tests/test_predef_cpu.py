"""The predefined Cornell-box scenes (-s 0..40) as the library builds them,
compared record by record with the scenes the reference's own loader
(gpuupbp/misc/scene_loader_predef.cpp, compiled for the CPU in oracle/_ref)
builds: triangle vertices and face normals, sphere boxes, (material, light)
records, materials, media, lights, global medium and background light.
Bit-exact except the directional light's frame, which the reference stores
normalised."""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# scenes the reference's command line refuses (config.cpp:835-838)
REFUSED = (3, 4, 9, 10)
RENDERABLE = [s for s in range(41) if s not in REFUSED]


def f32(x):
    return np.asarray(x, np.float32)


def same(a, b):
    return np.array_equal(f32(a), f32(b))


@pytest.fixture(scope="module")
def libs(oracle_available):
    if not oracle_available:
        pytest.skip("oracle/_ref not built")
    from gpuupbp_b200 import upbp
    try:
        upbp.load_library()
    except upbp.UpbpError:
        pytest.skip("libupbp_b200.so not built")
    import ref_cpu
    return upbp, ref_cpu


@pytest.mark.parametrize("sid", RENDERABLE)
def test_predefined_scene_matches_reference_loader(sid, libs):
    upbp, ref_cpu = libs
    args = ["-s", str(sid), "-r", "32x32", "-i", "1"]
    r = ref_cpu.RefRenderer(args)
    ref = r.scene()
    r.close()
    me = upbp.load_scene(args)

    # triangles: the reference's real list then its imaginary list
    tris = ref["tri_real"] + ref["tri_imag"]
    assert len(tris) == len(me["tri_material"])
    for i, t in enumerate(tris):
        assert same(t[:3], me["verts"][i]), i
        assert all(same(t[3], me["normals"][i][k]) for k in range(4)), i
        assert t[4] == [int(me["tri_material"][i]), int(me["tri_light"][i])], i
    # spheres: the reference keeps a box per sphere
    sphs = ref["sph_real"] + ref["sph_imag"]
    assert len(sphs) == len(me["sph_material"])
    for i, s in enumerate(sphs):
        c, rad = f32(me["spheres"][i, :3]), f32(me["spheres"][i, 3])
        assert same(s[0], c - rad) and same(s[1], c + rad), i
        assert s[2] == [int(me["sph_material"][i]), -1], i

    assert len(ref["materials"]) == len(me["materials"])
    for a, b in zip(ref["materials"], me["materials"]):
        mine = [b["diffuse"], b["phong"], b["phong_exponent"], b["mirror"], b["ior"], b["priority"], b["real"],
                b["medium"]]
        assert all(same(x, y) for x, y in zip(a, mine)), (a, mine)
    assert len(ref["media"]) == len(me["media"])
    for a, b in zip(ref["media"], me["media"]):
        mine = [b["absorption"], b["emission"], b["scattering"], b["continuation_prob"], b["mean_cosine"]]
        assert all(same(x, y) for x, y in zip(a, mine)), (a, mine)

    assert len(ref["lights"]) == len(me["lights"])
    for a, b in zip(ref["lights"], me["lights"]):
        assert a[0] == b["type"] and a[1] == b["mat_id"] and a[2] == b["med_id"]
        if a[0] == 0:    # area: p0, e1, e2, intensity
            p0 = f32(b["p0"])
            assert same(a[3], p0) and same(a[4], f32(b["p1"]) - p0) and same(a[5], f32(b["p2"]) - p0)
            assert same(a[6], b["intensity"])
        elif a[0] == 1:  # background: colour, scale
            assert same(a[3], b["intensity"]) and a[4] == b["scale"]
        elif a[0] == 2:  # directional: frame z (normalised direction), intensity
            d = f32(b["position"])
            assert np.allclose(f32(a[3]), d / np.sqrt((d * d).sum()), atol=1e-6)
            assert same(a[4], b["intensity"])
        else:            # point: position, intensity
            assert same(a[3], b["position"]) and same(a[4], b["intensity"])
    assert ref["global_medium"] == me["global_medium"]
    assert ref["background"] == me["background_light"]

    # the scene sphere (scene_loader.hpp:60-66) from the bounding box; an
    # empty box (no geometry) gives radius 1/2
    ext = me["bbox_max"] - me["bbox_min"]
    with np.errstate(over="ignore"):
        r2 = np.float32(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2])
    if r2 == 0 or r2 > 1e36:
        r2 = np.float32(1)
    assert np.isclose(np.sqrt(r2) * np.float32(.5), ref["scene_radius"], rtol=1e-6)
    assert np.allclose((me["bbox_max"] + me["bbox_min"]) * np.float32(.5), ref["scene_center"], atol=1e-6)


def test_predefined_scene_ids(libs):
    upbp, _ = libs
    L = upbp.load_library()
    sc = ctypes.c_void_p()
    for bad in (-1, 41, 1000):
        assert L.upbp_scene_load_predefined(bad, 32, 32, ctypes.byref(sc)) == -1  # UPBP_ERR_ARGS
    # the library builds the scenes the command line refuses; the command line
    # refuses them as the reference's does
    for sid in REFUSED:
        assert L.upbp_scene_load_predefined(sid, 32, 32, ctypes.byref(sc)) == 0
        L.upbp_scene_free(sc)
        with pytest.raises(upbp.UpbpError):
            upbp.parse_command_line(["-s", str(sid)])
    # scene 10 has no light at all
    assert L.upbp_scene_load_predefined(10, 32, 32, ctypes.byref(sc)) == 0
    assert L.upbp_scene_get_desc(sc).contents.light_count == 0
    L.upbp_scene_free(sc)
