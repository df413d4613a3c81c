"""Host-side parts of the library, no GPU needed: exported C ABI, command
line parser, OBJ/MTL/AUX loader and EXR writer, checked against the
reference's own parser and loader (oracle/_ref) where that build exists."""
import ctypes
import os
import re
import struct

import numpy as np
import pytest

from gpuupbp_b200 import scenes, upbp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "upbp.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\*\s]+?\b(upbp_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = upbp.load_library()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert sorted(upbp.EXPORTS) == names


CLI_CASES = [
    [],
    ["-a", "upbp_all"],
    ["-a", "upbp+pp3d+bp2d", "-l", "12", "-r", "64x48"],
    ["-a", "upbp_bb1d+bp2d", "-pbt", "L", "-qbt", "S", "-pbc", "-0.5"],
    ["-r_alpha", "0.75", "-r_alpha_pp3d", "0.5", "-r_initial", "-0.02", "-r_initial_surf", "0.01"],
    ["-r_initial_bb1d", "-0.004", "-r_alpha_bb1d", "0.9", "-pcpi", "-2", "-i", "7"],
    ["-previous", "-sn", "0", "-ignorespec", "1", "-ioff", "5"],
    ["-compatible", "-t", "3", "-o", "out_name.exr"],
    ["-speconly", "-log", "-pcpi", "300"],
]


@pytest.mark.parametrize("extra", CLI_CASES)
def test_command_line_matches_reference(extra, scene_dir, oracle_available):
    path = scenes.write_workload("box_medium", scene_dir, tiny=True)
    args = ["-s", "-1", path, "-r", "16x16"] + extra
    c = upbp.parse_command_line(args)
    if not oracle_available:
        pytest.skip("oracle/_ref not built")
    import ref_cpu
    r = ref_cpu.RefRenderer(args, threads=1)
    ref = r.describe()
    r.close()
    assert c.algorithm_flags == ref["algorithm_flags"]
    assert c.iteration_count == ref["iteration_count"]
    assert [c.res_x, c.res_y] == ref["res"]
    assert c.max_path_length == ref["max_path_length"]
    assert c.min_path_length == ref["min_path_length"]
    assert c.path_count_per_iter == pytest.approx(ref["path_count_per_iter"])
    assert c.query_beam_type == ref["query_beam_type"] and c.photon_beam_type == ref["photon_beam_type"]
    mine_init = [c.surf_radius_initial, c.pp3d_radius_initial, c.pb2d_radius_initial, c.bb1d_radius_initial,
                 c.bp2d_radius_initial]
    mine_alpha = [c.surf_radius_alpha, c.pp3d_radius_alpha, c.pb2d_radius_alpha, c.bb1d_radius_alpha,
                  c.bp2d_radius_alpha]
    assert np.allclose(mine_init, ref["radius_initial"], rtol=1e-6)
    assert np.allclose(mine_alpha, ref["radius_alpha"], rtol=1e-6)
    assert c.bb1d_used_light_subpath_count == pytest.approx(ref["bb1d_used"])
    assert c.ignore_fully_spec_paths == ref["ignore_spec"]
    assert c.iteration_offset == ref["ioff"]
    assert c.use_shading_normal == ref["shading_normal"]
    assert c.output_name.decode() == ref["output_name"]


def test_command_line_errors():
    for bad in (["-l", "0"], ["-r", "10"], ["-a", "upbp_foo"], ["-s", "3"], ["-bogus"], ["-i"]):
        with pytest.raises(upbp.UpbpError):
            upbp.parse_command_line(bad)


@pytest.mark.parametrize("workload", ["box_medium", "media_field", "dense_beams"])
def test_scene_loader_matches_reference(workload, scene_dir, oracle_available):
    L = upbp.load_library()
    path = scenes.write_workload(workload, scene_dir, tiny=True)
    sc = ctypes.c_void_p()
    assert L.upbp_scene_load_obj(path.encode(), 40, 30, ctypes.byref(sc)) == 0
    d = L.upbp_scene_get_desc(sc).contents
    mats = d.tri_material[:d.triangle_count]
    reals = [d.materials[m].real for m in range(d.material_count)]
    n_real = sum(1 for i in range(d.triangle_count) if reals[mats[i]])
    info = dict(tris=d.triangle_count, real=n_real, lights=d.light_count, materials=d.material_count,
                media=d.medium_count, global_medium=d.global_medium, background=d.background_light,
                bmin=list(d.bbox_min), bmax=list(d.bbox_max), origin=list(d.camera.origin),
                fov=d.camera.horizontal_fov_deg, spheres=d.sphere_count)
    L.upbp_scene_free(sc)
    assert info["tris"] == scenes.WORKLOADS[workload](tiny=True).triangle_count() and info["spheres"] == 0
    if not oracle_available:
        pytest.skip("oracle/_ref not built")
    import ref_cpu
    r = ref_cpu.RefRenderer(["-s", "-1", path, "-r", "40x30"], threads=1)
    ref = r.describe()
    r.close()
    assert info["real"] == ref["tri_real"] and info["tris"] - info["real"] == ref["tri_imag"]
    assert info["lights"] == ref["lights"] and info["materials"] == ref["materials"]
    assert info["media"] == ref["media"] and info["global_medium"] == ref["global_medium"]
    assert info["background"] == ref["background"]
    assert np.allclose(info["origin"], ref["camera_origin"], atol=1e-6)
    center = (np.array(info["bmin"]) + np.array(info["bmax"])) * 0.5
    assert np.allclose(center, ref["scene_center"], atol=1e-6)
    radius = 0.5 * np.sqrt(np.sum((np.array(info["bmax"], np.float32) - np.array(info["bmin"], np.float32)) ** 2))
    assert radius == pytest.approx(ref["scene_radius"], rel=1e-6)
    ipd = 40 / (2 * np.tan(info["fov"] * np.pi / 360))
    assert ipd == pytest.approx(ref["image_plane_dist"], rel=1e-5)


def test_scene_loader_errors(tmp_path):
    L = upbp.load_library()
    sc = ctypes.c_void_p()
    assert L.upbp_scene_load_obj(str(tmp_path / "missing.obj").encode(), 8, 8, ctypes.byref(sc)) == -2
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nf 1 2 3\n")
    (tmp_path / "bad.obj.aux").write_text("")
    assert L.upbp_scene_load_obj(str(bad).encode(), 8, 8, ctypes.byref(sc)) == -5
    assert L.upbp_scene_load_predefined(41, 8, 8, ctypes.byref(sc)) == -1
    assert L.upbp_scene_load_predefined(0, 0, 8, ctypes.byref(sc)) == -1
    assert L.upbp_scene_load_predefined(0, 8, 8, ctypes.byref(sc)) == 0
    L.upbp_scene_free(sc)


def read_exr_half(path):
    """Minimal reader for the uncompressed scanline HALF files the writer emits."""
    data = open(path, "rb").read()
    assert struct.unpack_from("<II", data, 0) == (20000630, 2)
    pos, attrs = 8, {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        pos = end + 1
        end = data.index(b"\0", pos)
        typ = data[pos:end].decode()
        pos = end + 1
        (size,) = struct.unpack_from("<I", data, pos)
        pos += 4
        attrs[name] = (typ, data[pos:pos + size])
        pos += size
    pos += 1
    x0, y0, x1, y1 = struct.unpack_from("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack_from(f"<{h}Q", data, pos)
    img = np.zeros((h, w, 3), np.float16)
    for off in offsets:
        y, n = struct.unpack_from("<ii", data, off)
        row = np.frombuffer(data, np.float16, count=3 * w, offset=off + 8).reshape(3, w)
        img[y, :, 2], img[y, :, 1], img[y, :, 0] = row[0], row[1], row[2]  # B, G, R
    assert attrs["compression"][1] == b"\0"
    return img


def test_exr_writer_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    img = (rng.standard_normal((7, 9, 3)) * np.array([1.0, 100.0, 1e-5])).astype(np.float32)
    img[0, 0] = [70000.0, -0.0, 6e-8]  # overflow to inf, negative zero, subnormal
    p = tmp_path / "x.exr"
    upbp.write_exr(str(p), img)
    back = read_exr_half(str(p))
    expected = img.astype(np.float16)  # IEEE round to nearest even
    assert np.array_equal(back.view(np.uint16), expected.view(np.uint16))


def test_bmp_writer_bytes(tmp_path):
    """24-bit BMP as the reference's save_bmp writes it (framebuffer.cpp:129-202):
    "BM", its 52-byte header, rows bottom up, BGR of pow(c, 1/gamma) * 255
    clamped and truncated, no row padding."""
    rng = np.random.default_rng(4)
    h, w, gamma = 5, 6, 2.2
    img = (rng.random((h, w, 3)) * 1.3 - 0.1).astype(np.float32)
    p = tmp_path / "x.bmp"
    upbp.write_image(str(p), img, gamma)
    data = p.read_bytes()
    assert data[:2] == b"BM" and len(data) == 54 + w * h * 3
    fields = struct.unpack_from("<IIIIiihhIIIIII", data, 2)
    assert fields == (54 + w * h * 3, 0, 54, 40, w, h, 1, 24, 0, w * h * 3, 2953, 2953, 0, 0)
    with np.errstate(invalid="ignore"):
        v = np.power(img.astype(np.float32), np.float32(1.0 / gamma)) * np.float32(255.0)
    v = np.where(np.isnan(v), 0.0, np.clip(v, 0.0, 255.0)).astype(np.uint8)
    expected = v[::-1, :, ::-1].tobytes()
    got = np.frombuffer(data, np.uint8, offset=54)
    # pow in float32 may differ from numpy's in the last ulp: at most one
    # byte value apart, and almost always equal
    diff = np.abs(got.astype(int) - np.frombuffer(expected, np.uint8).astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() > 0.95


def test_hdr_writer_bytes(tmp_path):
    """Radiance RGBE as the reference's save_hdr writes it (framebuffer.cpp:204-233)."""
    rng = np.random.default_rng(5)
    h, w = 4, 3
    img = (rng.random((h, w, 3)) * 10.0).astype(np.float32)
    img[0, 0] = 0.0
    img[1, 1] = [1e-33, 0.0, 0.0]
    p = tmp_path / "x.hdr"
    upbp.write_image(str(p), img)
    data = p.read_bytes()
    head = b"#?RADIANCE\n# SmallUPBP\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n" % (h, w)
    assert data.startswith(head) and len(data) == len(head) + 4 * w * h
    px = np.frombuffer(data, np.uint8, offset=len(head)).reshape(h, w, 4)
    for y in range(h):
        for x in range(w):
            c = img[y, x]
            v = float(max(c))
            if v < 1e-32:
                assert (px[y, x] == 0).all()
                continue
            m, e = np.frexp(np.float32(v))
            s = np.float32(m * np.float32(256.0) / np.float32(v))
            assert list(px[y, x, :3]) == [int(np.float32(ch) * s) for ch in c]
            assert px[y, x, 3] == e + 128


def test_image_writer_refuses_unknown_extension(tmp_path):
    with pytest.raises(upbp.UpbpError):
        upbp.write_image(str(tmp_path / "x.png"), np.zeros((2, 2, 3), np.float32))


def test_checkpoint_flags_parse():
    """-checkpoint / -resume (not in the reference) fill the configuration's
    paths and leave the output name alone."""
    from gpuupbp_b200 import upbp
    c = upbp.parse_command_line(["-s", "2", "-checkpoint", "/tmp/a.ckpt", "-resume", "/tmp/b.ckpt"])
    assert c.checkpoint_path == b"/tmp/a.ckpt" and c.resume_path == b"/tmp/b.ckpt"
    assert b"ckpt" not in c.output_name
    with pytest.raises(Exception):
        upbp.parse_command_line(["-s", "2", "-resume"])
