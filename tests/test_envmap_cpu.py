"""Environment-map background lights (light_background_em): the image the
library loads -- OpenEXR decoding, the scale and the rotation by a fraction
of a turn -- equals, bit for bit, the image the reference's loader hands to
its renderer (tinyexr LoadEXR + tinyexr_wrapper::load_image, compiled for
the CPU in oracle/_ref), for files that tinyexr's own encoder writes with
HALF and FLOAT channels and NONE, RLE, ZIPS and ZIP compression."""
import os
import sys

import numpy as np
import pytest

from gpuupbp_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


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


def both_images(upbp, ref_cpu, args):
    me = upbp.load_scene(args)
    r = ref_cpu.RefRenderer(args)
    ref = r.scene()
    r.close()
    w, h, px = ref["env"]
    return me, ref, np.array(px, np.float32).reshape(h, w, 3)


def test_env_workload_matches_reference_loader(libs, tmp_path):
    upbp, ref_cpu = libs
    path = scenes.write_workload("media_field_env", str(tmp_path), tiny=True)
    me, ref, img = both_images(upbp, ref_cpu, ["-s", "-1", path, "-r", "32x18"])
    assert me["env"] is not None and me["env"].shape == img.shape == (32, 64, 3)
    assert np.array_equal(me["env"], img)
    assert me["background_light"] == ref["background"] >= 0


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("compression", [0, 1, 2, 3])
def test_exr_decoding_matches_tinyexr(libs, tmp_path, half, compression):
    upbp, ref_cpu = libs
    path = scenes.write_workload("media_field_env", str(tmp_path), tiny=True)
    rng = np.random.default_rng(compression + 4 * half)
    img = (rng.random((24, 48, 3)) * 5).astype(np.float32)
    img[3, 5] = [1e-6, 60000.0, 0.0]   # a half subnormal and a large half
    img[7, 40] = [0.0, -2.5, 1e-30]
    exr = tmp_path / f"probe_{int(half)}_{compression}.exr"
    ref_cpu.save_exr(str(exr), img, half, compression)
    aux = [ln for ln in open(path + ".aux").read().splitlines() if not ln.startswith("light_background_em")]
    aux.append(f"light_background_em 1.5 0.5 {exr.name}")
    open(path + ".aux", "w").write("\n".join(aux) + "\n")
    me, _, ref_img = both_images(upbp, ref_cpu, ["-s", "-1", path, "-r", "32x18"])
    assert np.array_equal(me["env"], ref_img)


def test_env_errors(libs, tmp_path):
    upbp, _ = libs
    path = scenes.write_workload("media_field_env", str(tmp_path), tiny=True)
    aux = [ln for ln in open(path + ".aux").read().splitlines() if not ln.startswith("light_background_em")]
    for line, code in (("light_background_em 1 0 missing.exr", "I/O"), ("light_background_em 1 1.5 "
                       + os.path.basename(path) + ".env.exr", "invalid scene"), ("light_background_em 1", "invalid scene")):
        open(path + ".aux", "w").write("\n".join(aux + [line]) + "\n")
        with pytest.raises(upbp.UpbpError, match=code):
            upbp.load_scene(["-s", "-1", path, "-r", "8x8"])
