"""The beam map's two builds give the same estimates.

The beam map (the BVH over beam chunks that BB1D and BP2D search) is built
every iteration by locally-ordered clustering; with UPBP_BEAM_MAP=lbvh it is
the Morton-split LBVH, and a clustering that runs out of passes
(UPBP_PLOC_PASSES caps them) or fails its layout check is replaced by the
LBVH before any search walks it.  The trees differ, the neighbour pairs may
not: on the media field with all 921 600 light paths of the benchmark (a
few million chunks, so the many-cluster passes run), the three renderers
find the same BB1D and BP2D pairs, test nearly the same leaves (their
internal boxes differ), and render the same image up to the order of the
floating-point additions into each pixel.  The clustered tree also visits
fewer nodes, which is its point.
"""
import os

import numpy as np
import pytest

from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu

ARGS = ["-a", "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d", "-l", "12", "-r", "160x90", "-pcpi", "921600"]
ITERATIONS = [0, 1]


def _render(path, env):
    from gpuupbp_b200 import upbp
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        r = upbp.Renderer(["-s", "-1", path] + ARGS)  # the variables are read here
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    out = []
    for it in ITERATIONS:
        status = r.run_iteration(it)
        img = r.iteration_image().copy()
        st = r.stats()
        out.append({"status": status, "img": img, "passes": st["beam_map_passes"],
                    "bb1d": st["work"]["bb1d_query"], "bp2d": st["work"]["bp2d_query"]})
    r.close()
    return out


def test_clustered_and_lbvh_beam_maps_agree(scene_dir):
    path = scenes.write_workload("media_field", scene_dir)
    ploc = _render(path, {})
    lbvh = _render(path, {"UPBP_BEAM_MAP": "lbvh"})
    fallback = _render(path, {"UPBP_PLOC_PASSES": "1"})
    for a, b, c in zip(ploc, lbvh, fallback):
        assert a["passes"] > 1, a["passes"]          # clustered, many-cluster passes and the final block
        assert b["passes"] == 0 and c["passes"] == 0  # LBVH, chosen or as the fallback
        for k in ("bb1d", "bp2d"):
            assert a[k]["beam_hit"] == b[k]["beam_hit"] == c[k]["beam_hit"], (k, a[k], b[k], c[k])
            # the same LBVH build; the beams' order (appended by atomics in
            # the light pass) breaks Morton ties, so node visits agree to a
            # few in millions, not exactly
            for w in ("nodes", "beam_cand"):
                assert abs(c[k][w] - b[k][w]) <= 1e-4 * b[k][w] + 16, (k, w, c[k], b[k])
        # the clustered tree: fewer node visits, leaf tests within 2% (the
        # boxes of the two trees' internal nodes differ, the leaves do not)
        assert a["bb1d"]["nodes"] < 0.95 * b["bb1d"]["nodes"], (a["bb1d"], b["bb1d"])
        assert abs(a["bb1d"]["beam_cand"] - b["bb1d"]["beam_cand"]) <= 0.02 * b["bb1d"]["beam_cand"]
        assert a["status"] == b["status"] == c["status"]
        for x in (a, c):
            rel = np.abs(x["img"] - b["img"]) / (np.abs(b["img"]) + 1e-3)
            assert np.isfinite(x["img"]).all()
            assert float(np.mean(np.all(rel < 1e-4, axis=-1))) >= 0.999
