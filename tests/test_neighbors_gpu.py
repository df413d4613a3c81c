"""Photon neighbour sets of the five range queries equal a brute-force search
with the same exact predicates, bit for bit (oracle/neighbors.py).  Queries
are drawn around the stored photons so the sets are not empty, plus
segments through the media."""
import numpy as np
import pytest

import neighbors
from cases import command_line
from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu


def _renderer(scene_dir, workload, tiny, case_args):
    from gpuupbp_b200 import upbp
    path = scenes.write_workload(workload, scene_dir, tiny=tiny)
    r = upbp.Renderer(["-s", "-1", path] + case_args)
    r.run_iteration(0)
    return r


def _check(r, kind, queries, brute):
    sets, counts = r.query(kind, queries)
    assert counts.max() < 4096
    nonempty = 0
    for q, got in zip(queries, sets):
        want = np.sort(brute(q))
        assert len(got) == len(np.unique(got)), "duplicate neighbour"
        assert np.array_equal(np.sort(got), want)
        nonempty += len(want) > 0
    return nonempty


@pytest.mark.parametrize("workload,tiny,args", [
    ("box_medium", False, ["-a", "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d", "-l", "8", "-r", "64x64", "-r_initial", "-0.02"]),
    ("dense_beams", True, ["-a", "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d", "-l", "16", "-r", "48x48",
                           "-r_initial_bb1d", "-0.004", "-r_initial_bp2d", "-0.004", "-pbc", "-0.5"]),
])
def test_neighbour_sets_equal_brute_force(scene_dir, workload, tiny, args):
    r = _renderer(scene_dir, workload, tiny, args)
    st = r.stats()
    rb1, rb2, rpb, rpp, rsu, _ = st["radius"]
    rng = np.random.default_rng(11)
    surf, med, beams = r.photons(0), r.photons(1), r.photons(2)
    assert len(surf) and len(med) and len(beams)
    slots_s = surf[:, 3].view(np.uint32)
    slots_m = med[:, 3].view(np.uint32)

    def around(pts, scale, n):
        p = pts[rng.integers(0, len(pts), n), :3]
        return p + rng.normal(size=(n, 3)).astype(np.float32) * scale

    def points_q(x):
        q = np.zeros((len(x), 8), np.float32)
        q[:, :3] = x
        return q

    # SURF / PP3D: points within the radius
    q = points_q(around(surf, rsu, 300))
    n = _check(r, 0, q, lambda qq: slots_s[neighbors.points_in_radius(surf, qq[:3], np.float32(rsu) ** 2)])
    assert n > 50
    q = points_q(around(med, rpp, 300))
    n = _check(r, 1, q, lambda qq: slots_m[neighbors.points_in_radius(med, qq[:3], np.float32(rpp) ** 2)])
    assert n > 50
    # PB2D: segments passing near medium photons
    c = around(med, rpb, 300)
    d = rng.normal(size=(300, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q = np.zeros((300, 8), np.float32)
    q[:, :3] = c - d * 0.3
    q[:, 3:6] = d
    q[:, 6] = rng.uniform(0.0, 0.1, 300)
    q[:, 7] = rng.uniform(0.3, 0.6, 300)
    n = _check(r, 2, q, lambda qq: slots_m[neighbors.points_near_segment(med, qq, np.float32(rpb) ** 2)])
    assert n > 50
    # BB1D: segments crossing near beams; only beams of the first pbc paths when BP2D is on
    pbc = int(r.config.bb1d_used_light_subpath_count) if r.config.bb1d_used_light_subpath_count > 0 else \
        int(np.floor(-r.config.bb1d_used_light_subpath_count * r.config.path_count_per_iter))
    mask_on = bool(r.config.algorithm_flags & (1 << 7))
    pick = beams[rng.integers(0, len(beams), 300)]
    t = rng.uniform(0, 1, 300).astype(np.float32) * pick[:, 3]
    c = pick[:, :3] + pick[:, 4:7] * t[:, None] + rng.normal(size=(300, 3)).astype(np.float32) * rb1
    q[:, :3] = c - d * 0.3
    q[:, 3:6] = d
    n = _check(r, 3, q, lambda qq: neighbors.beams_near_segment(beams, qq, np.float32(rb1) ** 2,
                                                                 pbc if mask_on else None))
    assert n > 20
    # BP2D: points near beams
    q = points_q(pick[:, :3] + pick[:, 4:7] * t[:, None] + rng.normal(size=(300, 3)).astype(np.float32) * rb2)
    n = _check(r, 4, q, lambda qq: neighbors.beams_near_point(beams, qq[:3], np.float32(rb2) ** 2))
    assert n > 50
    r.close()
