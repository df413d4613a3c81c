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


def _check(r, kind, queries, brute, items=None, ill_posed=None):
    """Neighbour sets equal brute force; with ill_posed(query, item) the
    pairs it flags are left out of the comparison on both sides."""
    sets, counts = r.query(kind, queries)
    assert counts.max() < 4096
    nonempty = 0
    for q, got in zip(queries, sets):
        want = np.sort(brute(q))
        assert len(got) == len(np.unique(got)), "duplicate neighbour"
        if ill_posed is not None:
            got = np.array([i for i in got if not ill_posed(q, items[i])], np.uint32)
            want = np.array([i for i in want if not ill_posed(q, items[i])], np.int64)
        if not np.array_equal(np.sort(got), want) and items is not None:
            diff = np.setxor1d(got, want)
            print("query", q.tolist(), "differs on", [items[i].tolist() for i in diff])
        assert np.array_equal(np.sort(got), want)
        nonempty += len(want) > 0
    return nonempty


def _beam_pair_ill_posed(q, beam, r):
    """A query segment / beam pair whose acceptance hangs on rounding: the
    true (float64) closest points of the two lines fall outside either
    segment, or their distance is within 1% of the radius.  The predicate's
    closest points are inexact (its t2 divides by d1.d2), so for such a pair
    the accepted set depends on how candidates are culled -- brute force over
    all beams accepts it on noise, the reference's and this build's walks only
    if the query passes near the beam segment."""
    o1, d1 = q[:3].astype(np.float64), q[3:6].astype(np.float64)
    o2, d2, length = beam[:3].astype(np.float64), beam[4:7].astype(np.float64), float(beam[3])
    b = d1 @ d2
    den = (d1 @ d1) * (d2 @ d2) - b * b
    if den < 1e-12:
        return True
    w = o1 - o2
    t1 = (b * (d2 @ w) - (d2 @ d2) * (d1 @ w)) / den
    t2 = ((d1 @ d1) * (d2 @ w) - b * (d1 @ w)) / den
    dist = np.linalg.norm((o1 + d1 * t1) - (o2 + d2 * t2))
    return not (q[6] < t1 < q[7] and 0.0 < t2 < length and dist < 0.99 * float(r))


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


def _media_renderer(scene_dir):
    return _renderer(scene_dir, "media_field", True,
                     ["-a", "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d", "-l", "12", "-r", "64x64"])


def _beam_frames(beams, rb1, rng, n):
    # the light pass appends beams in no fixed order: pick by content
    long_ = beams[beams[:, 3] > 8 * rb1]
    long_ = long_[np.lexsort(long_[:, :7].T[::-1])]
    assert len(long_) > 100
    b = long_[rng.integers(0, len(long_), n)].astype(np.float64)
    d2 = b[:, 4:7] / np.linalg.norm(b[:, 4:7], axis=1, keepdims=True)
    a = rng.normal(size=(n, 3))
    u = a - d2 * np.sum(a * d2, axis=1, keepdims=True)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    mid = b[:, :3] + d2 * (b[:, 3] * rng.uniform(0.2, 0.8, n))[:, None]
    return d2, u, np.cross(d2, u), mid


def test_bb1d_near_parallel_queries_equal_brute_force(scene_dir):
    """BB1D queries almost parallel to a beam (1 - dd^2 from 1.5e-5 up) at a
    distance just under the radius, on the media scene whose coordinates are
    large against the radius: the predicate's t1 carries its largest error
    there.  The set must equal brute force."""
    r = _media_renderer(scene_dir)
    rb1 = np.float32(r.stats()["radius"][0])
    beams = r.photons(2)
    rng = np.random.default_rng(23)
    n = 2000
    d2, u, v, mid = _beam_frames(beams, rb1, rng, n)
    sin2 = 10.0 ** rng.uniform(np.log10(1.5e-5), -3.0, n)
    d1 = np.sqrt(1.0 - sin2)[:, None] * d2 + np.sqrt(sin2)[:, None] * u
    centre = mid + v * (float(rb1) * rng.uniform(0.5, 0.999, n))[:, None]
    half = 20.0 * float(rb1)
    q = np.zeros((n, 8), np.float32)
    q[:, :3] = centre - d1 * half
    q[:, 3:6] = d1
    q[:, 7] = 2 * half
    # half of the segments end short of the closest approach, by up to the
    # size of the predicate's error in t1, where only that error accepts them
    short = np.arange(n) % 2 == 1
    extent = float(np.abs(beams[:, :3]).max())
    q[short, 7] = half - rng.uniform(0.0, 0.02 * extent, short.sum())
    nonempty = _check(r, 3, q, lambda qq: neighbors.beams_near_segment(beams, qq, rb1 ** 2), beams,
                      lambda qq, bb: _beam_pair_ill_posed(qq, bb, rb1))
    assert nonempty > n // 4
    r.close()


def test_bb1d_near_perpendicular_queries_equal_brute_force(scene_dir):
    """BB1D queries almost perpendicular to a beam (|d1.d2| from 1e-7 to
    1e-2).  The predicate computes the beam's closest point by dividing by
    d1.d2, so it can land far from where the query passes; the beam must
    still be reported once, exactly as brute force reports it.  Pairs whose
    true closest points lie outside the segments (a collinear neighbour beam,
    say) are ill-posed and left out (_beam_pair_ill_posed)."""
    r = _media_renderer(scene_dir)
    rb1 = np.float32(r.stats()["radius"][0])
    beams = r.photons(2)
    rng = np.random.default_rng(29)
    n = 3000
    d2, u, v, mid = _beam_frames(beams, rb1, rng, n)
    eps = 10.0 ** rng.uniform(-7.0, -2.0, n) * rng.choice([-1.0, 1.0], n)
    d1 = u + eps[:, None] * d2
    d1 /= np.linalg.norm(d1, axis=1, keepdims=True)
    w = np.cross(d1, d2)
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    centre = mid + w * (float(rb1) * rng.uniform(0.0, 0.999, n))[:, None]
    half = float(rb1) * rng.uniform(2.0, 10.0, n)
    q = np.zeros((n, 8), np.float32)
    q[:, :3] = centre - d1 * half[:, None]
    q[:, 3:6] = d1
    q[:, 7] = 2 * half
    nonempty = _check(r, 3, q, lambda qq: neighbors.beams_near_segment(beams, qq, rb1 ** 2), beams)
    assert nonempty > n // 4
    r.close()
