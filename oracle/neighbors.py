"""Brute-force photon neighbour sets (oracle restatement).

Every photon or beam is tested against the estimators' exact predicates of
gpuupbp/kernel/intersection.cuh:
  point_point               (lines 64-69)    SURF, PP3D
  test_intersection_bre     (lines 82-103)   PB2D (query ray), BP2D (beam ray)
  test_intersection_beam_beam (lines 117-171, with beam_beam at 33-53) BB1D
evaluated in IEEE float32 one operation at a time in the reference's
expression order (numpy never fuses a multiply-add), so the result is the
set a correctly rounded evaluation of those expressions defines.  No
acceleration structure: the set cannot depend on one.

Test infrastructure only.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def _dot(ax, ay, az, bx, by, bz):
    return (ax * bx + ay * by) + az * bz


def points_in_radius(points: np.ndarray, x, r2) -> np.ndarray:
    """Indices of rows of points (x, y, z, ...) with |x - p|^2 <= r2."""
    p = points[:, :3].astype(f32)
    q = np.asarray(x, f32)
    dx, dy, dz = q[0] - p[:, 0], q[1] - p[:, 1], q[2] - p[:, 2]
    return np.nonzero(_dot(dx, dy, dz, dx, dy, dz) <= f32(r2))[0]


def ray_disc(o, d, tmin, tmax, p: np.ndarray, r2) -> np.ndarray:
    """Mask of points p (N x 3) whose disc of squared radius r2, facing the
    ray (o, d), is crossed at a distance in (tmin, tmax)."""
    o = np.asarray(o, f32)
    d = np.asarray(d, f32)
    vx, vy, vz = p[:, 0] - o[0], p[:, 1] - o[1], p[:, 2] - o[2]
    t = _dot(vx, vy, vz, d[0], d[1], d[2])
    inside = (t > f32(tmin)) & (t < f32(tmax))
    ex = (o[0] + d[0] * t) - p[:, 0]
    ey = (o[1] + d[1] * t) - p[:, 1]
    ez = (o[2] + d[2] * t) - p[:, 2]
    return inside & (_dot(ex, ey, ez, ex, ey, ez) <= f32(r2))


def points_near_segment(points: np.ndarray, query, r2) -> np.ndarray:
    q = np.asarray(query, f32)
    return np.nonzero(ray_disc(q[0:3], q[3:6], q[6], q[7], points[:, :3].astype(f32), r2))[0]


def beams_near_point(beams: np.ndarray, x, r2) -> np.ndarray:
    """beams: N x 8 (origin xyz, length, direction xyz, path bits)."""
    b = beams.astype(f32)
    x = np.asarray(x, f32)
    hits = []
    # vectorised over beams: each beam is its own ray
    vx, vy, vz = x[0] - b[:, 0], x[1] - b[:, 1], x[2] - b[:, 2]
    t = _dot(vx, vy, vz, b[:, 4], b[:, 5], b[:, 6])
    inside = (t > f32(0.0)) & (t < b[:, 3])
    ex = (b[:, 0] + b[:, 4] * t) - x[0]
    ey = (b[:, 1] + b[:, 5] * t) - x[1]
    ez = (b[:, 2] + b[:, 6] * t) - x[2]
    hits = inside & (_dot(ex, ey, ez, ex, ey, ez) <= f32(r2))
    return np.nonzero(hits)[0]


def beams_near_segment(beams: np.ndarray, query, r2, path_limit: int | None = None) -> np.ndarray:
    """BB1D neighbour set of query (o, d, tmin, tmax); with path_limit only
    beams of light paths below that index qualify."""
    b = beams.astype(f32)
    q = np.asarray(query, f32)
    o1, d1, min1, max1 = q[0:3], q[3:6], q[6], q[7]
    o2x, o2y, o2z, len2 = b[:, 0], b[:, 1], b[:, 2], b[:, 3]
    d2x, d2y, d2z = b[:, 4], b[:, 5], b[:, 6]
    cx = d1[1] * d2z - d1[2] * d2y
    cy = d1[2] * d2x - d1[0] * d2z
    cz = d1[0] * d2y - d1[1] * d2x
    s2 = _dot(cx, cy, cz, cx, cy, cz)
    ad = _dot(o2x - o1[0], o2y - o1[1], o2z - o1[2], cx, cy, cz)
    ok = ~(ad * ad >= f32(r2) * s2)
    dd = _dot(d1[0], d1[1], d1[2], d2x, d2y, d2z)
    dd2m1 = dd * dd - f32(1.0)
    ok &= ~((dd2m1 < f32(1e-5)) & (dd2m1 > f32(-1e-5)))
    d1o1 = _dot(d1[0], d1[1], d1[2], o1[0], o1[1], o1[2])
    d1o2 = _dot(d1[0], d1[1], d1[2], o2x, o2y, o2z)
    with np.errstate(divide="ignore", invalid="ignore"):
        t1 = ((d1o1 - d1o2) - dd * (_dot(d2x, d2y, d2z, o1[0], o1[1], o1[2]) - _dot(d2x, d2y, d2z, o2x, o2y, o2z))) / dd2m1
        ok &= ~((t1 <= min1) | (t1 >= max1))
        t2 = ((t1 + d1o1) - d1o2) / dd
        ok &= ~((t2 <= f32(0.0)) | (t2 >= len2) | np.isnan(t2))
    if path_limit is not None:
        path = beams[:, 7].astype(np.float32).view(np.uint32)
        ok &= path < np.uint32(path_limit)
    return np.nonzero(ok)[0]
