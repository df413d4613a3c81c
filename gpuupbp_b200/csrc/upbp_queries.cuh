// Range queries over the per-iteration photon maps.  Each walker visits the
// BVH leaves whose box (built dilated by the map's largest query radius) the
// query touches, and
// calls f for every photon or beam that passes the estimator's exact
// predicate; the neighbour set is therefore defined by the predicate alone
// (the reference's OptiX intersection programs apply the same predicates,
// gpuupbp/kernel/pde/program_*.cu).  The estimators and the diagnostic
// neighbour-set query both use these walkers.
#pragma once

#include "upbp_paths.cuh"

namespace upbp {

// Photons within radius r of x (SURF, PP3D): f(vertex slot).
template <class F>
UPBP_D void points_in_radius(const PointMap& map, float3 x, float r2, F&& f)
{
    unsigned cand = 0, hits = 0;
    const bool ok = bvh_walk(
        map.bvh, [&](float3 lo, float3 hi) { return inside(lo, hi, x); },
        [&](int i) {
            const float4 pp = __ldg(&map.pos[i]);
            cand++;
            if (pred_point_point(x, xyz(pp), r2)) {
                hits++;
                f(fbits(pp.w));
            }
            return true;
        });
    count_work(kCtrPointCand, cand);
    count_work(kCtrPointHit, hits);
    if (!ok) flag_status(kErrTraversalStack);
}

// Photons whose disc of radius r the query segment (o, d, (tmin, tmax))
// crosses (PB2D): f(vertex slot, distance along the query, squared radius).
template <class F>
UPBP_D void points_near_segment(const PointMap& map, float3 o, float3 d, float tmin, float tmax, float r2, F&& f)
{
    const float3 inv = safe_inv(d), oinv = oinv_of(o, inv);
    unsigned cand = 0, hits = 0;
    const bool ok = bvh_walk(
        map.bvh, [&](float3 lo, float3 hi) { return slab(lo, hi, inv, oinv, tmin, tmax); },
        [&](int i) {
            const float4 pp = __ldg(&map.pos[i]);
            float dist, rad2;
            cand++;
            if (pred_ray_disc(o, d, tmin, tmax, xyz(pp), r2, dist, rad2)) {
                hits++;
                f(fbits(pp.w), dist, rad2);
            }
            return true;
        });
    count_work(kCtrPointCand, cand);
    count_work(kCtrPointHit, hits);
    if (!ok) flag_status(kErrTraversalStack);
}

// Photon beams passing within sqrt(r2) of the query segment (BB1D); with
// need_mask only beams of the first bb1d_used_light_subpath_count light
// paths.  f(beam index, distance, sin theta, t along query, t along beam).
// Beams are stored as chunks; a beam is reported only through the chunk that
// holds its closest point, so each beam appears at most once.  med >= 0
// skips beams of other media before the predicate (the estimator only merges
// beams in the query segment's medium, functs_bb1d.cuh:66).
struct BeamSegHit {
    unsigned beam;
    float dist, sin_theta, t1, t2;
};

// Segment [tmin, tmax] of (o, d) vs chunk k of n of a beam, with the box
// test of the beam-map walk (same box, same dilation, same arithmetic).
UPBP_D bool chunk_reached(float3 bo, float3 bd, float len, unsigned k, unsigned n, float dilate, float3 o, float3 d,
                          float tmin, float tmax)
{
    float3 lo, hi;
    chunk_box(bo, bd, len, k, n, lo, hi);
    dilate_box(lo, hi, dilate);
    const float3 inv = safe_inv(d);
    return slab(lo, hi, inv, oinv_of(o, inv), tmin, tmax);
}

// The BB1D test of one beam-map leaf against a query segment: the path mask,
// the medium filter and the exact beam-beam predicate, which looks at the
// whole beam, so every chunk of an accepted beam passes it; one of them
// reports the beam.  That is the chunk holding the beam's closest point t2
// when the walk reaches its box.  The predicate's t2 can be far from the
// true closest point (it divides by d1.d2, which is tiny for nearly
// perpendicular lines), and then the chunk holding it can lie outside the
// query's reach: in that case the first chunk of the beam whose box the query
// reaches reports instead (a check that is only needed when the computed
// closest points are far apart).  A chunk whose own box passes the walk's box test
// is always visited, so exactly one chunk reports each accepted beam, and
// the set equals a test of every beam (a chunk reached only as part of a
// leaf of several chunks never reports).  cand counts the leaves that reach
// the predicate; own_box tells that the walk reached this chunk through a
// leaf of its own (so its box passed).  The query's medium is `med`, or,
// when med_src is set, med_src->w: read, like the chunk's medium and range,
// only for pairs the predicate accepts (three of four are rejected, and each
// record read is one more L1 lookup per lane).
UPBP_D bool beam_chunk_vs_segment(const BeamMap& map, int i, float3 o, float3 d, float tmin, float tmax, float r2,
                                  bool own_box, bool need_mask, int med, const float4* med_src, unsigned& cand,
                                  BeamSegHit& h)
{
    const float4 s1 = __ldg(&map.seg[3 * i + 1]);
    const unsigned bits = fbits(s1.w);
    if (need_mask && !(bits >> 31)) return false;
    const float4 s0 = __ldg(&map.seg[3 * i]);
    cand++;
    if (!pred_beam_beam(o, d, tmin, tmax, xyz(s0), xyz(s1), s0.w, r2, h.dist, h.sin_theta, h.t1, h.t2)) return false;
    const float4 s2 = __ldg(&map.seg[3 * i + 2]);
    if (med_src) med = (int)fbits(__ldg(med_src).w);
    if (med >= 0 && (int)fbits(s2.z) != med) return false;
    h.beam = bits & 0x7fffffffu;
    const bool mine = h.t2 >= s2.x && h.t2 < s2.y;
    const float3 bo = xyz(s0), bd = xyz(s1);
    // Usual case: the computed closest points lie within the dilation of each
    // other (less a rounding margin), so the query passes through the dilated
    // own box of the chunk holding t2 at t1, and the walk reached that chunk.
    const float3 gap = (o + d * h.t1) - (bo + bd * h.t2);
    const float inner = map.dilate - 2.f * c_params.cull_eps;
    if (inner > 0.f && dot(gap, gap) <= inner * inner) return mine;
    const unsigned kc = fbits(s2.w), k = kc & 0xffffu, n = kc >> 16;
    // a leaf of several chunks is visited when any of its chunks is in
    // reach, so this chunk's own box decides, as for every other chunk
    if (!own_box && !chunk_reached(bo, bd, s0.w, k, n, map.dilate, o, d, tmin, tmax)) return false;
    if (mine) return true;
    if (chunk_reached(bo, bd, s0.w, chunk_of(h.t2, s0.w, n), n, map.dilate, o, d, tmin, tmax)) return false;
    for (unsigned j = 0; j < k; j++)
        if (chunk_reached(bo, bd, s0.w, j, n, map.dilate, o, d, tmin, tmax)) return false;
    return true;
}

template <class F>
UPBP_D void beams_near_segment(const BeamMap& map, float3 o, float3 d, float tmin, float tmax, float r2,
                               bool need_mask, int med, F&& f)
{
    const float3 inv = safe_inv(d), oinv = oinv_of(o, inv);
    unsigned cand = 0, hits = 0, visits = 0;
    bool overflow = false;
    WalkState s;
    walk_begin(s, map.bvh);
    while (s.node != kWalkDone) {
        const int leaf = walk_step(
            s, map.bvh, [&](float3 lo, float3 hi) { return slab(lo, hi, inv, oinv, tmin, tmax); }, overflow, visits);
        BeamSegHit h;
        if (leaf >= 0 &&
            beam_chunk_vs_segment(map, leaf, o, d, tmin, tmax, r2, false, need_mask, med, nullptr, cand, h)) {
            hits++;
            f(h.beam, h.dist, h.sin_theta, h.t1, h.t2);
        }
    }
    count_work(kCtrNodes, visits);
    count_work(kCtrBeamCand, cand);
    count_work(kCtrBeamHit, hits);
    if (overflow) flag_status(kErrTraversalStack);
}

// Photon beams whose disc of radius sqrt(r2) contains x (BP2D):
// f(beam index, distance along the beam, squared radius).
template <class F>
UPBP_D void beams_near_point(const BeamMap& map, float3 x, float r2, F&& f)
{
    unsigned cand = 0, hits = 0;
    const bool ok = bvh_walk(
        map.bvh, [&](float3 lo, float3 hi) { return inside(lo, hi, x); },
        [&](int i) {
            const float4 s0 = __ldg(&map.seg[3 * i]), s1 = __ldg(&map.seg[3 * i + 1]);
            const float4 s2 = __ldg(&map.seg[3 * i + 2]);
            float dist, rad2;
            cand++;
            if (pred_ray_disc(xyz(s0), xyz(s1), 0.f, s0.w, x, r2, dist, rad2) && dist >= s2.x && dist < s2.y) {
                hits++;
                f(fbits(s1.w) & 0x7fffffffu, dist, rad2);
            }
            return true;
        });
    count_work(kCtrBeamCand, cand);
    count_work(kCtrBeamHit, hits);
    if (!ok) flag_status(kErrTraversalStack);
}

}  // namespace upbp
