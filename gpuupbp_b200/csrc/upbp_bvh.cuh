// BVH traversal: closest hit and all-hits over triangles, and range queries
// (point-in-radius, segment-near-point, segment/point-vs-beam) over the
// per-iteration photon maps.  Traversal stacks live in registers/local memory,
// bounded at kStackDepth; overflow sets kErrTraversalStack and drops the
// remaining subtree (never an unbounded loop).
#pragma once

#include <climits>

#include "upbp_device.cuh"

namespace upbp {

constexpr int kStackDepth = 64;

// Adds v to work counter `which`, one atomic per warp.
UPBP_D void count_work(int which, unsigned v)
{
    const unsigned m = __activemask();
    const unsigned total = __reduce_add_sync(m, v);
    if ((threadIdx.x & 31) == __ffs(m) - 1 && total) atomicAdd(c_work_ptr() + which, (unsigned long long)total);
}

// Reserves n < 256 consecutive slots of `counter` for each lane of the
// converged group that calls it, with one atomic per group; returns the
// lane's first slot.  The prefix over the group is summed bit by bit from
// ballots, so any mask of active lanes works.
UPBP_D unsigned warp_reserve(unsigned* counter, unsigned n)
{
    const unsigned m = __activemask();
    const unsigned lane = threadIdx.x & 31;
    const unsigned below = m & ((1u << lane) - 1u);
    unsigned prefix = 0, total = 0;
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const unsigned bits = __ballot_sync(m, (n >> b) & 1u);
        prefix += (unsigned)__popc(bits & below) << b;
        total += (unsigned)__popc(bits) << b;
    }
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if ((int)lane == leader && total) base = atomicAdd(counter, total);
    base = __shfl_sync(m, base, leader);
    return base + prefix;
}

// warp_reserve for one slot per lane.
UPBP_D unsigned warp_reserve1(unsigned* counter)
{
    const unsigned m = __activemask();
    const unsigned lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (unsigned)__popc(m));
    base = __shfl_sync(m, base, leader);
    return base + (unsigned)__popc(m & ((1u << lane) - 1u));
}

UPBP_D float3 safe_inv(float3 d) { return make_float3(1.f / d.x, 1.f / d.y, 1.f / d.z); }

// Inverse direction and origin * inverse direction of a ray, the inputs of
// slab().
UPBP_D float3 oinv_of(float3 o, float3 inv) { return make_float3(o.x * inv.x, o.y * inv.y, o.z * inv.z); }

// Segment [tmin, tmax] of the ray o + t d vs box [lo, hi], with inv = 1/d and
// oinv = o * inv per ray: one multiply-add per plane.  An axis with a zero
// direction component yields NaN or infinite bounds, which fminf/fmaxf drop
// or which never reject, so the test never misses a box the segment touches.
// The photon maps' boxes already include the query radius (BoxSource.dilate).
UPBP_D bool slab(float3 lo, float3 hi, float3 inv, float3 oinv, float tmin, float tmax)
{
    const float tx0 = fmaf(lo.x, inv.x, -oinv.x), tx1 = fmaf(hi.x, inv.x, -oinv.x);
    const float ty0 = fmaf(lo.y, inv.y, -oinv.y), ty1 = fmaf(hi.y, inv.y, -oinv.y);
    const float tz0 = fmaf(lo.z, inv.z, -oinv.z), tz1 = fmaf(hi.z, inv.z, -oinv.z);
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    return tn <= tf;
}

UPBP_D bool inside(float3 lo, float3 hi, float3 x)
{
    return x.x >= lo.x && x.x <= hi.x && x.y >= lo.y && x.y <= hi.y && x.z >= lo.z && x.z <= hi.z;
}

struct NodeBoxes {
    float3 llo, lhi, rlo, rhi;
    int l, r;
};

UPBP_D NodeBoxes load_node(const BvhNode* nodes, int i)
{
    const BvhNode* n = nodes + i;
    const float4 a = __ldg(&n->a), b = __ldg(&n->b), c = __ldg(&n->c);
    const int4 k = __ldg(&n->link);
    NodeBoxes r;
    r.llo = make_float3(a.x, a.y, a.z);
    r.lhi = make_float3(a.w, b.x, b.y);
    r.rlo = make_float3(b.z, b.w, c.x);
    r.rhi = make_float3(c.y, c.z, c.w);
    r.l = k.x;
    r.r = k.y;
    return r;
}

// A compressed node decoded into the children's boxes (each containing the
// exact box) and links in BvhNode form.
UPBP_D NodeBoxes load_qnode(const QNode* q, int i)
{
    const float4 a = __ldg(&q[i].a);
    const uint4 b = __ldg(&q[i].b);
    const unsigned e = __float_as_uint(a.w);
    const float sx = qnode_step(e & 0xffu), sy = qnode_step((e >> 8) & 0xffu), sz = qnode_step((e >> 16) & 0xffu);
    NodeBoxes r;
    r.llo = make_float3(qnode_plane(b.x, 0, sx, a.x), qnode_plane(b.x, 1, sy, a.y), qnode_plane(b.x, 2, sz, a.z));
    r.lhi = make_float3(qnode_plane(b.x, 3, sx, a.x), qnode_plane(b.y, 0, sy, a.y), qnode_plane(b.y, 1, sz, a.z));
    r.rlo = make_float3(qnode_plane(b.y, 2, sx, a.x), qnode_plane(b.y, 3, sy, a.y), qnode_plane(b.z, 0, sz, a.z));
    r.rhi = make_float3(qnode_plane(b.z, 1, sx, a.x), qnode_plane(b.z, 2, sy, a.y), qnode_plane(b.z, 3, sz, a.z));
    const int g = (int)(b.w & 0x3fffffffu);
    r.l = (b.w >> 30) & 1u ? leaf_link(g, 1) : g;
    r.r = (b.w >> 31) ? leaf_link(g + 1, 1) : g + 1;
    return r;
}

// Segment [tmin, tmax] of a ray (inv = 1/d, oinv = o * inv) against both
// children of compressed node i, the dequantisation folded into the plane
// distances: a plane origin + q * step lies at t = q * (step * inv) +
// (origin * inv - oinv), one multiply-add per plane after six per node.
// The rounding differs from slab() on the decoded planes by a few units in
// the last place of t, far inside the margins the stored boxes carry.
UPBP_D void qnode_slab(const QNode* q, int i, float3 inv, float3 oinv, float tmin, float tmax, bool& hl, bool& hr,
                       int& l, int& r)
{
    const float4 a = __ldg(&q[i].a);
    const uint4 b = __ldg(&q[i].b);
    const unsigned e = __float_as_uint(a.w);
    const float sx = qnode_step(e & 0xffu) * inv.x, sy = qnode_step((e >> 8) & 0xffu) * inv.y,
                sz = qnode_step((e >> 16) & 0xffu) * inv.z;
    const float ox = fmaf(a.x, inv.x, -oinv.x), oy = fmaf(a.y, inv.y, -oinv.y), oz = fmaf(a.z, inv.z, -oinv.z);
    auto t = [](unsigned word, int byte, float s, float o) { return fmaf((float)((word >> (8 * byte)) & 0xffu), s, o); };
    {
        const float x0 = t(b.x, 0, sx, ox), y0 = t(b.x, 1, sy, oy), z0 = t(b.x, 2, sz, oz);
        const float x1 = t(b.x, 3, sx, ox), y1 = t(b.y, 0, sy, oy), z1 = t(b.y, 1, sz, oz);
        const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
        const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
        hl = tn <= tf;
    }
    {
        const float x0 = t(b.y, 2, sx, ox), y0 = t(b.y, 3, sy, oy), z0 = t(b.z, 0, sz, oz);
        const float x1 = t(b.z, 1, sx, ox), y1 = t(b.z, 2, sy, oy), z1 = t(b.z, 3, sz, oz);
        const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
        const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
        hr = tn <= tf;
    }
    const int g = (int)(b.w & 0x3fffffffu);
    l = (b.w >> 30) & 1u ? leaf_link(g, 1) : g;
    r = (b.w >> 31) ? leaf_link(g + 1, 1) : g + 1;
}

// Visits every leaf whose box (dilated by pad) passes `test_box`; calls
// leaf(sorted_index) which returns false to stop.  Returns false if the
// traversal stack overflowed.
template <class BoxTest, class Leaf>
UPBP_D bool bvh_walk(const BvhView& bvh, BoxTest&& test_box, Leaf&& leaf)
{
    if (bvh.count == 0) return true;
    int stack[kStackDepth];
    int sp = 0;
    int node = bvh.count > 1 ? 0 : ~0;
    bool ok = true;
    unsigned visits = 0;
    for (;;) {
        if (node < 0) {
            const int first = leaf_first(node), cnt = leaf_count(node);
            bool go = true;
            for (int i = 0; i < cnt && go; i++) go = leaf(first + i);
            if (!go) {
                count_work(kCtrNodes, visits);
                return ok;
            }
        } else {
            visits++;
            const NodeBoxes nb = load_node(bvh.nodes, node);
            const bool hl = test_box(nb.llo, nb.lhi);
            const bool hr = test_box(nb.rlo, nb.rhi);
            if (hl && hr) {
                if (sp < kStackDepth) {
                    stack[sp++] = nb.r;
                } else {
                    ok = false;
                }
                node = nb.l;
                continue;
            }
            if (hl) {
                node = nb.l;
                continue;
            }
            if (hr) {
                node = nb.r;
                continue;
            }
        }
        if (sp == 0) {
            count_work(kCtrNodes, visits);
            return ok;
        }
        node = stack[--sp];
    }
}

// Resumable form of bvh_walk: walk_step() advances by exactly one internal
// node or one leaf, so a warp can move all its lanes in lock step and give a
// lane that finished its query a new one (the range-query search kernels).
// Visits the same leaves in the same order as bvh_walk.
constexpr int kWalkDone = INT_MIN;

struct WalkState {
    int node;  // next node: >= 0 internal, < 0 ~leaf, kWalkDone when finished
    int sp;
    int stack[kStackDepth];
};

UPBP_D void walk_begin(WalkState& s, const BvhView& bvh)
{
    s.sp = 0;
    s.node = bvh.count == 0 ? kWalkDone : (bvh.count > 1 ? 0 : ~0);
}

UPBP_D void walk_pop(WalkState& s) { s.node = s.sp > 0 ? s.stack[--s.sp] : kWalkDone; }

// One step of a walk with s.node != kWalkDone.  Returns the sorted index of
// the primitive this step reached (one per step through a leaf), or -1 after
// an internal node.
template <class BoxTest>
UPBP_D int walk_step(WalkState& s, const BvhView& bvh, BoxTest&& test_box, bool& overflow, unsigned& visits)
{
    const int node = s.node;
    if (node < 0) {
        const int first = leaf_first(node), cnt = leaf_count(node);
        if (cnt > 1)
            s.node = leaf_link(first + 1, cnt - 1);
        else
            walk_pop(s);
        return first;
    }
    visits++;
    const NodeBoxes nb = load_node(bvh.nodes, node);
    const bool hl = test_box(nb.llo, nb.lhi);
    const bool hr = test_box(nb.rlo, nb.rhi);
    if (hl && hr) {
        if (s.sp < kStackDepth)
            s.stack[s.sp++] = nb.r;
        else
            overflow = true;
        s.node = nb.l;
    } else if (hl) {
        s.node = nb.l;
    } else if (hr) {
        s.node = nb.r;
    } else {
        walk_pop(s);
    }
    return -1;
}

// Moller-Trumbore, double sided; identical arithmetic to the oracle's test.
UPBP_D bool tri_intersect(const float4* tri, int s, float3 o, float3 d, float& t, float& u, float& v)
{
    const float4 a = __ldg(&tri[3 * s]), b = __ldg(&tri[3 * s + 1]), c = __ldg(&tri[3 * s + 2]);
    const float3 v0 = xyz(a), e1 = xyz(b), e2 = xyz(c);
    const float3 p = cross(d, e2);
    const float det = dot(e1, p);
    if (det == 0.f) return false;
    const float inv = 1.f / det;
    const float3 sv = o - v0;
    u = dot(sv, p) * inv;
    if (u < 0.f || u > 1.f) return false;
    const float3 q = cross(sv, e1);
    v = dot(d, q) * inv;
    if (v < 0.f || u + v > 1.f) return false;
    t = dot(e2, q) * inv;
    return true;
}

struct TriHit {
    float t, u, v;  // sphere hits: (u, v, w) is the normal
    float w;
    int prim;       // original triangle index; ~index for a sphere
};

// Ray-sphere roots as the reference's sphere intersection program finds them
// (gpuupbp/kernel/intersector.cu:35-97): the near root of the unit-direction
// quadratic, refined once by solving again from its own point when it lies
// farther than the radius, and the far root of the (refined) solve.  Normals
// are (point - centre) / radius.  False when the ray misses the sphere.
UPBP_D bool sphere_roots(float4 s, float3 ro, float3 rd, float& t1, float3& n1, float& t2, float3& n2)
{
    const float radius = s.w;
    const float3 o = ro - make_float3(s.x, s.y, s.z);
    const float l = 1.f / length(rd);
    const float3 d = rd * l;
    float b = dot(o, d);
    float c = dot(o, o) - radius * radius;
    float disc = b * b - c;
    if (!(disc > 0.f)) return false;
    float sdisc = sqrtf(disc);
    const float root1 = -b - sdisc;
    float root11 = 0.f;
    const bool refine = fabsf(root1) > radius;
    if (refine) {
        const float3 o1 = o + root1 * d;
        b = dot(o1, d);
        c = dot(o1, o1) - radius * radius;
        disc = b * b - c;
        if (disc > 0.f) {
            sdisc = sqrtf(disc);
            root11 = -b - sdisc;
        }
    }
    const float inv_r = 1.f / radius;
    t1 = (root1 + root11) * l;
    n1 = (o + (root1 + root11) * d) * inv_r;
    const float root2 = (-b + sdisc) + (refine ? root1 : 0.f);
    t2 = root2 * l;
    n2 = (o + root2 * d) * inv_r;
    return true;
}

UPBP_D void sphere_hit(TriHit& h, float t, float3 n, int k)
{
    h.t = t;
    h.u = n.x;
    h.v = n.y;
    h.w = n.z;
    h.prim = ~k;
}

// Closest triangle hit with t in [tmin, best] (updates best); ordered
// traversal, near child first.
UPBP_D bool closest_triangle(const TriView& tv, float3 o, float3 d, float tmin, float& best, TriHit& hit,
                             bool& overflow)
{
    bool found = false;
    const float3 inv = safe_inv(d);
    int stack[kStackDepth];
    int sp = 0;
    int node = tv.bvh.count > 1 ? 0 : ~0;
    unsigned visits = 0, tests = 0;
    for (;;) {
        if (node < 0) {
            const int first = leaf_first(node), cnt = leaf_count(node);
            for (int s = first; s < first + cnt; s++) {
                float t, u, v;
                tests++;
                if (tri_intersect(tv.tri, s, o, d, t, u, v) && t >= tmin && t <= best) {
                    best = t;
                    hit.t = t;
                    hit.u = u;
                    hit.v = v;
                    hit.prim = __float_as_int(__ldg(&tv.tri[3 * s]).w);
                    found = true;
                }
            }
        } else {
            visits++;
            const NodeBoxes nb = load_node(tv.bvh.nodes, node);
            // entry distances for ordering
            const float3 t0l = (nb.llo - o) * inv, t1l = (nb.lhi - o) * inv;
            const float3 t0r = (nb.rlo - o) * inv, t1r = (nb.rhi - o) * inv;
            const float nl = fmaxf(fmaxf(fminf(t0l.x, t1l.x), fminf(t0l.y, t1l.y)), fmaxf(fminf(t0l.z, t1l.z), tmin));
            const float fl = fminf(fminf(fmaxf(t0l.x, t1l.x), fmaxf(t0l.y, t1l.y)), fminf(fmaxf(t0l.z, t1l.z), best));
            const float nr = fmaxf(fmaxf(fminf(t0r.x, t1r.x), fminf(t0r.y, t1r.y)), fmaxf(fminf(t0r.z, t1r.z), tmin));
            const float fr = fminf(fminf(fmaxf(t0r.x, t1r.x), fmaxf(t0r.y, t1r.y)), fminf(fmaxf(t0r.z, t1r.z), best));
            const bool hl = nl <= fl * 1.00001f + 1e-7f, hr = nr <= fr * 1.00001f + 1e-7f;
            if (hl && hr) {
                const bool left_first = nl <= nr;
                if (sp < kStackDepth) {
                    stack[sp++] = left_first ? nb.r : nb.l;
                } else {
                    overflow = true;
                }
                node = left_first ? nb.l : nb.r;
                continue;
            }
            if (hl) {
                node = nb.l;
                continue;
            }
            if (hr) {
                node = nb.r;
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    count_work(kCtrNodes, visits);
    count_work(kCtrTris, tests);
    return found;
}

// Analytic spheres (predefined scenes) are tested after the tree walks.  The
// fixed-slot copy of the device code (upbp_slot0.cu) is compiled without
// them and runs only scenes that have none: the sphere loops kept registers
// live across the path kernels' walks (0.7 ms per iteration on a triangle
// scene).
#ifdef UPBP_NO_SPHERES
constexpr bool kSceneSpheres = false;
#else
constexpr bool kSceneSpheres = true;
#endif

// Closest triangle hit with t in [tmin, tmax], or closer sphere hit with t in
// (tmin, tmax): a sphere reports its near root when that lies in range, else
// its far root.  The spheres are tested after the tree, so that nothing of
// theirs is live during the walk.
UPBP_D bool closest_hit(const TriView& tv, float3 o, float3 d, float tmin, float tmax, TriHit& hit, bool& overflow)
{
    bool found = false;
    float best = tmax;
    if (tv.bvh.count > 0) found = closest_triangle(tv, o, d, tmin, best, hit, overflow);
    for (int k = 0; kSceneSpheres && k < tv.sphere_count; k++) {
        float t1, t2;
        float3 n1, n2;
        if (!sphere_roots(__ldg(&tv.spheres[k]), o, d, t1, n1, t2, n2)) continue;
        if (t1 > tmin && t1 < best) {
            best = t1;
            sphere_hit(hit, t1, n1, k);
            found = true;
        } else if (t2 > tmin && t2 < best) {
            best = t2;
            sphere_hit(hit, t2, n2, k);
            found = true;
        }
    }
    if (kSceneSpheres) count_work(kCtrTris, (unsigned)tv.sphere_count);
    count_work(kCtrRays, 1u);
    return found;
}

// Every triangle hit with t in [tmin, tmax], then every sphere root with t in
// (tmin, tmax) (near root first: the reference's any-hit program ignores
// each hit, so both roots are reported); calls f(hit) for each, f returns
// false to stop.
template <class F>
UPBP_D bool all_hits(const TriView& tv, float3 o, float3 d, float tmin, float tmax, F&& f)
{
    const float3 inv = safe_inv(d);
    unsigned tests = 0;
    bool go = true;
    count_work(kCtrRays, 1u);
    const bool ok = bvh_walk(
        tv.bvh,
        [&](float3 lo, float3 hi) {
            const float3 t0 = (lo - o) * inv, t1 = (hi - o) * inv;
            const float n = fmaxf(fmaxf(fminf(t0.x, t1.x), fminf(t0.y, t1.y)), fmaxf(fminf(t0.z, t1.z), tmin));
            const float fa = fminf(fminf(fmaxf(t0.x, t1.x), fmaxf(t0.y, t1.y)), fminf(fmaxf(t0.z, t1.z), tmax));
            return n <= fa * 1.00001f + 1e-7f;
        },
        [&](int s) {
            float t, u, v;
            tests++;
            if (tri_intersect(tv.tri, s, o, d, t, u, v) && t >= tmin && t <= tmax) {
                TriHit h;
                h.t = t;
                h.u = u;
                h.v = v;
                h.prim = __float_as_int(__ldg(&tv.tri[3 * s]).w);
                go = f(h);
                return go;
            }
            return true;
        });
    for (int k = 0; kSceneSpheres && k < tv.sphere_count && go; k++) {
        float t1, t2;
        float3 n1, n2;
        tests++;
        if (!sphere_roots(__ldg(&tv.spheres[k]), o, d, t1, n1, t2, n2)) continue;
        TriHit h;
        if (t1 > tmin && t1 < tmax) {
            sphere_hit(h, t1, n1, k);
            go = f(h);
        }
        if (go && t2 > tmin && t2 < tmax) {
            sphere_hit(h, t2, n2, k);
            go = f(h);
        }
    }
    count_work(kCtrTris, tests);
    return ok;
}

}  // namespace upbp
