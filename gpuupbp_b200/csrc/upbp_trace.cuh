// Media-aware ray casting: the closest real surface behind any low-priority
// boundaries, the imaginary (medium-boundary) crossings in distance order, the
// split of the ray into per-medium segments, and free-flight sampling.
// Semantics follow the reference's intersect_ (gpuupbp/kernel/intersector.cuh:45-371)
// including its priority-stack rules and bounded arrays
// (MAX_VOLUME_SEGMENTS 10, MAX_INTERSECTIONS 10, MAX_STACK_ELEMENT 20,
// MAX_IMAGINARY_INTERSECTIONS 8 in kernel/defs.cuh:53-70): an overflow makes
// the sample fail with the matching status bit instead of faulting.
#pragma once

#include "upbp_bvh.cuh"
#include "upbp_shading.cuh"

namespace upbp {

constexpr int kMaxVolSegments = 10;
constexpr int kMaxRealHits = 10;
constexpr int kMaxStack = 20;
constexpr int kMaxImagHits = 8;

enum : unsigned { kSampleScattering = 1u << 1, kOcclusionTest = 1u << 2 };

struct Boundary {
    int mat, med;
};

// Priority stack of crossed boundaries (element order: ascending priority,
// ties keep insertion order; top = last).
struct BoundaryStack {
    int size;
    Boundary el[kMaxStack];
    int pri[kMaxStack];

    UPBP_D void clear() { size = 0; }
    UPBP_D bool push(Boundary b, int p)
    {
        if (size == kMaxStack) return false;
        int i = size - 1;
        while (i >= 0 && pri[i] > p) {
            el[i + 1] = el[i];
            pri[i + 1] = pri[i];
            i--;
        }
        el[i + 1] = b;
        pri[i + 1] = p;
        size++;
        return true;
    }
    UPBP_D bool pop(Boundary b, int p)
    {
        for (int i = size - 1; i >= 0 && pri[i] >= p; i--) {
            if (pri[i] == p && el[i].mat == b.mat && el[i].med == b.med) {
                for (int j = i; j < size - 1; j++) {
                    el[j] = el[j + 1];
                    pri[j] = pri[j + 1];
                }
                size--;
                return true;
            }
        }
        return false;
    }
    UPBP_D void pop_top() { size--; }
    UPBP_D const Boundary& top() const { return el[size - 1]; }
    UPBP_D int top_priority() const { return pri[size - 1]; }
    UPBP_D const Boundary& second() const { return el[size - 2]; }
};

struct LiteHit {
    float dist;
    int mat, med;
    int enter;
};

struct VolSeg {
    float3 att;
    float3 emis;
    float dmin, dmax;
    float pdf_for, pdf_rev;
    int med;
};

struct LiteSeg {
    float dmin, dmax;
    int med;
};

struct Isect {
    float dist;
    int mat, med, light;
    float3 normal;
    float3 shading_normal;
    bool enter;
    UPBP_D bool on_surface() const { return mat >= 0; }
    UPBP_D bool in_medium() const { return mat < 0; }
};

UPBP_D int boundary_priority(int mat) { return mat >= 0 ? c_params.materials[mat].priority : kGlobalMediumPriority; }

UPBP_D bool is_real_material(int mat) { return mat >= 0 && c_params.materials[mat].real; }

// Sets an iteration's status bits; with -assert also counts the event under
// its lowest bit (the reference's exception program prints one line per
// such event, kernel/exception.cu:27-52).
UPBP_D void flag_status(unsigned bits)
{
    atomicOr(c_params.status, bits);
    if (c_params.assert_counts && bits) atomicAdd(&c_params.assert_counts[__ffs(bits)], 1u);
}

// The reference's GPU_ASSERT (kernel/defs.cuh:90-96) with -assert: counts a
// failed condition.  The reference's exception also ends the launch index;
// here the path goes on, so the images with and without -assert agree.
UPBP_D void check_assert(bool cond)
{
    if (!cond && c_params.assert_counts) atomicAdd(&c_params.assert_counts[0], 1u);
}

// A sphere normal component as the reference's closest-hit and any-hit
// programs read it back from the hit attributes (intersector.cu:130-132): the
// attribute word holds the component's bits, __float_as_int is applied to the
// word, so the word is first converted to float by value, and the int read
// from that float's bits becomes the component.  The result is large and
// positive for every nonzero component instead of the unit normal; it decides
// `enter` and the shading frame at sphere hits, so it is kept for parity.
UPBP_D float sphere_attribute_component(float x)
{
    return __int2float_rn(__float_as_int(__uint2float_rn(__float_as_uint(x))));
}

// Fills surface data of a triangle or sphere hit (intersector.cu fill_isect;
// a sphere's shading normal is its normal and it is no emitter).
UPBP_D void fill_hit(const TriView& tv, const TriHit& h, float3 ray_dir, Isect& r)
{
    if (kSceneSpheres && h.prim < 0) {
        const int mat = __ldg(&tv.sph_mat[~h.prim]);
        const float3 nrm = make_float3(sphere_attribute_component(h.u), sphere_attribute_component(h.v),
                                       sphere_attribute_component(h.w));
        r.dist = h.t;
        r.mat = mat;
        r.med = c_params.materials[mat].medium;
        r.light = -1;
        r.normal = nrm;
        r.enter = dot(nrm, ray_dir) < 0.f;
        r.shading_normal = nrm;
        return;
    }
    const float4* n = tv.normals + 4 * (size_t)h.prim;
    const float3 face = xyz(__ldg(&n[3]));
    float3 sn;
    if (c_params.use_shading_normal) {
        const float3 n0 = xyz(__ldg(&n[0])), n1 = xyz(__ldg(&n[1])), n2 = xyz(__ldg(&n[2]));
        sn = normalize(n0 * (1.f - h.u - h.v) + n1 * h.u + n2 * h.v);
    } else {
        sn = face;
    }
    const int2 rec = __ldg(&tv.record[h.prim]);
    r.dist = h.t;
    r.mat = rec.x;
    r.med = c_params.materials[rec.x].medium;
    r.light = rec.y;
    r.normal = face;
    r.enter = dot(face, ray_dir) < 0.f;
    r.shading_normal = sn;
}

UPBP_D bool init_boundary_stack(BoundaryStack& s)
{
    s.clear();
    return s.push(Boundary{-1, c_params.global_medium}, kGlobalMediumPriority);
}

// Casts a ray through the scene.  On return `hit` tells whether a surface or
// a medium scattering point was found (result.dist), `segs` holds the medium
// segments up to that point (with sampling pdfs) and `lsegs` the segments up
// to the next real surface.  Returns a status bit (0 on success).
// Kept out of line: inlined into every caller it made the path kernels too large
// for the instruction cache.
__device__ __noinline__ unsigned intersect_scene(bool& hit, float3 ro, float3 rd, Isect& result, BoundaryStack& bstack,
                                unsigned options, unsigned sflags, VolSeg* segs, int& nseg, LiteSeg* lsegs,
                                int& nlseg, Rng& rng)
{
    hit = false;
    const bool occlusion = (options & kOcclusionTest) != 0;
    const bool sample_media = (options & kSampleScattering) != 0 && !occlusion;

    Isect tmp = result;
    float dist = 0.f;

    LiteHit real_hits[kMaxRealHits];
    int n_real = 0;
    const int top_priority = bstack.top_priority();
    const float first_eps = (sflags & kOriginInMedium) ? 0.f : kEpsRay;
    float t_max, miss_dist;
    if (occlusion) {
        t_max = tmp.dist - kEpsRay;
        miss_dist = tmp.dist;
    } else {
        t_max = kInfinity;
        miss_dist = kInfinity;
    }

    BoundaryStack scopy = bstack;
    float t_min = first_eps;
    bool not_yet_real;
    do {
        not_yet_real = false;
        tmp.dist = kInfinity;
        TriHit th;
        bool ovf = false;
        if (closest_hit(c_params.real, ro, rd, t_min, t_max, th, ovf)) fill_hit(c_params.real, th, rd, tmp);
        if (ovf) flag_status(kErrTraversalStack);
        hit = tmp.dist != kInfinity;
        if (hit) {
            dist = tmp.dist;
            const int priority = boundary_priority(tmp.mat);
            const Boundary top = scopy.top();
            if (tmp.med < 0) tmp.med = top.med;
            if (priority < top_priority && priority != kThinWallPriority) {
                const Boundary e{tmp.mat, tmp.med};
                if (tmp.enter) {
                    if (n_real == kMaxRealHits) return kErrIntersectionArray;
                    real_hits[n_real++] = LiteHit{tmp.dist, tmp.mat, tmp.med, 1};
                    if (!scopy.push(e, priority)) return kErrBoundaryStack;
                } else if (scopy.pop(e, priority)) {
                    if (n_real == kMaxRealHits) return kErrIntersectionArray;
                    real_hits[n_real++] = LiteHit{tmp.dist, tmp.mat, tmp.med, 0};
                }
                not_yet_real = true;
                t_min = dist + kEpsRay;
                // the reference shrinks an occlusion query by the skipped distance
                // twice (intersector.cuh:167-170); kept for parity
                t_max = occlusion ? miss_dist - dist - kEpsRay : kInfinity;
            }
        }
    } while (not_yet_real && t_max > t_min);

    if (!hit || not_yet_real) {
        hit = false;
        dist = miss_dist;
    }
    result = tmp;
    result.dist = dist;

    // imaginary boundaries before the real hit
    bool scattered = false;
    LiteHit imag[kMaxImagHits];
    int n_imag = -1;
    if (!is_real_material(bstack.top().mat) && dist > first_eps + kEpsRay) {
        n_imag = 0;
        bool overflow = false;
        const bool ok = all_hits(c_params.imag, ro, rd, first_eps, dist - kEpsRay, [&](const TriHit& h) {
            Isect ih;
            fill_hit(c_params.imag, h, rd, ih);
            if (n_imag == kMaxImagHits) {
                overflow = true;
                return false;
            }
            // sorted insert by distance, after equal distances
            int i = n_imag - 1;
            while (i >= 0 && imag[i].dist > ih.dist) {
                imag[i + 1] = imag[i];
                i--;
            }
            imag[i + 1] = LiteHit{ih.dist, ih.mat, ih.med, ih.enter ? 1 : 0};
            n_imag++;
            return true;
        });
        if (!ok) flag_status(kErrTraversalStack);
        if (overflow) return kErrIntersectionStack;

        scopy = bstack;
        float dmin = 0.f;
        for (int i = 0; i < n_imag; i++) {
            const LiteHit& ih = imag[i];
            const int pr = boundary_priority(ih.mat);
            const Boundary e{ih.mat, ih.med};
            if (ih.enter) {
                if (pr >= scopy.top_priority()) {
                    if (nlseg == kMaxVolSegments) return kErrVolSegmentArray;
                    lsegs[nlseg++] = LiteSeg{dmin, ih.dist, scopy.top().med};
                    dmin = ih.dist;
                }
                if (!scopy.push(e, pr)) return kErrBoundaryStack;
            } else {
                if (pr == scopy.top_priority() && e.mat == scopy.top().mat && e.med == scopy.top().med) {
                    if (nlseg == kMaxVolSegments) return kErrVolSegmentArray;
                    lsegs[nlseg++] = LiteSeg{dmin, ih.dist, scopy.top().med};
                    dmin = ih.dist;
                }
                scopy.pop(e, pr);
            }
        }
        if (dmin < dist) {
            if (nlseg == kMaxVolSegments) return kErrVolSegmentArray;
            lsegs[nlseg++] = LiteSeg{dmin, dist, scopy.top().med};
        }
    } else {
        if (nlseg == kMaxVolSegments) return kErrVolSegmentArray;
        lsegs[nlseg++] = LiteSeg{0.f, dist, bstack.top().med};
    }

    const bool origin_in_medium = (sflags & kOriginInMedium) != 0;
    const bool end_in_medium = (sflags & kEndInMedium) != 0;
    int popped = 0;
    for (int i = 0; i < nlseg; i++) {
        const LiteSeg sg = lsegs[i];
        const int cur = sg.med;
        if (cur < 0) continue;
        const DMedium& m = c_params.media[min(cur, c_params.medium_count - 1)];
        unsigned f = 0;
        if (origin_in_medium && sg.dmin == 0.f) f |= kOriginInMedium;
        if (end_in_medium && sg.dmax == dist) f |= kEndInMedium;
        float pf = 1.f, pr = 1.f;
        float dmax = sg.dmax;
        if (m.has_scattering) {
            if (sample_media) {
                float u;
                do {
                    u = rng.uniform();
                } while (u == 0.f);
                const float span = sg.dmax - sg.dmin;
                const float s = sample_distance(m, span, u, pf, f, pr);
                if (s < span) {
                    result.dist = sg.dmin + s;
                    result.mat = -1;
                    result.med = cur;
                    result.light = -1;
                    result.normal = v3(0.f);
                    result.enter = false;
                    hit = true;
                    scattered = true;
                    dmax = result.dist;
                }
            } else {
                pf = distance_pdf(m, sg.dmin, sg.dmax, f, pr);
            }
        }
        if (nseg == kMaxVolSegments) return kErrVolSegmentArray;
        segs[nseg++] = VolSeg{attenuation(m, dmax - sg.dmin), emission(m, sg.dmin, dmax), sg.dmin, dmax, pf, pr, cur};

        if (n_imag >= 0) {
            for (int j = popped; j < n_imag; j++) {
                const LiteHit& ih = imag[j];
                if (ih.dist > dmax) break;
                if (ih.enter) {
                    if (!bstack.push(Boundary{ih.mat, ih.med}, boundary_priority(ih.mat))) return kErrBoundaryStack;
                } else if (bstack.size > 1) {
                    bstack.pop(Boundary{ih.mat, ih.med}, boundary_priority(ih.mat));
                }
                popped++;
            }
        }
        if (scattered) break;
    }

    for (int j = 0; j < n_real; j++) {
        const LiteHit& h = real_hits[j];
        if (h.dist > result.dist) break;
        if (h.enter) {
            if (!bstack.push(Boundary{h.mat, h.med}, boundary_priority(h.mat))) return kErrBoundaryStack;
        } else if (bstack.size > 1) {
            bstack.pop(Boundary{h.mat, h.med}, boundary_priority(h.mat));
        }
    }
    return 0;
}

// Occlusion query from `p` toward `dir` up to t_max (intersector.cuh:375-397).
UPBP_D unsigned occluded(bool& hit, float3 p, float3 dir, float t_max, const BoundaryStack& bstack, unsigned sflags,
                         VolSeg* segs, int& nseg, Rng& rng)
{
    BoundaryStack scopy = bstack;
    Isect tmp;
    tmp.dist = t_max;
    tmp.mat = tmp.med = tmp.light = -1;
    tmp.normal = v3(0.f);
    tmp.enter = false;
    LiteSeg lsegs[kMaxVolSegments];
    int nl = 0;
    nseg = 0;
    return intersect_scene(hit, p, dir, tmp, scopy, kOcclusionTest, sflags, segs, nseg, lsegs, nl, rng);
}

UPBP_D float relative_ior(const Isect& is, const BoundaryStack& st)
{
    if (!is.on_surface()) return -1.f;
    const DMaterial& m1 = c_params.materials[is.mat];
    const float ior1 = m1.ior;
    if (ior1 < 0.f) return -1.f;
    float ior2 = 1.f;
    if (is.enter) {
        const int mid = st.top().mat;
        if (mid >= 0 && c_params.materials[mid].real) ior2 = c_params.materials[mid].ior;
        return ior2 < 0.f ? -1.f : ior2 / ior1;
    }
    const int mid = st.size > 1 ? st.second().mat : st.top().mat;
    if (mid >= 0 && c_params.materials[mid].real) ior2 = c_params.materials[mid].ior;
    return ior2 < 0.f ? -1.f : ior1 / ior2;
}

UPBP_D unsigned update_stack_on_refract(const Isect& is, BoundaryStack& st)
{
    if (is.enter) {
        if (is.med >= 0 && !st.push(Boundary{is.mat, is.med}, boundary_priority(is.mat))) return kErrBoundaryStack;
    } else if (st.size > 1) {
        st.pop_top();
    }
    return 0;
}

}  // namespace upbp
