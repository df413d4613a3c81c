// Subpath state, recursive MIS quantities and the light-vertex / beam record
// packing.  The MIS recursion follows the reference's equations
// (gpuupbp/kernel/functs_shared.cuh:37-154 sample_scattering, Eq 4.47-4.49;
// path_weight.cuh:35-51 get_pde_factor, Eq 4.23).
#pragma once

#include "upbp_misdbg.cuh"
#include "upbp_trace.cuh"

namespace upbp {

struct VertexWeights {
    float d_shared, d_bpt, d_pde;
    float for_inv;     // 1 / pr_{T,i}
    float rev_inv;     // 1 / pl_{T,i-1}
    float for_ratio;   // prob_r{i} / pr_{T,i}
    float rev_ratio;   // prob_l{i} / pl_{T,i}
    bool prev_in_medium, prev_specular;
};

struct StateWeights {
    VertexWeights w;
    float last_sin_theta;
    float d_bpt_a, d_bpt_b, d_pde_a, d_pde_b;
};

struct PathState {
    BoundaryStack stack;
    float3 origin, dir, throughput;
    unsigned path_length;
    bool is_infinite_light;
    bool is_specular_path;
    StateWeights sw;
};

// f_i of Eq 4.23 for a subpath whose last vertex is i-1.
UPBP_D float pde_factor(bool in_medium, bool specular, float for_inv, float for_ratio, float rev_inv, float rev_ratio,
                        float sin_theta)
{
    const DeviceParams& p = c_params;
    const float fp = p.photon_beam_type == kLongBeam ? for_inv : for_ratio;
    const float rp = p.camera_beam_type == kLongBeam ? rev_inv : rev_ratio;
    return float(!in_medium && !specular) * p.mis_factor_surf +
           float(in_medium) * (p.mis_factor_pp3d + p.mis_factor_pb2d * rp + p.mis_factor_bp2d * fp +
                               p.mis_factor_bb1d * sin_theta * fp * rp);
}

// Direction sampling, Russian roulette and the MIS update at a vertex
// (functs_shared.cuh:37-154).  Returns a status; cont=false ends the walk.
UPBP_D unsigned sample_scattering(bool& cont, const Bsdf& bsdf, float3 hitpoint, const Isect& isect, PathState& s,
                                  Rng& rng)
{
    const float r0 = rng.uniform(), r1 = rng.uniform(), r2 = rng.uniform(), r3 = rng.uniform();
    float for_pdf, cos_out, sin_theta;
    unsigned ev;
    float3 dir;
    const float3 f = bsdf_sample(bsdf, r0, r1, r2, dir, for_pdf, cos_out, ev, sin_theta);
    s.dir = dir;
    if (is_black_or_negative(f)) {
        cont = false;
        return 0;
    }
    check_assert(for_pdf > 0.f);  // functs_shared.cuh:56
    const bool specular = (ev & (kEvReflect | kEvRefract)) != 0;
    float rev_pdf = for_pdf;
    if (!specular) rev_pdf = bsdf_pdf(bsdf, s.dir, true);
    const float cp = bsdf.cont_prob;
    if (cp == 0.f || (cp < 1.f && r3 > cp)) {
        cont = false;
        return 0;
    }
    for_pdf *= cp;
    rev_pdf *= cp;
    StateWeights& sw = s.sw;
    const float bpt_i_sub_1 = !sw.w.prev_specular && !specular;
    if (specular) {
        sw.d_bpt_a = cos_out / for_pdf;
        sw.d_bpt_b = cos_out * sw.w.d_bpt / sw.w.rev_inv;
        sw.d_pde_a = cos_out / for_pdf;
        sw.d_pde_b = cos_out * sw.w.d_pde / sw.w.rev_inv;
    } else {
        sw.d_bpt_a = cos_out / for_pdf;
        sw.d_bpt_b = (cos_out / for_pdf) * (sw.w.d_shared * bpt_i_sub_1 + rev_pdf * sw.w.d_bpt / sw.w.rev_inv);
        sw.d_pde_a = cos_out / for_pdf;
        sw.d_pde_b = (cos_out / for_pdf) * (sw.w.d_shared * bpt_i_sub_1 * c_params.subpath_count_bpt +
                                            rev_pdf * sw.w.d_pde / sw.w.rev_inv);
    }
    sw.w.d_shared = 1.f / for_pdf;
    s.is_specular_path = s.is_specular_path && specular;
    s.origin = hitpoint;
    s.throughput *= f * (cos_out / for_pdf);
    sw.w.prev_in_medium = bsdf.in_medium();
    sw.w.prev_specular = specular;
    sw.last_sin_theta = sin_theta;
    if (ev & kEvRefract) {
        if (update_stack_on_refract(isect, s.stack)) return kErrBoundaryStack;
    }
    cont = true;
    return 0;
}

UPBP_D float seg_for_pdf(const VolSeg* sg, int n)
{
    float p = 1.f;
    for (int i = 0; i < n; i++) p *= sg[i].pdf_for;
    return p;
}
UPBP_D float seg_rev_pdf(const VolSeg* sg, int n)
{
    float p = 1.f;
    for (int i = 0; i < n; i++) p *= sg[i].pdf_rev;
    return p;
}
UPBP_D float3 seg_attenuation(const VolSeg* sg, int n)
{
    float3 a = v3(1.f);
    for (int i = 0; i < n; i++) a *= sg[i].att;
    return a;
}

// ---------------------------------------------------------------- records

enum : unsigned { kVtxInMedium = 1u << 8, kVtxBehindSurf = 1u << 9 };

UPBP_D float ubits(unsigned u) { return __uint_as_float(u); }
UPBP_D unsigned fbits(float f) { return __float_as_uint(f); }

// frame_src is the vector the BSDF frame was built from (set_from_z input).
UPBP_D void store_vertex(LightVertexRec* rec, float3 hit, float3 thr, unsigned path_length, bool in_medium,
                         bool behind_surf, const Bsdf& b, float3 frame_src, const VertexWeights& w)
{
    const unsigned meta = (path_length & 0xffu) | (in_medium ? kVtxInMedium : 0u) | (behind_surf ? kVtxBehindSurf : 0u) |
                          ((unsigned)b.flags << 16);
    const unsigned ids = ((unsigned)b.id & 0x0fffffffu) | (w.prev_in_medium ? (1u << 28) : 0u) |
                         (w.prev_specular ? (1u << 29) : 0u);
    float4* q = rec->q;
    q[0] = make_float4(hit.x, hit.y, hit.z, ubits(meta));
    q[1] = make_float4(thr.x, thr.y, thr.z, b.cont_prob);
    q[2] = make_float4(w.d_shared, w.d_bpt, w.d_pde, w.for_inv);
    q[3] = make_float4(w.rev_inv, w.for_ratio, w.rev_ratio, ubits(ids));
    if (b.on_surface()) {
        q[4] = make_float4(frame_src.x, frame_src.y, frame_src.z, b.ior);
        q[5] = make_float4(b.local_dir_fix.x, b.local_dir_fix.y, b.local_dir_fix.z, b.cos_fix_geom);
        q[6] = make_float4(b.geom_normal.x, b.geom_normal.y, b.geom_normal.z, b.reflect_coeff);
        q[7] = make_float4(b.diff_prob, b.phong_prob, b.refl_prob, b.refr_prob);
    } else {
        q[4] = make_float4(frame_src.x, frame_src.y, frame_src.z, b.mean_cosine);
        q[5] = make_float4(b.world_dir_fix.x, b.world_dir_fix.y, b.world_dir_fix.z, 0.f);
        q[6] = make_float4(0.f, 0.f, 0.f, 0.f);
        q[7] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

struct LightVertex {
    float3 hit, thr;
    unsigned path_length;
    bool in_medium, behind_surf;
    Bsdf bsdf;
    VertexWeights w;
};

// A light-vertex record unpacked; q(i) returns float4 i of the record (read
// from global memory, or from registers after a warp's gather).
template <class Fetch>
UPBP_D void read_vertex(Fetch&& q, LightVertex& v)
{
    const float4 q0 = q(0), q1 = q(1), q2 = q(2), q3 = q(3);
    const float4 q4 = q(4), q5 = q(5);
    const unsigned meta = fbits(q0.w), ids = fbits(q3.w);
    v.hit = xyz(q0);
    v.thr = xyz(q1);
    v.path_length = meta & 0xffu;
    v.in_medium = (meta & kVtxInMedium) != 0;
    v.behind_surf = (meta & kVtxBehindSurf) != 0;
    v.w.d_shared = q2.x;
    v.w.d_bpt = q2.y;
    v.w.d_pde = q2.z;
    v.w.for_inv = q2.w;
    v.w.rev_inv = q3.x;
    v.w.for_ratio = q3.y;
    v.w.rev_ratio = q3.z;
    v.w.prev_in_medium = (ids >> 28) & 1u;
    v.w.prev_specular = (ids >> 29) & 1u;
    Bsdf& b = v.bsdf;
    b.flags = (int)(meta >> 16);
    b.id = (int)(ids & 0x0fffffffu);
    b.cont_prob = q1.w;
    b.frame.set_from_z(xyz(q4));
    if (b.on_surface()) {
        const float4 q6 = q(6), q7 = q(7);
        b.ior = q4.w;
        b.local_dir_fix = xyz(q5);
        b.cos_fix_geom = q5.w;
        b.geom_normal = xyz(q6);
        b.reflect_coeff = q6.w;
        b.diff_prob = q7.x;
        b.phong_prob = q7.y;
        b.refl_prob = q7.z;
        b.refr_prob = q7.w;
        b.gcell = -1;
    } else {
        const DMedium& m = c_params.media[b.id];
        b.mean_cosine = q4.w;
        b.world_dir_fix = xyz(q5);
        b.scatter_coef = m.scattering;
        b.scatter_pos = !is_black_or_negative(m.scattering);
        b.gcell = guide_cell(c_params.guide, v.hit, b.id);
    }
}

UPBP_D void load_vertex(const LightVertexRec* rec, LightVertex& v)
{
    read_vertex([&](int i) { return __ldg(&rec->q[i]); }, v);
}


struct Beam {
    float3 o, d;
    float length;
    int med;
    float3 thr;
    float for_pdf, rev_pdf;
    unsigned flags, path_idx, path_length;
    bool infinite;
    float origin_offset;  // distance from the light vertex that traced the ray to the beam's origin
    StateWeights sw;
};

UPBP_D void store_beam(BeamRec* rec, const Beam& b)
{
    float4* q = rec->q;
    const VertexWeights& w = b.sw.w;
    const unsigned bits = (w.prev_in_medium ? 1u : 0u) | (w.prev_specular ? 2u : 0u) | (b.infinite ? 4u : 0u);
    q[0] = make_float4(b.o.x, b.o.y, b.o.z, b.length);
    q[1] = make_float4(b.d.x, b.d.y, b.d.z, ubits((unsigned)b.med));
    q[2] = make_float4(b.thr.x, b.thr.y, b.thr.z, b.for_pdf);
    q[3] = make_float4(b.rev_pdf, ubits(b.flags), ubits(b.path_idx), ubits(b.path_length));
    q[4] = make_float4(w.d_shared, w.d_bpt, w.d_pde, w.for_inv);
    q[5] = make_float4(w.rev_inv, w.for_ratio, w.rev_ratio, ubits(bits));
    q[6] = make_float4(b.sw.last_sin_theta, b.sw.d_bpt_a, b.sw.d_bpt_b, b.sw.d_pde_a);
    q[7] = make_float4(b.sw.d_pde_b, b.origin_offset, 0.f, 0.f);
}

// A beam record unpacked; q(i) returns float4 i of the record.
template <class Fetch>
UPBP_D void read_beam(Fetch&& q, Beam& b)
{
    const float4 q0 = q(0), q1 = q(1), q2 = q(2), q3 = q(3);
    const float4 q4 = q(4), q5 = q(5), q6 = q(6), q7 = q(7);
    b.o = xyz(q0);
    b.length = q0.w;
    b.d = xyz(q1);
    b.med = (int)fbits(q1.w);
    b.thr = xyz(q2);
    b.for_pdf = q2.w;
    b.rev_pdf = q3.x;
    b.flags = fbits(q3.y);
    b.path_idx = fbits(q3.z);
    b.path_length = fbits(q3.w);
    b.sw.w.d_shared = q4.x;
    b.sw.w.d_bpt = q4.y;
    b.sw.w.d_pde = q4.z;
    b.sw.w.for_inv = q4.w;
    b.sw.w.rev_inv = q5.x;
    b.sw.w.for_ratio = q5.y;
    b.sw.w.rev_ratio = q5.z;
    const unsigned bits = fbits(q5.w);
    b.sw.w.prev_in_medium = bits & 1u;
    b.sw.w.prev_specular = (bits >> 1) & 1u;
    b.infinite = (bits >> 2) & 1u;
    b.sw.last_sin_theta = q6.x;
    b.sw.d_bpt_a = q6.y;
    b.sw.d_bpt_b = q6.z;
    b.sw.d_pde_a = q6.w;
    b.sw.d_pde_b = q7.x;
    b.origin_offset = q7.y;
}

UPBP_D void load_beam(const BeamRec* rec, Beam& b)
{
    read_beam([&](int i) { return __ldg(&rec->q[i]); }, b);
}

// ---------------------------------------------------------------- exact predicates
// Evaluated with round-to-nearest intrinsics so no multiply-add is fused:
// the accept/reject decision is bit-identical to a plain IEEE evaluation of
// the same expressions (the brute-force neighbour oracle).  Expressions follow
// gpuupbp/kernel/intersection.cuh:33-173.

UPBP_D float dot_rn(float3 a, float3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
UPBP_D float3 sub_rn(float3 a, float3 b) { return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
UPBP_D float3 axpy_rn(float3 o, float3 d, float t)
{
    return make_float3(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)), __fadd_rn(o.z, __fmul_rn(d.z, t)));
}
UPBP_D float3 cross_rn(float3 a, float3 b)
{
    return make_float3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                       __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

UPBP_D bool pred_point_point(float3 a, float3 b, float r2)
{
    const float3 d = sub_rn(a, b);
    return dot_rn(d, d) <= r2;
}

// Query ray (o, d) on (tmin, tmax) vs a disc of squared radius r2 at p.
UPBP_D bool pred_ray_disc(float3 o, float3 d, float tmin, float tmax, float3 p, float r2, float& dist, float& rad2)
{
    const float3 v = sub_rn(p, o);
    const float t = dot_rn(v, d);
    if (!(t > tmin && t < tmax)) return false;
    const float3 e = sub_rn(axpy_rn(o, d, t), p);
    const float h = dot_rn(e, e);
    if (!(h <= r2)) return false;
    dist = t;
    rad2 = h;
    return true;
}

// Two beams (test_intersection_beam_beam with the trimmed pre-filter).
UPBP_D bool pred_beam_beam(float3 o1, float3 d1, float min1, float max1, float3 o2, float3 d2, float max2, float r2,
                           float& distance, float& sin_theta, float& t1, float& t2)
{
    const float3 c = cross_rn(d1, d2);
    const float s2 = dot_rn(c, c);
    const float ad = dot_rn(sub_rn(o2, o1), c);
    if (__fmul_rn(ad, ad) >= __fmul_rn(r2, s2)) return false;
    const float dd = dot_rn(d1, d2);
    const float dd2m1 = __fsub_rn(__fmul_rn(dd, dd), 1.f);
    if (dd2m1 < 1e-5f && dd2m1 > -1e-5f) return false;
    const float d1o1 = dot_rn(d1, o1), d1o2 = dot_rn(d1, o2);
    t1 = __fdiv_rn(__fsub_rn(__fsub_rn(d1o1, d1o2), __fmul_rn(dd, __fsub_rn(dot_rn(d2, o1), dot_rn(d2, o2)))), dd2m1);
    if (t1 <= min1 || t1 >= max1) return false;
    t2 = __fdiv_rn(__fsub_rn(__fadd_rn(t1, d1o1), d1o2), dd);
    if (t2 <= 0.f || t2 >= max2 || isnan(t2)) return false;
    sin_theta = __fsqrt_rn(s2);
    distance = __fdiv_rn(fabsf(ad), sin_theta);
    return true;
}

}  // namespace upbp
