// Scattering models, media, lights and camera mapping.  Every formula follows
// the reference's device code so that, fed the same random numbers, a path
// takes the same decisions:
//   sampling warps        gpuupbp/kernel/sample.cuh:31-205
//   HG phase function     gpuupbp/kernel/phase_function.cuh:34-137
//   homogeneous media     gpuupbp/kernel/medium.cuh:33-171
//   surface BSDF          gpuupbp/kernel/bsdf.cuh:61-660
//   lights                gpuupbp/kernel/light.cuh:38-543
//   camera                gpuupbp/kernel/camera.cuh:33-76
#pragma once

#include "upbp_device.cuh"
#include "upbp_guide.cuh"

namespace upbp {

// ---------------------------------------------------------------- warps

UPBP_D float3 sample_cos_hemisphere(float u0, float u1, float* pdf)
{
    const float phi = 2.f * kPi * u0;
    const float r = sqrtf(u1);
    float3 d = make_float3(cosf(phi) * r, sinf(phi) * r, sqrtf(1.f - u1));
    if (pdf) *pdf = d.z * kInvPi;
    return d;
}

UPBP_D float3 sample_power_cos_hemisphere(float u0, float u1, float power)
{
    const float phi = 2.f * kPi * u0;
    const float ct = powf(u1, 1.f / (power + 1.f));
    const float st = sqrtf(1.f - ct * ct);
    return make_float3(cosf(phi) * st, sinf(phi) * st, ct);
}

UPBP_D float power_cos_hemisphere_pdf(float3 n, float3 d, float power)
{
    const float c = fmaxf(0.f, dot(n, d));
    return (power + 1.f) * powf(c, power) * (kInvPi * .5f);
}

UPBP_D float3 sample_uniform_sphere(float u0, float u1, float* pdf)
{
    const float phi = 2.f * kPi * u0;
    const float s = 2.f * sqrtf(u1 - u1 * u1);
    if (pdf) *pdf = kInvPi * .25f;
    return make_float3(cosf(phi) * s, sinf(phi) * s, 1.f - 2.f * u1);
}

UPBP_D float uniform_sphere_pdf() { return kInvPi * .25f; }

UPBP_D float2 sample_concentric_disc(float u0, float u1)
{
    float phi, r;
    const float a = 2.f * u0 - 1.f, b = 2.f * u1 - 1.f;
    if (a > -b) {
        if (a > b) {
            r = a;
            phi = (kPi / 4.f) * (b / a);
        } else {
            r = b;
            phi = (kPi / 4.f) * (2.f - (a / b));
        }
    } else {
        if (a < b) {
            r = -a;
            phi = (kPi / 4.f) * (4.f + (b / a));
        } else {
            r = -b;
            phi = b != 0.f ? (kPi / 4.f) * (6.f - (a / b)) : 0.f;
        }
    }
    return make_float2(r * cosf(phi), r * sinf(phi));
}

UPBP_D float fresnel_dielectric(float cos_inc, float ior)
{
    if (ior < 0.f) return 1.f;
    if (cos_inc < 0.f) cos_inc = -cos_inc;
    const float sin_t2 = ior * ior * (1.f - cos_inc * cos_inc);
    const float cos_t = sqrtf(fmaxf(0.f, 1.f - sin_t2));
    const float t1 = ior * cos_t;
    const float r_par = (cos_inc - t1) / (cos_inc + t1);
    const float t2 = ior * cos_inc;
    const float r_perp = (t2 - cos_t) / (t2 + cos_t);
    return .5f * (r_par * r_par + r_perp * r_perp);
}

UPBP_D float pdf_w_to_a(float pdf_w, float dist, float cos_there) { return pdf_w * fabsf(cos_there) / (dist * dist); }

// ---------------------------------------------------------------- HG phase

UPBP_D float hg_pdf(float3 dir_fix, float3 dir_gen, float g, float* sin_theta)
{
    const float ct = -dot(dir_gen, dir_fix);
    if (sin_theta) *sin_theta = sqrtf(fmaxf(0.f, 1.f - ct * ct));
    if (fabsf(g) < 1e-3f) return uniform_sphere_pdf();
    const float g2 = g * g;
    const float d = 1.f + g2 - (g + g) * ct;
    return d > 0.f ? uniform_sphere_pdf() * (1.f - g2) / (d * sqrtf(d)) : 0.f;
}

// Samples around frame.z (= -dir_fix).  Returns the pdf as the phase value.
UPBP_D float hg_sample(float3 dir_fix, float g, float u0, float u1, const Frame& frame, float3& dir_gen, float& pdf,
                       float* sin_theta)
{
    if (fabsf(g) < 1e-3f) {
        dir_gen = sample_uniform_sphere(u0, u1, &pdf);
        if (sin_theta) {
            const float ct = -dot(dir_gen, dir_fix);
            *sin_theta = sqrtf(fmaxf(0.f, 1.f - ct * ct));
        }
    } else {
        const float g2 = g * g, two_g = g + g;
        const float s = (1.f - g2) / (1.f - g + two_g * u0);
        const float ct = (1.f + g2 - s * s) / two_g;
        const float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
        const float phi = 2.f * kPi * u1;
        const float d = 1.f + g2 - two_g * ct;
        dir_gen = frame.to_world(make_float3(cosf(phi) * st, sinf(phi) * st, ct));
        pdf = d > 0.f ? (uniform_sphere_pdf() * (1.f - g2) / (d * sqrtf(d))) : 0.f;
        if (sin_theta) *sin_theta = st;
    }
    return pdf;
}

// ---------------------------------------------------------------- media

UPBP_D float3 attenuation(const DMedium& m, float dist)
{
    return make_float3(expf(-m.attenuation.x * dist), expf(-m.attenuation.y * dist), expf(-m.attenuation.z * dist));
}

UPBP_D float3 emission(const DMedium& m, float dmin, float dmax)
{
    const float d = dmax - dmin;
    return m.emission * d;
}

// Free-flight sample within [0, dist_to_boundary]; see medium.cuh:64-119.
UPBP_D float sample_distance(const DMedium& m, float dist_to_boundary, float rnd, float& for_pdf, unsigned flags,
                             float& rev_pdf)
{
    if (m.min_pos_att != 0.f && m.has_scattering) {
        const float s = -logf(rnd) / m.min_pos_att;
        if (s < dist_to_boundary) {
            const float att = expf(-m.min_pos_att * s);
            for_pdf = m.min_pos_att * att;
            rev_pdf = (flags & kOriginInMedium) ? for_pdf : att;
            return s;
        }
        const float att = expf(-m.min_pos_att * dist_to_boundary);
        for_pdf = att;
        rev_pdf = (flags & kOriginInMedium) ? m.min_pos_att * att : att;
        return dist_to_boundary;
    }
    for_pdf = 1.f;
    rev_pdf = 1.f;
    return dist_to_boundary;
}

// Pdf of sampling along [dmin, dmax]; see medium.cuh:126-156.
UPBP_D float distance_pdf(const DMedium& m, float dmin, float dmax, unsigned flags, float& rev_pdf)
{
    float for_pdf = 1.f;
    rev_pdf = 1.f;
    if (m.min_pos_att != 0.f && m.has_scattering) {
        const float att = fmaxf(expf(-m.min_pos_att * (dmax - dmin)), 1e-35f);
        const float minatt = fmaxf(m.min_pos_att * att, 1e-35f);
        for_pdf = (flags & kEndInMedium) ? minatt : att;
        rev_pdf = (flags & kOriginInMedium) ? minatt : att;
    }
    return for_pdf;
}

// ---------------------------------------------------------------- BSDF

enum : int { kBsdfInMedium = 1, kBsdfFromLight = 2, kBsdfValid = 4, kBsdfDelta = 8 };
enum : unsigned { kEvDiffuse = 1, kEvPhong = 2, kEvReflect = 4, kEvRefract = 8, kEvScatter = 16 };

struct Bsdf {
    Frame frame;
    float cont_prob;
    int flags;
    int id;                  // material (surface) or medium index
    // surface
    float3 local_dir_fix;
    float3 geom_normal;      // local
    float cos_fix_geom;
    float reflect_coeff;
    float diff_prob, phong_prob, refl_prob, refr_prob;
    float ior;
    // medium
    float3 world_dir_fix;
    float mean_cosine;
    float3 scatter_coef;
    bool scatter_pos;
    int gcell;               // learned-proposal cell of a medium vertex (-1: phase function only)

    UPBP_D bool valid() const { return flags & kBsdfValid; }
    UPBP_D bool delta() const { return flags & kBsdfDelta; }
    UPBP_D bool in_medium() const { return flags & kBsdfInMedium; }
    UPBP_D bool on_surface() const { return !(flags & kBsdfInMedium); }
    UPBP_D bool from_light() const { return flags & kBsdfFromLight; }
    UPBP_D float cos_fix() const { return local_dir_fix.z; }
    UPBP_D float d_factor() const { return on_surface() ? fabsf(local_dir_fix.z) : 1.f; }
    UPBP_D float3 dir_fix() const { return on_surface() ? frame.to_world(local_dir_fix) : world_dir_fix; }
};

// Pdf of a camera subpath scattering at a medium vertex from direction of
// travel `travel` into `out`: the blend (1 - a) hg + a mixture of the phase
// function (value hg) and the learned mixture, a the table entry's
// selection probability, or hg where the vertex is not guided.
// Kept out of line: the unguided callers, the common case, pay only the
// test of the cell.
__device__ __noinline__ float guide_mix(int cell, float3 travel, float3 out, float hg)
{
    const float4* e = guide_entry(c_params.guide, cell, travel);
    if (!e) return hg;
    const float a = guide_entry_alpha(e);
    return (1.f - a) * hg + a * vmf_mix_pdf(e, out);
}

UPBP_D float guide_pdf(const Bsdf& b, float3 travel, float3 out, float hg)
{
    return b.gcell < 0 ? hg : guide_mix(b.gcell, travel, out, hg);
}

// The same at a point of medium `med` that is not a vertex (a query beam's
// merge point).
__device__ __noinline__ float guide_mix_at(float3 x, int med, float3 travel, float3 out, float hg)
{
    return guide_mix(guide_cell(c_params.guide, x, med), travel, out, hg);
}

UPBP_D float guide_pdf_at(float3 x, int med, float3 travel, float3 out, float hg)
{
    return c_params.guide.entries ? guide_mix_at(x, med, travel, out, hg) : hg;
}

// Samples the blend of the phase function and the learned mixture: r2 picks
// the mixture with the entry's selection probability a (and, rescaled, the
// mixture's lobe), the phase function otherwise.
__device__ __noinline__ float3 guide_sample(const Bsdf& b, float r0, float r1, float r2, float3& dir_gen, float& pdf,
                                            float& sin_theta)
{
    const float4* e = guide_entry(c_params.guide, b.gcell, -b.world_dir_fix);
    const float a = e ? guide_entry_alpha(e) : 0.f;
    if (!e || r2 >= a) {
        hg_sample(b.world_dir_fix, b.mean_cosine, r0, r1, b.frame, dir_gen, pdf, &sin_theta);
        if (!e) return b.scatter_coef * pdf;
    } else {
        dir_gen = vmf_mix_sample(e, r2 / a, r0, r1);
    }
    const float p = hg_pdf(b.world_dir_fix, dir_gen, b.mean_cosine, &sin_theta);
    pdf = (1.f - a) * p + a * vmf_mix_pdf(e, dir_gen);
    return b.scatter_coef * p;
}

UPBP_D void bsdf_component_probs(Bsdf& b, const DMaterial& m)
{
    b.reflect_coeff = fresnel_dielectric(b.local_dir_fix.z, b.ior);
    const float ad = luminance(m.diffuse);
    const float ap = luminance(m.phong);
    const float ar = b.reflect_coeff * luminance(m.mirror);
    const float at = (1.f - b.reflect_coeff) * (m.ior > 0.f ? 1.f : 0.f);
    const float total = ad + ap + ar + at;
    if (total < 1e-9f) {
        b.diff_prob = b.phong_prob = b.refl_prob = b.refr_prob = 0.f;
        b.cont_prob = 0.f;
        return;
    }
    b.diff_prob = ad / total;
    b.phong_prob = ap / total;
    b.refl_prob = ar / total;
    b.refr_prob = at / total;
    const float3 tmp = m.diffuse + m.phong + b.reflect_coeff * m.mirror;
    b.cont_prob = max_component(tmp) + (1.f - b.reflect_coeff);
    b.cont_prob = fminf(1.f, fmaxf(0.f, b.cont_prob));
}

// Surface setup (bsdf.cuh:179-223, surface branch).
UPBP_D void bsdf_setup_surface(Bsdf& b, float3 ray_dir, float3 normal, float3 shading_normal, int mat_id,
                               bool from_light, float ior)
{
    b.flags = from_light ? kBsdfFromLight : 0;
    b.gcell = -1;
    const DMaterial& m = c_params.materials[mat_id];
    b.id = mat_id;
    b.frame.set_from_z(shading_normal);
    b.local_dir_fix = b.frame.to_local(-ray_dir);
    b.geom_normal = b.frame.to_local(normal);
    b.cos_fix_geom = dot(b.local_dir_fix, b.geom_normal);
    if (fabsf(b.local_dir_fix.z) < kEpsCosine || fabsf(b.cos_fix_geom) < kEpsCosine) {
        b.flags = 0;
        return;
    }
    b.ior = ior;
    bsdf_component_probs(b, m);
    if (b.diff_prob == 0.f && b.phong_prob == 0.f) b.flags |= kBsdfDelta;
    b.flags |= kBsdfValid;
}

UPBP_D void bsdf_setup_medium(Bsdf& b, float3 ray_dir, int med_id, bool from_light, float3 x)
{
    b.flags = (from_light ? kBsdfFromLight : 0) | kBsdfInMedium;
    const int idx = min(med_id, c_params.medium_count - 1);
    const DMedium& m = c_params.media[idx];
    b.id = idx;
    b.gcell = guide_cell(c_params.guide, x, idx);
    b.world_dir_fix = -ray_dir;
    b.frame.set_from_z(-b.world_dir_fix);
    b.cont_prob = m.cont_prob;
    b.mean_cosine = m.mean_cosine;
    b.scatter_coef = m.scattering;
    b.scatter_pos = !is_black_or_negative(m.scattering);
    b.flags |= kBsdfValid;
}

UPBP_D float3 eval_diffuse(const Bsdf& b, const DMaterial& m, float3 lg, float* fpdf, float* rpdf)
{
    if (b.diff_prob == 0.f) return v3(0.f);
    if (b.local_dir_fix.z < kEpsCosine || lg.z < kEpsCosine) return v3(0.f);
    if (fpdf) *fpdf += b.diff_prob * fmaxf(0.f, lg.z * kInvPi);
    if (rpdf) *rpdf += b.diff_prob * fmaxf(0.f, b.local_dir_fix.z * kInvPi);
    return m.diffuse * kInvPi;
}

UPBP_D float3 eval_phong(const Bsdf& b, const DMaterial& m, float3 lg, float* fpdf, float* rpdf)
{
    if (b.phong_prob == 0.f) return v3(0.f);
    if (b.local_dir_fix.z < kEpsCosine || lg.z < kEpsCosine) return v3(0.f);
    const float3 refl = make_float3(-b.local_dir_fix.x, -b.local_dir_fix.y, b.local_dir_fix.z);
    const float dr = dot(refl, lg);
    if (dr <= kEpsPhong) return v3(0.f);
    const float pw = powf(dr, m.phong_exponent);
    if (!is_positive(pw)) return v3(0.f);
    if (fpdf || rpdf) {
        const float p = b.phong_prob * power_cos_hemisphere_pdf(refl, lg, m.phong_exponent);
        if (fpdf) *fpdf += p;
        if (rpdf) *rpdf += p;
    }
    return m.phong * (m.phong_exponent + 2.f) * .5f * kInvPi * pw;
}

UPBP_D void pdf_phong(const Bsdf& b, const DMaterial& m, float3 lg, float* fpdf, float* rpdf)
{
    if (b.phong_prob == 0.f) return;
    const float3 refl = make_float3(-b.local_dir_fix.x, -b.local_dir_fix.y, b.local_dir_fix.z);
    const float dr = dot(refl, lg);
    if (dr <= kEpsPhong) return;
    const float p = power_cos_hemisphere_pdf(refl, lg, m.phong_exponent) * b.phong_prob;
    if (fpdf) *fpdf += p;
    if (rpdf) *rpdf += p;
}

// BSDF value for a generated world direction (bsdf.cuh:339-402).
UPBP_D float3 bsdf_eval(const Bsdf& b, float3 dir_gen, float& cos_gen, float* fpdf, float* rpdf, float* sin_theta)
{
    if (b.on_surface()) {
        if (fpdf) *fpdf = 0.f;
        if (rpdf) *rpdf = 0.f;
        if (sin_theta) *sin_theta = 0.f;
        const float3 lg = b.frame.to_local(dir_gen);
        const float cg = lg.z;
        const float cgg = dot(lg, b.geom_normal);
        cos_gen = fabsf(cg);
        if (cos_gen < kEpsCosine || fabsf(cgg) < kEpsCosine) return v3(0.f);
        if (cg * b.cos_fix() < 0.f || cgg * b.cos_fix_geom < 0.f) return v3(0.f);
        const DMaterial& m = c_params.materials[b.id];
        float3 r = eval_diffuse(b, m, lg, fpdf, rpdf);
        r += eval_phong(b, m, lg, fpdf, rpdf);
        return r;
    }
    cos_gen = 1.f;
    if (!b.scatter_pos) {
        if (fpdf) *fpdf = 0.f;
        if (rpdf) *rpdf = 0.f;
        if (sin_theta) *sin_theta = 0.f;
        return v3(0.f);
    }
    const float p = hg_pdf(b.world_dir_fix, dir_gen, b.mean_cosine, sin_theta);
    // light subpaths sample the phase function; camera subpaths its blend
    // with the learned proposal (the phase function is symmetric, so p is
    // also its reverse pdf)
    const bool light = b.from_light();
    if (fpdf) *fpdf = light ? p : guide_pdf(b, -b.world_dir_fix, dir_gen, p);
    if (rpdf) *rpdf = light ? guide_pdf(b, -dir_gen, b.world_dir_fix, p) : p;
    return b.scatter_coef * p;
}

// Pdf of a generated direction, forward or reverse (bsdf.cuh:408-458).
UPBP_D float bsdf_pdf(const Bsdf& b, float3 dir_gen, bool reverse)
{
    if (b.on_surface()) {
        const float3 lg = b.frame.to_local(dir_gen);
        const float cg = lg.z;
        const float cgg = dot(lg, b.geom_normal);
        if (fabsf(cg) < kEpsCosine || fabsf(cgg) < kEpsCosine) return 0.f;
        if (cg * b.cos_fix() < 0.f || cgg * b.cos_fix_geom < 0.f) return 0.f;
        float fp = 0.f, rp = 0.f;
        const DMaterial& m = c_params.materials[b.id];
        if (b.diff_prob != 0.f) {
            fp += b.diff_prob * fmaxf(0.f, lg.z * kInvPi);
            rp += b.diff_prob * fmaxf(0.f, b.local_dir_fix.z * kInvPi);
        }
        pdf_phong(b, m, lg, &fp, &rp);
        return reverse ? rp : fp;
    }
    const float p = hg_pdf(b.world_dir_fix, dir_gen, b.mean_cosine, nullptr);
    // the camera side's pdfs use the learned proposal's blend (bsdf_eval)
    if (b.from_light() == reverse) return reverse ? guide_pdf(b, -dir_gen, b.world_dir_fix, p)
                                                  : guide_pdf(b, -b.world_dir_fix, dir_gen, p);
    return p;
}

// Samples a direction (bsdf.cuh:571-658).
UPBP_D float3 bsdf_sample(const Bsdf& b, float r0, float r1, float r2, float3& dir_gen, float& pdf, float& cos_gen,
                          unsigned& event, float& sin_theta)
{
    if (b.on_surface()) {
        unsigned ev;
        if (r2 < b.diff_prob)
            ev = kEvDiffuse;
        else if (r2 < b.diff_prob + b.phong_prob)
            ev = kEvPhong;
        else if (r2 < b.diff_prob + b.phong_prob + b.refl_prob)
            ev = kEvReflect;
        else
            ev = kEvRefract;
        event = ev;
        sin_theta = 0.f;
        pdf = 0.f;
        float3 result = v3(0.f);
        float3 lg = v3(0.f);
        const DMaterial& m = c_params.materials[b.id];
        if (ev == kEvDiffuse) {
            if (b.local_dir_fix.z < kEpsCosine) return v3(0.f);
            float up;
            lg = sample_cos_hemisphere(r0, r1, &up);
            pdf += up * b.diff_prob;
            result += m.diffuse * kInvPi;
            if (is_black_or_negative(result)) return v3(0.f);
            result += eval_phong(b, m, lg, &pdf, nullptr);
        } else if (ev == kEvPhong) {
            lg = sample_power_cos_hemisphere(r0, r1, m.phong_exponent);
            const float3 refl = make_float3(-b.local_dir_fix.x, -b.local_dir_fix.y, b.local_dir_fix.z);
            Frame f;
            f.set_from_z(refl);
            lg = f.to_world(lg);
            const float dr = dot(refl, lg);
            if (dr <= kEpsPhong) return v3(0.f);
            pdf_phong(b, m, lg, &pdf, nullptr);
            result += m.phong * (m.phong_exponent + 2.f) * .5f * kInvPi * powf(dr, m.phong_exponent);
            if (is_black_or_negative(result)) return v3(0.f);
            result += eval_diffuse(b, m, lg, &pdf, nullptr);
        } else if (ev == kEvReflect) {
            lg = make_float3(-b.local_dir_fix.x, -b.local_dir_fix.y, b.local_dir_fix.z);
            pdf += b.refl_prob;
            result += b.reflect_coeff * m.mirror / fabsf(lg.z);
            if (is_black_or_negative(result)) return v3(0.f);
        } else {
            if (b.ior < 0.f) return v3(0.f);
            float ci = b.local_dir_fix.z, ct;
            const float eta = b.ior;
            if (ci < 0.f) {
                ci = -ci;
                ct = 1.f;
            } else {
                ct = -1.f;
            }
            const float si2 = 1.f - ci * ci;
            const float st2 = eta * eta * si2;
            if (!(st2 < 1.f)) return v3(0.f);
            ct *= sqrtf(fmaxf(0.f, 1.f - st2));
            lg = make_float3(-eta * b.local_dir_fix.x, -eta * b.local_dir_fix.y, ct);
            pdf += b.refr_prob;
            const float rc = 1.f - b.reflect_coeff;
            result += b.from_light() ? v3(rc / fabsf(ct)) : v3(rc * eta * eta / fabsf(ct));
            if (is_black_or_negative(result)) return v3(0.f);
        }
        dir_gen = b.frame.to_world(lg);
        lg = b.frame.to_local(dir_gen);
        const float cg = lg.z;
        const float cgg = dot(lg, b.geom_normal);
        cos_gen = fabsf(cg);
        if (cos_gen < kEpsCosine || fabsf(cgg) < kEpsCosine) return v3(0.f);
        const bool refr = ev == kEvRefract;
        if ((refr && cg * b.cos_fix() > 0.f) || (!refr && cg * b.cos_fix() < 0.f) ||
            (refr && cgg * b.cos_fix_geom > 0.f) || (!refr && cgg * b.cos_fix_geom < 0.f))
            return v3(0.f);
        return result;
    }
    cos_gen = 1.f;
    event = kEvScatter;
    if (!b.scatter_pos) {
        dir_gen = v3(0.f);
        pdf = 0.f;
        sin_theta = 0.f;
        return v3(0.f);
    }
    if (!b.from_light() && b.gcell >= 0) return guide_sample(b, r0, r1, r2, dir_gen, pdf, sin_theta);
    hg_sample(b.world_dir_fix, b.mean_cosine, r0, r1, b.frame, dir_gen, pdf, &sin_theta);
    return b.scatter_coef * pdf;
}

// ---------------------------------------------------------------- lights

// Environment map (gpuupbp/kernel/env_map.cuh, distribution.cuh): lat-long
// mapping, bilinear radiance lookup and sampling of the sin-weighted
// luminance distribution, as piecewise-constant 1-D distributions (a
// marginal over rows, a conditional per row) inverted by binary search.
UPBP_D float3 env_dir(float u, float v)
{
    const float phi = u * 2.f * kPi, theta = v * kPi;
    const float st = sinf(theta);
    return make_float3(-st * cosf(phi), st * sinf(phi), cosf(theta));
}

UPBP_D float2 env_uv(float3 d)
{
    const float phi = (d.x != 0.f || d.y != 0.f) ? atan2f(d.y, d.x) : 0.f;
    const float theta = acosf(d.z);
    return make_float2(fminf(fmaxf(.5f - phi * .5f * kInvPi, 0.f), 1.f), fminf(fmaxf(theta * kInvPi, 0.f), 1.f));
}

UPBP_D float3 env_pixel(const DEnvMap& m, int x, int y) { return xyz(__ldg(&m.img[(size_t)y * m.width + x])); }

UPBP_D float3 env_radiance(const DEnvMap& m, float u, float v)
{
    const float xf = u * m.width, yf = v * m.height;
    const int x1 = min(max((int)xf, 0), m.width - 1), y1 = min(max((int)yf, 0), m.height - 1);
    const int x2 = x1 == m.width - 1 ? x1 : x1 + 1, y2 = y1 == m.height - 1 ? y1 : y1 + 1;
    const float tx = xf - (float)x1, ty = yf - (float)y1;
    return (1.f - ty) * ((1.f - tx) * env_pixel(m, x1, y1) + tx * env_pixel(m, x2, y1)) +
           ty * ((1.f - tx) * env_pixel(m, x1, y2) + tx * env_pixel(m, x2, y2));
}

// sin(theta) at the centre of the row holding v
UPBP_D float env_sin_theta(float v, float height)
{
    const float row = v < 1.f ? (float)((int)(v * height)) : height - 1.f;
    return sinf(kPi * (row + .5f) / height);
}

// Samples one 1-D distribution of n values (function at f, cdf at f + n... as
// laid out by the host); returns the continuous coordinate in [0, 1).
UPBP_D float env_sample_1d(const float* func, const float* cdf, int n, float integral, float u, float& pdf, int& off)
{
    int first = 0, len = n + 1;
    while (len > 0) {  // last cdf entry <= u
        const int half = len >> 1, mid = first + half;
        if (__ldg(&cdf[mid]) <= u) {
            first = mid + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    off = min(max(first - 1, 0), n - 1);
    const float c0 = __ldg(&cdf[off]), c1 = __ldg(&cdf[off + 1]);
    float du = u - c0;
    if (c1 - c0 > 0.f) du /= (c1 - c0);
    pdf = integral > 0.f ? __ldg(&func[off]) / integral : 0.f;
    return ((float)off + du) / (float)n;
}

// Direction sampled from the map, its solid-angle pdf and radiance.
UPBP_D float3 env_sample(const DEnvMap& m, float u0, float u1, float& pdf_w, float3& radiance)
{
    const size_t row = 2 * (size_t)m.nu + 1;
    const float* marg = m.dist + row * m.nv;
    float pv, pu;
    int v;
    const float fv = env_sample_1d(marg, marg + m.nu, m.nv, m.marg_int, u1, pv, v);
    int unused;
    const float* cond = m.dist + row * v;
    const float fu = env_sample_1d(cond, cond + m.nu, m.nu, __ldg(&m.row_int[v]), u0, pu, unused);
    pdf_w = m.norm * (pu * pv) / env_sin_theta(fv, (float)m.height);
    radiance = env_radiance(m, fu, fv);
    return env_dir(fu, fv);
}

// Radiance the map sends along -dir (dir points from the scene to the map)
// and the solid-angle pdf of sampling dir; radiance 0 where that pdf is 0.
UPBP_D float3 env_lookup(const DEnvMap& m, float3 dir, float& pdf_w)
{
    const float2 uv = env_uv(normalize(dir));
    float3 radiance = env_radiance(m, uv.x, uv.y);
    const int iu = min(max((int)(uv.x * m.nu), 0), m.nu - 1);
    const int iv = min(max((int)(uv.y * m.nv), 0), m.nv - 1);
    const float ri = __ldg(&m.row_int[iv]);
    const size_t row = 2 * (size_t)m.nu + 1;
    float p = 0.f;
    if (ri * m.marg_int != 0.f) p = (__ldg(&m.dist[row * iv + iu]) * __ldg(&m.dist[row * m.nv + iv])) / (ri * m.marg_int);
    pdf_w = m.norm * p / env_sin_theta(uv.y, (float)m.height);
    if (pdf_w == 0.f) radiance = v3(0.f);
    return radiance;
}

UPBP_D bool light_is_finite(const DLight& l) { return l.type == kLightArea || l.type == kLightPoint; }
UPBP_D bool light_is_delta(const DLight& l) { return l.type == kLightDirectional || l.type == kLightPoint; }

// Next-event sample toward the light (light.cuh illuminate).
UPBP_D float3 light_illuminate(const DLight& l, float3 x, float u0, float u1, float3& dir_to_light, float& dist,
                               float& direct_pdf_w, float& emission_pdf_w, float& cos_at_light)
{
    switch (l.type) {
    case kLightArea: {
        const float su = sqrtf(u0);
        const float bu = 1.f - su, bv = u1 * su;
        const float3 p = l.p0 + l.e1 * bu + l.e2 * bv;
        dir_to_light = p - x;
        const float d2 = dot(dir_to_light, dir_to_light);
        dist = sqrtf(d2);
        dir_to_light = dir_to_light / dist;
        const float cn = dot(l.frame.z, -dir_to_light);
        if (cn < kEpsCosine) return v3(0.f);
        direct_pdf_w = l.inv_area * d2 / cn;
        cos_at_light = cn;
        emission_pdf_w = l.inv_area * cn * kInvPi;
        return l.intensity;
    }
    case kLightBackground: {
        float3 radiance = l.intensity;
        if (l.env) {
            dir_to_light = env_sample(c_params.env, u0, u1, direct_pdf_w, radiance);
            radiance = radiance * l.scale;
        } else {
            dir_to_light = sample_uniform_sphere(u0, u1, &direct_pdf_w);
        }
        dist = kInfinity;
        emission_pdf_w = direct_pdf_w * kInvPi * c_params.inv_radius_sqr;
        cos_at_light = 1.f;
        return radiance;
    }
    case kLightDirectional: {
        dir_to_light = -l.frame.z;
        dist = kInfinity;
        direct_pdf_w = 1.f;
        cos_at_light = 1.f;
        emission_pdf_w = kInvPi * c_params.inv_radius_sqr;
        return l.intensity;
    }
    default: {
        dir_to_light = l.position - x;
        const float d2 = dot(dir_to_light, dir_to_light);
        direct_pdf_w = d2;
        dist = sqrtf(d2);
        dir_to_light = dir_to_light / dist;
        cos_at_light = 1.f;
        emission_pdf_w = uniform_sphere_pdf();
        return l.intensity;
    }
    }
}

// Emission sample (light.cuh emit).
UPBP_D float3 light_emit(const DLight& l, float d0, float d1, float p0, float p1, float3& pos, float3& dir,
                         float& emission_pdf_w, float& direct_pdf_a, float& cos_light)
{
    switch (l.type) {
    case kLightArea: {
        const float su = sqrtf(p0);
        pos = l.p0 + l.e1 * (1.f - su) + l.e2 * (p1 * su);
        float3 lo = sample_cos_hemisphere(d0, d1, &emission_pdf_w);
        emission_pdf_w *= l.inv_area;
        lo.z = fmaxf(lo.z, kEpsCosine);
        dir = l.frame.to_world(lo);
        direct_pdf_a = l.inv_area;
        cos_light = lo.z;
        return l.intensity * lo.z;
    }
    case kLightBackground: {
        float fp;
        float3 radiance = l.intensity;
        if (l.env) {
            dir = -env_sample(c_params.env, d0, d1, fp, radiance);
            radiance = radiance * l.scale;
        } else {
            dir = sample_uniform_sphere(d0, d1, &fp);
        }
        const float2 xy = sample_concentric_disc(p0, p1);
        Frame f;
        f.set_from_z(dir);
        pos = c_params.scene_center + c_params.scene_radius * (-dir + f.x * xy.x + f.y * xy.y);
        emission_pdf_w = fp * kInvPi * c_params.inv_radius_sqr;
        direct_pdf_a = fp;
        cos_light = 1.f;
        return radiance;
    }
    case kLightDirectional: {
        const float2 xy = sample_concentric_disc(p0, p1);
        pos = c_params.scene_center + c_params.scene_radius * (-l.frame.z + l.frame.x * xy.x + l.frame.y * xy.y);
        dir = l.frame.z;
        emission_pdf_w = kInvPi * c_params.inv_radius_sqr;
        direct_pdf_a = 1.f;
        cos_light = 1.f;
        return l.intensity;
    }
    default: {
        pos = l.position;
        dir = sample_uniform_sphere(d0, d1, &emission_pdf_w);
        direct_pdf_a = 1.f;
        cos_light = 1.f;
        return l.intensity;
    }
    }
}

// Radiance of a light hit by a ray (light.cuh get_radiance).
UPBP_D float3 light_radiance(const DLight& l, float3 ray_dir, float& direct_pdf_a, float& emission_pdf_w)
{
    if (l.type == kLightArea) {
        const float c = fmaxf(0.f, dot(l.frame.z, -ray_dir));
        if (c == 0.f) return v3(0.f);
        direct_pdf_a = l.inv_area;
        emission_pdf_w = fmaxf(0.f, dot(l.frame.z, -ray_dir)) * kInvPi * l.inv_area;
        return l.intensity;
    }
    if (l.type == kLightBackground) {
        float fp = uniform_sphere_pdf();
        float3 radiance = l.intensity;
        if (l.env) radiance = l.scale * env_lookup(c_params.env, ray_dir, fp);
        direct_pdf_a = fp;
        emission_pdf_w = fp * (kInvPi * c_params.inv_radius_sqr);
        return radiance;
    }
    return v3(0.f);
}

// ---------------------------------------------------------------- camera

UPBP_D float3 transform_point(const float* m, float3 v)
{
    float w = m[15];
    w += m[12] * v.x;
    w += m[13] * v.y;
    w += m[14] * v.z;
    const float iw = 1.f / w;
    float x = m[3];
    x += v.x * m[0];
    x += v.y * m[1];
    x += v.z * m[2];
    float y = m[7];
    y += v.x * m[4];
    y += v.y * m[5];
    y += v.z * m[6];
    float z = m[11];
    z += v.x * m[8];
    z += v.y * m[9];
    z += v.z * m[10];
    return make_float3(x * iw, y * iw, z * iw);
}

UPBP_D float2 world_to_raster(const DCamera& c, float3 p)
{
    const float3 t = transform_point(c.world_to_raster, p);
    return make_float2(t.x, t.y);
}

UPBP_D bool raster_inside(const DCamera& c, float2 r)
{
    return r.x >= 0.f && r.y >= 0.f && r.x < c.res_x && r.y < c.res_y;
}

}  // namespace upbp
