// Camera pass: one thread per pixel.  Emitter hits, next-event estimation,
// BPT connections to one random light subpath, and the five photon density
// estimators as range queries over the per-iteration photon maps.
// Follows __raygen__trace_camera (gpuupbp/kernel/trace_camera.cu:49-390),
// functs_camera.cuh:41-527 and the estimator bodies in gpuupbp/kernel/pde/
// (functs_pp.cuh:44-136, functs_pb2d.cuh:57-342, functs_bb1d.cuh:57-397,
// functs_bp2d.cuh:51-229).
#pragma once

#include <type_traits>

#include "upbp_build.cuh"
#include "upbp_queries.cuh"

namespace upbp {

UPBP_D unsigned generate_camera_sample(float2& screen, unsigned pixel, PathState& s, Rng& rng)
{
    const DeviceParams& p = c_params;
    const DCamera& cam = p.camera;
    const int res_x = int(cam.res_x);
    const unsigned x = pixel % res_x, y = pixel / res_x;
    // The reference draws both jitter values inside one make_float2 call, whose
    // argument order C++ leaves unspecified; the host-compiled oracle evaluates
    // right to left, so the first draw is the y jitter.  Same below for NEE.
    const float j1 = rng.uniform();
    const float j0 = rng.uniform();
    screen = make_float2(float(x) + j0, float(y) + j1);
    const float3 wr = transform_point(cam.raster_to_world, make_float3(screen.x, screen.y, 0.f));
    s.origin = cam.origin;
    s.dir = normalize(wr - cam.origin);
    UPBP_MISDBG(mis_origin(false, pixel, cam.origin, cam.direction, 0u));
    const float cos_at_cam = dot(cam.direction, s.dir);
    const float ip_dist = cam.image_plane_dist / cos_at_cam;
    const float camera_pdf_w = (ip_dist * ip_dist) / cos_at_cam;
    s.throughput = v3(1.f);
    s.path_length = 1;
    s.is_specular_path = true;
    s.is_infinite_light = false;
    VertexWeights& w = s.sw.w;
    w.d_shared = p.light_subpath_count / camera_pdf_w;
    w.d_bpt = 0.f;
    w.d_pde = 0.f;
    w.prev_specular = false;
    w.prev_in_medium = false;
    if (!init_boundary_stack(s.stack)) return kErrBoundaryStack;
    if (cam.mat_id != -1 && cam.med_id != -1) {
        if (!s.stack.push(Boundary{cam.mat_id, cam.med_id}, boundary_priority(cam.mat_id))) return kErrBoundaryStack;
    }
    return 0;
}

// Emitter hit, MIS Eq D.32/D.33 (functs_camera.cuh:107-165).
UPBP_D float3 light_hit_radiance(const DLight& l, const PathState& s, float rs_rev, float* w_out = nullptr)
{
    const DeviceParams& p = c_params;
    if (s.is_specular_path && p.ignore_fully_spec_paths) return v3(0.f);
    const float pick = 1.f / float(p.light_count);
    float direct_pdf_a, emission_pdf_w;
    const float3 rad = light_radiance(l, s.dir, direct_pdf_a, emission_pdf_w);
    if (is_black_or_negative(rad)) return v3(0.f);
    if (s.path_length == 1) return rad;
    if (p.estimator_techniques && !(p.estimator_techniques & kBpt)) return s.is_specular_path ? rad : v3(0.f);
    direct_pdf_a *= pick;
    emission_pdf_w *= pick;
    const VertexWeights& wc = s.sw.w;
    const float bpt = !wc.prev_specular;
    const float w_camera = direct_pdf_a * bpt * wc.d_shared + emission_pdf_w * rs_rev * wc.d_bpt;
    if (w_out) *w_out = 1.f / (0.f + 1.f + w_camera);
    return (1.f / (0.f + 1.f + w_camera)) * rad;
}

// Next-event estimation, MIS Eq D.36/D.37 (functs_camera.cuh:170-344), in
// two halves: nee_sample draws the light sample and evaluates the BSDF in the
// camera pass (it consumes the path's random numbers); nee_finish traces the
// occlusion ray and applies the MIS weight in nee_connect_kernel.
struct NeeSample {
    float3 dir, rad, f;
    float dist, k, w_light, a, rpdf, sin_theta;
    UPBP_MISDBG(int light;)
};

UPBP_D bool nee_sample(NeeSample& ns, float3 hit, const Bsdf& bsdf, Rng& rng)
{
    const DeviceParams& p = c_params;
    const float pick = 1.f / float(p.light_count);
    const int lid = int(rng.uniform() * float(p.light_count));
    const float u1 = rng.uniform();
    const float u0 = rng.uniform();
    const DLight& l = p.lights[lid];
    if (!light_is_finite(l) && p.media[p.global_medium].has_attenuation) return false;
    float3 dir;
    float dist, direct_pdf_w, emission_pdf_w, cos_at_light;
    const float3 rad = light_illuminate(l, hit, u0, u1, dir, dist, direct_pdf_w, emission_pdf_w, cos_at_light);
    if (is_black_or_negative(rad)) return false;
    float fpdf, rpdf, cos_to_light, sin_theta;
    const float3 f = bsdf_eval(bsdf, dir, cos_to_light, &fpdf, &rpdf, &sin_theta);
    if (is_black_or_negative(f)) return false;
    const float cp = bsdf.cont_prob;
    fpdf *= light_is_delta(l) ? 0.f : cp;
    rpdf *= cp;
    ns.dir = dir;
    ns.dist = dist;
    ns.rad = rad;
    ns.f = f;
    ns.w_light = fpdf / (pick * direct_pdf_w);
    ns.a = emission_pdf_w * cos_to_light / (direct_pdf_w * cos_at_light);
    ns.k = cos_to_light / (pick * direct_pdf_w);
    ns.rpdf = rpdf;
    ns.sin_theta = sin_theta;
    UPBP_MISDBG(ns.light = lid;)
    return true;
}

UPBP_D unsigned nee_finish(float3& contrib, const NeeSample& ns, float3 hit, bool in_medium, const BoundaryStack& stack,
                           const VertexWeights& wc, VolSeg* segs, float* w_out = nullptr, int* nseg_out = nullptr)
{
    contrib = v3(0.f);
    int nseg = 0;
    bool occ;
    Rng unused;
    unused.state = unused.inc = 0;  // occlusion rays draw no random numbers
    const unsigned st = occluded(occ, hit, ns.dir, ns.dist, stack, in_medium ? kOriginInMedium : 0u, segs, nseg, unused);
    if (st) return st;
    if (occ) return 0;
    float n_rev = 1.f, n_for = 1.f;
    float3 att = v3(1.f);
    if (nseg > 0) {
        n_rev = seg_rev_pdf(segs, nseg);
        n_for = seg_for_pdf(segs, nseg);
        att = seg_attenuation(segs, nseg);
        if (!is_positive(att)) return 0;
    }
    const float ft = pde_factor(in_medium, false, 1.f / n_rev, wc.rev_ratio, wc.for_inv, wc.for_ratio, ns.sin_theta);
    const float b = !wc.prev_specular;
    const float w_camera = ns.a * n_rev * (ft + b * wc.d_shared + (ns.rpdf / wc.rev_inv) * wc.d_bpt);
    // the reference's w_light omits the camera-side sampling pdf of the
    // light ray's media (functs_camera.cuh:296); the emitter-hit weight of
    // the same path includes it
    const float w_light = c_params.mis_exact ? ns.w_light * n_for : ns.w_light;
    const float mis = 1.f / (w_light + 1.f + w_camera);
    if (w_out) *w_out = mis;
    if (nseg_out) *nseg_out = nseg;
    contrib = (ns.k * (ns.rad * att * ns.f)) * mis;
    if (is_black_or_negative(contrib)) contrib = v3(0.f);
    return 0;
}

// BPT connection of a camera and a light vertex, Eq 4.50/4.51
// (functs_camera.cuh:349-527).
UPBP_D unsigned connect_vertices(float3& contrib, const LightVertex& lv, const Bsdf& cb, float3 chit, const PathState& s,
                                 Rng& rng, VolSeg* segs, float* w_out = nullptr, int* nseg_out = nullptr)
{
    contrib = v3(0.f);
    float3 dir = lv.hit - chit;
    const float d2 = dot(dir, dir);
    const float dist = sqrtf(d2);
    dir /= dist;
    float cos_c, c_fpdf, c_rpdf, sin_c;
    const float3 cf = bsdf_eval(cb, dir, cos_c, &c_fpdf, &c_rpdf, &sin_c);
    if (is_black_or_negative(cf)) return 0;
    c_fpdf *= cb.cont_prob;
    c_rpdf *= cb.cont_prob;
    float cos_l, l_fpdf, l_rpdf, sin_l;
    const float3 lf = bsdf_eval(lv.bsdf, -dir, cos_l, &l_fpdf, &l_rpdf, &sin_l);
    if (is_black_or_negative(lf)) return 0;
    l_fpdf *= lv.bsdf.cont_prob;
    l_rpdf *= lv.bsdf.cont_prob;
    const float g = cos_l * cos_c / d2;
    if (g < 0.f) return 0;
    const float c_fpdf_a = pdf_w_to_a(c_fpdf, dist, cos_l);
    const float l_fpdf_a = pdf_w_to_a(l_fpdf, dist, cos_c);
    unsigned sflags = 0;
    if (cb.in_medium()) sflags |= kOriginInMedium;
    if (lv.in_medium) sflags |= kEndInMedium;
    int nseg = 0;
    bool occ;
    const unsigned st = occluded(occ, chit, dir, dist, s.stack, sflags, segs, nseg, rng);
    if (st) return st;
    if (occ) return 0;
    float rs_for = 1.f, rs_rev = 1.f;
    float3 att = v3(1.f);
    if (nseg > 0) {
        rs_for = seg_for_pdf(segs, nseg);
        rs_rev = seg_rev_pdf(segs, nseg);
        att = seg_attenuation(segs, nseg);
        if (!is_positive(att)) return 0;
    }
    const VertexWeights& wl = lv.w;
    const VertexWeights& wc = s.sw.w;
    const float f_s = pde_factor(lv.bsdf.in_medium(), false, wl.for_inv, wl.for_ratio, 1.f / rs_for, wl.rev_ratio, sin_l);
    const float bs = !wl.prev_specular;
    const float w_light = c_fpdf_a * rs_for * (f_s + bs * wl.d_shared + (l_rpdf / wl.rev_inv) * wl.d_bpt);
    const float f_t = pde_factor(cb.in_medium(), false, 1.f / rs_rev, wc.rev_ratio, wc.for_inv, wc.for_ratio, sin_c);
    const float bt = !wc.prev_specular;
    const float w_camera = l_fpdf_a * rs_rev * (f_t + bt * wc.d_shared + (c_rpdf / wc.rev_inv) * wc.d_bpt);
    const float mis = 1.f / (w_light + 1.f + w_camera);
    if (w_out) *w_out = mis;
    if (nseg_out) *nseg_out = nseg;
    contrib = (g * cf * lf * att) * mis;
    if (is_black_or_negative(contrib)) contrib = v3(0.f);
    return 0;
}

// SURF / PP3D merge of a camera vertex with one photon, Eq 4.52/4.17/4.53
// (functs_pp.cuh:44-136).
UPBP_D float3 eval_point_merge(const LightVertex& lv, unsigned cam_len, const VertexWeights& wc, const Bsdf& cb,
                                bool medium, float* w_out = nullptr)
{
    const DeviceParams& p = c_params;
    const unsigned plen = lv.path_length + cam_len;
    if (plen > p.max_path_length || plen < p.min_path_length) return v3(0.f);
    const float3 pdir = lv.bsdf.dir_fix();
    float cos_c, fpdf, rpdf, sin_theta;
    const float3 f = bsdf_eval(cb, pdir, cos_c, &fpdf, &rpdf, &sin_theta);
    if (is_black_or_negative(f)) return v3(0.f);
    fpdf *= cb.cont_prob;
    rpdf *= lv.bsdf.cont_prob;
    const VertexWeights& wl = lv.w;
    const float ff = p.photon_beam_type == kLongBeam ? wl.for_inv : wl.for_ratio;
    const float rf = p.camera_beam_type == kLongBeam ? wc.for_inv : wc.for_ratio;
    const float val = medium ? 1.f / p.mis_factor_pp3d : 1.f / p.mis_factor_surf;
    const float bs = !wl.prev_specular;
    const float w_light = val * (wl.d_shared * bs * p.subpath_count_bpt + fpdf * wl.d_pde / wl.rev_inv);
    const float w_local =
        1.f + float(medium) * val * (p.mis_factor_bb1d * sin_theta * ff * rf + p.mis_factor_bp2d * ff + p.mis_factor_pb2d * rf);
    const float bt = !wc.prev_specular;
    const float w_camera = val * (wc.d_shared * bt * p.subpath_count_bpt + rpdf * wc.d_pde / wc.rev_inv);
    const float mis = 1.f / (w_light + w_local + w_camera);
    if (w_out) *w_out = mis;
    return mis * f * lv.thr;
}

struct QuerySeg {
    float3 o, d;
    float dmin, dmax;
    int med;
    float for_pdf, rev_pdf;
    unsigned flags;
    unsigned cam_path_length;
};

// PB2D: camera query beam x photon point (functs_pb2d.cuh:57-201).
UPBP_D float3 eval_pb2d(const QuerySeg& q, const StateWeights& cw, const LightVertex& lv, float isect_dist, float rad2,
                        float* w_out = nullptr, bool guided = true)
{
    const DeviceParams& p = c_params;
    const unsigned plen = lv.path_length + q.cam_path_length;
    if (plen > p.max_path_length || plen < p.min_path_length) return v3(0.f);
    const DMedium& m = p.media[q.med];
    float3 att = attenuation(m, isect_dist - q.dmin);
    const float pdf = component(att, m.min_pos_att_idx);
    if (p.camera_beam_type == kShortBeam) att /= pdf;
    float rs_for = m.min_pos_att * pdf;
    float rs_rev = (q.flags & kOriginInMedium) ? rs_for : pdf;
    const float ratio = 1.f / m.min_pos_att;
    if (!is_positive(att)) return v3(0.f);
    rs_for *= q.for_pdf;
    rs_rev *= q.rev_pdf;
    VertexWeights wc = cw.w;
    if (q.cam_path_length > 1u) {
        const float f_i = pde_factor(wc.prev_in_medium, wc.prev_specular, 1.f / rs_rev, wc.rev_ratio, wc.for_inv,
                                     wc.for_ratio, cw.last_sin_theta);
        wc.d_pde = cw.d_pde_a * f_i + cw.d_pde_b;
        wc.d_bpt = cw.d_bpt_a * f_i + cw.d_bpt_b;
    }
    const float3 pdir = lv.bsdf.dir_fix();
    float sin_theta;
    const float ph = hg_pdf(-q.d, pdir, m.mean_cosine, &sin_theta);
    const float3 f = v3(ph);
    if (is_black_or_negative(f)) return v3(0.f);
    const float fpdf = (guided ? guide_pdf_at(q.o + q.d * isect_dist, q.med, q.d, pdir, ph) : ph) * m.cont_prob;
    const float rpdf = ph * lv.bsdf.cont_prob;
    wc.d_shared *= isect_dist * isect_dist;
    wc.d_shared /= rs_for;
    wc.d_bpt /= rs_for;
    wc.d_pde /= rs_for;
    wc.for_inv = 1.f / rs_for;
    wc.rev_inv = 1.f / rs_rev;
    wc.for_ratio = ratio;
    wc.rev_ratio = ratio;
    const float kernel = (1.f - rad2 / p.radius_pb2d_2) / (p.radius_pb2d_2 * kPi * .5f);
    if (!is_positive(kernel)) return v3(0.f);
    const float3 unweighted = lv.thr * att * m.scattering * f * kernel;
    if (is_black_or_negative(unweighted)) return v3(0.f);
    const VertexWeights& wl = lv.w;
    const float ff = p.photon_beam_type == kLongBeam ? wl.for_inv : wl.for_ratio;
    const float rf = p.camera_beam_type == kLongBeam ? wc.for_inv : wc.for_ratio;
    const float val = 1.f / (p.mis_factor_pb2d * rf);
    const float bs = !wl.prev_specular;
    const float w_light = val * (wl.d_shared * bs * p.subpath_count_bpt + fpdf * wl.d_pde / wl.rev_inv);
    const float w_local = 1.f + val * (p.mis_factor_bb1d * sin_theta * ff * rf + p.mis_factor_bp2d * ff + p.mis_factor_pp3d);
    const float bt = !wc.prev_specular;
    const float w_camera = val * (wc.d_shared * bt * p.subpath_count_bpt + rpdf * wc.d_pde / wc.rev_inv);
    const float mis = 1.f / (w_light + w_local + w_camera);
    if (w_out) *w_out = mis;
    return mis * unweighted;
}

// BB1D: camera query beam x photon beam (functs_bb1d.cuh:57-248).
UPBP_D float3 eval_bb1d(const QuerySeg& q, const StateWeights& cw, const Beam& lb, float bb_dist, float sin_theta,
                        float tc, float tp, float* w_out = nullptr, bool guided = true)
{
    const DeviceParams& p = c_params;
    const unsigned plen = lb.path_length + q.cam_path_length;
    if (plen > p.max_path_length || plen < p.min_path_length) return v3(0.f);
    const DMedium& m = p.media[q.med];
    float3 att_c = attenuation(m, tc - q.dmin);
    const float pc = component(att_c, m.min_pos_att_idx);
    if (p.camera_beam_type == kShortBeam) att_c /= pc;
    float rsf_c = m.min_pos_att * pc;
    float rsr_c = (q.flags & kOriginInMedium) ? rsf_c : pc;
    const float ratio = 1.f / m.min_pos_att;
    float3 att_p = attenuation(m, tp);
    const float pp = component(att_p, m.min_pos_att_idx);
    if (p.photon_beam_type == kShortBeam) att_p /= pp;
    float rsf_p = m.min_pos_att * pp;
    float rsr_p = (lb.flags & kOriginInMedium) ? rsf_p : pp;
    const float3 att = att_c * att_p;
    if (!is_positive(att)) return v3(0.f);
    rsf_c *= q.for_pdf;
    rsr_c *= q.rev_pdf;
    VertexWeights wc = cw.w;
    if (q.cam_path_length > 1u) {
        const float f_i = pde_factor(wc.prev_in_medium, wc.prev_specular, 1.f / rsr_c, wc.rev_ratio, wc.for_inv,
                                     wc.for_ratio, cw.last_sin_theta);
        wc.d_pde = cw.d_pde_a * f_i + cw.d_pde_b;
        wc.d_bpt = cw.d_bpt_a * f_i + cw.d_bpt_b;
    }
    rsf_p *= lb.for_pdf;
    rsr_p *= lb.rev_pdf;
    VertexWeights wl = lb.sw.w;
    if (lb.path_length > 1u) {
        const float f_i = pde_factor(wl.prev_in_medium, wl.prev_specular, wl.for_inv, wl.for_ratio, 1.f / rsr_p,
                                     wl.rev_ratio, lb.sw.last_sin_theta);
        wl.d_pde = lb.sw.d_pde_a * f_i + lb.sw.d_pde_b;
        wl.d_bpt = lb.sw.d_bpt_a * f_i + lb.sw.d_bpt_b;
    }
    const float ph = hg_pdf(-q.d, -lb.d, m.mean_cosine, nullptr);
    const float3 f = v3(ph);
    if (is_black_or_negative(f)) return v3(0.f);
    const float fpdf = (guided ? guide_pdf_at(q.o + q.d * tc, q.med, q.d, -lb.d, ph) : ph) * m.cont_prob;
    const float rpdf = ph * m.cont_prob;
    wc.d_shared *= tc * tc;
    wc.d_shared /= rsf_c;
    wc.d_bpt /= rsf_c;
    wc.d_pde /= rsf_c;
    wc.for_inv = 1.f / rsf_c;
    wc.rev_inv = 1.f / rsr_c;
    wc.for_ratio = ratio;
    wc.rev_ratio = ratio;
    {
        // The reference multiplies by the squared distance from the beam's
        // origin, and not for first-segment beams of finite lights
        // (functs_bb1d.cuh:191), kept for parity.  The exact form (mis_exact)
        // measures the distance from the light vertex and skips it only after
        // an infinite light, as every other merge does.
        const bool skip = lb.path_length == 1 && lb.infinite == (p.mis_exact != 0);
        const float dl = tp + (p.mis_exact ? lb.origin_offset : 0.f);
        if (!skip) wl.d_shared *= dl * dl;
    }
    wl.d_shared /= rsf_p;
    wl.d_bpt /= rsf_p;
    wl.d_pde /= rsf_p;
    wl.for_inv = 1.f / rsf_p;
    wl.rev_inv = 1.f / rsr_p;
    wl.for_ratio = ratio;
    wl.rev_ratio = ratio;
    const float kernel = (1.f - bb_dist * bb_dist / p.radius_bb1d_2) * 3.f / (4.f * p.radius_bb1d * sin_theta);
    if (!is_positive(kernel)) return v3(0.f);
    const float3 unweighted = lb.thr * m.scattering * att * f * kernel;
    if (is_black_or_negative(unweighted)) return v3(0.f);
    const float ff = p.photon_beam_type == kLongBeam ? wl.for_inv : wl.for_ratio;
    const float rf = p.camera_beam_type == kLongBeam ? wc.for_inv : wc.for_ratio;
    const float val = 1.f / (p.mis_factor_bb1d * sin_theta * ff * rf);
    const float bs = !wl.prev_specular;
    const float w_light = val * (wl.d_shared * bs * p.subpath_count_bpt + fpdf * wl.d_pde / wl.rev_inv);
    const float w_local = 1.f + val * (p.mis_factor_bp2d * ff + p.mis_factor_pb2d * rf + p.mis_factor_pp3d);
    const float bt = !wc.prev_specular;
    const float w_camera = val * (wc.d_shared * bt * p.subpath_count_bpt + rpdf * wc.d_pde / wc.rev_inv);
    const float mis = 1.f / (w_light + w_local + w_camera);
    if (w_out) *w_out = mis;
    return mis * unweighted;
}

// BP2D: photon beam x camera point (functs_bp2d.cuh:51-198).
UPBP_D float3 eval_bp2d(const Beam& lb, unsigned cam_len, const VertexWeights& wc, const Bsdf& cb, float isect_dist,
                        float rad2, float* w_out = nullptr)
{
    const DeviceParams& p = c_params;
    const unsigned plen = lb.path_length + cam_len;
    if (plen > p.max_path_length || plen < p.min_path_length) return v3(0.f);
    const DMedium& m = p.media[lb.med];
    float3 att = attenuation(m, isect_dist);
    const float pdf = component(att, m.min_pos_att_idx);
    if (p.photon_beam_type == kShortBeam) att /= pdf;
    float rs_for = m.min_pos_att * pdf;
    float rs_rev = (lb.flags & kOriginInMedium) ? rs_for : pdf;
    const float ratio = 1.f / m.min_pos_att;
    if (!is_positive(att)) return v3(0.f);
    rs_for *= lb.for_pdf;
    rs_rev *= lb.rev_pdf;
    VertexWeights wl = lb.sw.w;
    if (lb.path_length > 1u) {
        const float f_i = pde_factor(wl.prev_in_medium, wl.prev_specular, wl.for_inv, wl.for_ratio, 1.f / rs_rev,
                                     wl.rev_ratio, lb.sw.last_sin_theta);
        wl.d_pde = lb.sw.d_pde_a * f_i + lb.sw.d_pde_b;
        wl.d_bpt = lb.sw.d_bpt_a * f_i + lb.sw.d_bpt_b;
    }
    const float3 cdir = cb.dir_fix();
    float sin_theta;
    const float ph = hg_pdf(cdir, -lb.d, m.mean_cosine, &sin_theta);
    const float3 f = v3(ph);
    if (is_black_or_negative(f)) return v3(0.f);
    const float fpdf = guide_pdf(cb, -cdir, -lb.d, ph) * cb.cont_prob;
    const float rpdf = ph * m.cont_prob;
    // the reference measures the distance from the beam's origin, which lies
    // past the light vertex when the beam starts at a medium boundary
    // (functs_bp2d.cuh:137-140); the exact form measures it from the vertex
    const float dl = p.mis_exact ? lb.origin_offset + isect_dist : isect_dist;
    if (!(lb.path_length == 1 && lb.infinite)) wl.d_shared *= dl * dl;
    wl.d_shared /= rs_for;
    wl.d_bpt /= rs_for;
    wl.d_pde /= rs_for;
    wl.for_inv = 1.f / rs_for;
    wl.rev_inv = 1.f / rs_rev;
    wl.for_ratio = ratio;
    wl.rev_ratio = ratio;
    const float kernel = (1.f - rad2 / p.radius_bp2d_2) / (p.radius_bp2d_2 * kPi * .5f);
    if (!is_positive(kernel)) return v3(0.f);
    const float3 unweighted = lb.thr * att * m.scattering * f * kernel;
    if (is_black_or_negative(unweighted)) return v3(0.f);
    const float ff = p.photon_beam_type == kLongBeam ? wl.for_inv : wl.for_ratio;
    const float rf = p.camera_beam_type == kLongBeam ? wc.for_inv : wc.for_ratio;
    const float val = 1.f / (p.mis_factor_bp2d * ff);
    const float bs = !wl.prev_specular;
    const float w_light = val * (wl.d_shared * bs * p.subpath_count_bpt + fpdf * wl.d_pde / wl.rev_inv);
    const float w_local = 1.f + val * (p.mis_factor_bb1d * sin_theta * ff * rf + p.mis_factor_pb2d * rf + p.mis_factor_pp3d);
    const float bt = !wc.prev_specular;
    const float w_camera = val * (wc.d_shared * bt * p.subpath_count_bpt + rpdf * wc.d_pde / wc.rev_inv);
    const float mis = 1.f / (w_light + w_local + w_camera);
    if (w_out) *w_out = mis;
    return mis * unweighted;
}

// Emits one segment-query record per scattering medium segment of a camera
// ray, with the attenuation and sampling pdfs accumulated over the segments
// before it (the segment loop of eval_pb2d_segments / eval_bb1d_segments,
// functs_pb2d.cuh:226-342, functs_bb1d.cuh:273-397, both variants).
UPBP_D void emit_segment_queries(float3 ro, float3 rd, const VolSeg* segs, int nseg, const LiteSeg* lsegs, int nlseg,
                                 bool use_lite, unsigned sflags, unsigned cam_path_length, const StateWeights& cw,
                                 float3 throughput, unsigned pixel, unsigned path)
{
    const DeviceParams& p = c_params;
    float3 att = v3(1.f);
    float fpdf = 1.f, rpdf = 1.f;
    const int n = use_lite ? nlseg : nseg;
    for (int i = 0; i < n; i++) {
        const float dmin = use_lite ? lsegs[i].dmin : segs[i].dmin;
        const float dmax = use_lite ? lsegs[i].dmax : segs[i].dmax;
        const int med = use_lite ? lsegs[i].med : segs[i].med;
        const DMedium& m = p.media[med];
        if (m.has_scattering) {
            const unsigned k = warp_reserve1(&p.queue_count[0]);
            if (k < p.seg_capacity) {
                float4* q = p.seg_queue[k].q;
                const float3 w = throughput * att;
                const unsigned flags = kEndInMedium | (i == 0 ? sflags : 0u);
                q[0] = make_float4(ro.x, ro.y, ro.z, dmin);
                q[1] = make_float4(rd.x, rd.y, rd.z, dmax);
                q[2] = make_float4(w.x, w.y, w.z, ubits((unsigned)med));
                q[3] = make_float4(fpdf, rpdf, ubits(flags), ubits((pixel << 8) | (cam_path_length & 0xffu)));
                const VertexWeights& vw = cw.w;
                const unsigned bits = (vw.prev_in_medium ? 1u : 0u) | (vw.prev_specular ? 2u : 0u);
                q[4] = make_float4(vw.d_shared, vw.d_bpt, vw.d_pde, vw.for_inv);
                q[5] = make_float4(vw.rev_inv, vw.for_ratio, vw.rev_ratio, ubits(bits));
                q[6] = make_float4(cw.last_sin_theta, cw.d_bpt_a, cw.d_bpt_b, cw.d_pde_a);
                q[7] = make_float4(cw.d_pde_b, ubits(path), ubits(event_key(cam_path_length, kEvSegment)), 0.f);
            }
        }
        if (use_lite) {
            att *= attenuation(m, dmax - dmin);
            if (!is_positive(att)) return;
            float sr;
            const float sf = distance_pdf(m, dmin, dmax, i == 0 ? sflags : 0u, sr);
            fpdf *= sf;
            rpdf *= sr;
        } else {
            if (p.camera_beam_type == kShortBeam)
                att *= segs[i].att / segs[i].pdf_for;
            else
                att *= segs[i].att;
            if (!is_positive(att)) return;
            fpdf *= segs[i].pdf_for;
            rpdf *= segs[i].pdf_rev;
        }
    }
}

// Unpacks segment-query record k: the query, the camera-side MIS state, the
// path weight before the segment and the packed pixel / camera path length.
template <class Fetch>
UPBP_D void read_seg_query(Fetch&& r, QuerySeg& q, StateWeights& cw, float3& weight, unsigned& pk, unsigned& path,
                           unsigned& key)
{
    const float4 q0 = r(0), q1 = r(1), q2 = r(2), q3 = r(3);
    const float4 q4 = r(4), q5 = r(5), q6 = r(6), q7 = r(7);
    q.o = xyz(q0);
    q.dmin = q0.w;
    q.d = xyz(q1);
    q.dmax = q1.w;
    q.med = (int)fbits(q2.w);
    weight = xyz(q2);
    q.for_pdf = q3.x;
    q.rev_pdf = q3.y;
    q.flags = fbits(q3.z);
    pk = fbits(q3.w);
    q.cam_path_length = pk & 0xffu;
    cw.w.d_shared = q4.x;
    cw.w.d_bpt = q4.y;
    cw.w.d_pde = q4.z;
    cw.w.for_inv = q4.w;
    cw.w.rev_inv = q5.x;
    cw.w.for_ratio = q5.y;
    cw.w.rev_ratio = q5.z;
    const unsigned bits = fbits(q5.w);
    cw.w.prev_in_medium = bits & 1u;
    cw.w.prev_specular = (bits >> 1) & 1u;
    cw.last_sin_theta = q6.x;
    cw.d_bpt_a = q6.y;
    cw.d_bpt_b = q6.z;
    cw.d_pde_a = q6.w;
    cw.d_pde_b = q7.x;
    path = fbits(q7.y);
    key = fbits(q7.z);
}

UPBP_D void load_seg_query(unsigned k, QuerySeg& q, StateWeights& cw, float3& weight, unsigned& pk, unsigned& path,
                           unsigned& key)
{
    const float4* r = c_params.seg_queue[k].q;
    read_seg_query([&](int i) { return __ldg(&r[i]); }, q, cw, weight, pk, path, key);
}

// True if the contribution with event key `key` of camera path `path` is one
// the reference makes (no deferred connection of the path failed before it).
UPBP_D bool event_kept(unsigned path, unsigned key) { return key < c_params.path_err[path]; }

// Step of BPT connection k of a vertex (keys stay below the point merges).
UPBP_D unsigned bpt_step(unsigned k) { return min(kEvBpt + k, kEvPoint - 1u); }

// Adds c into pixel px of the camera image (pixel 0xffffff: no pixel).
UPBP_D void splat_camera(unsigned px, float3 c)
{
    if ((c.x != 0.f || c.y != 0.f || c.z != 0.f) && px != 0xffffffu) {
        float* fb = c_params.cam_fb + 3 * (size_t)px;
        atomicAdd(fb + 0, c.x);
        atomicAdd(fb + 1, c.y);
        atomicAdd(fb + 2, c.z);
    }
}

// PB2D, BB1D and BP2D as range queries, each in two kernels.
// A long query segment crosses hundreds of beam chunks (or photons) and a
// short one a few, and every accepted neighbour costs a full MIS evaluation;
// run inside one walk per thread, both leave most lanes of a warp idle.
//
// range_search_kernel<kMode>: persistent warps walk a photon map's compressed
// nodes (QNode) with one query per lane, one internal node per step; a lane
// whose query is finished
// takes the next one in Morton order from a global counter, so lanes stay
// busy until the queue is empty.  A child that is a leaf is not visited: its
// (query, primitive) pair goes into a per-warp ring in shared memory, and
// whenever 32 pairs are waiting all lanes run the exact leaf test on one pair
// each, so the test never runs on a partly idle warp.  Accepted pairs are
// gathered the same way and written out 32 at a time (one atomic per 32
// hits).  A search covers one round of the query order: once the hit list
// is 3/4 full no lane takes a new query, the lanes finish the queries they
// hold, and the host evaluates the list and starts the next round where this
// one stopped.  Pairs past the capacity are dropped but still counted, and
// such a round is repeated.
//
// range_eval_kernel<kMode>: one accepted pair per thread, the records of a
// warp's 32 pairs read together (gather_records); recomputes the pair's
// geometry with the same predicate, evaluates the estimator with its MIS
// weight and adds it into the camera image.
enum : int { kModePb2d = 0, kModeBb1d, kModeBp2d, kRangeModes };
template <int kMode> struct RangeMode {
    static_assert(kMode >= 0 && kMode < kRangeModes, "range-query mode");
    static constexpr bool seg = kMode != kModeBp2d;  // segment queries (else point queries)
    static constexpr bool beams = kMode != kModePb2d;  // beam map (else medium photon map)
    static constexpr int kern = kMode == kModePb2d ? kKernPb2d : kMode == kModeBb1d ? kKernBb1d : kKernBp2d;
    // query geometry of waiting pairs in shared memory (long BB1D queries;
    // the short PB2D and BP2D ones refill lanes too often for its flushes)
    static constexpr bool shared_geo = kMode == kModeBb1d;
};

enum : unsigned { kQuerySurf = 1u, kQueryPp3d = 2u, kQueryBp2d = 4u };

template <int kMode>
UPBP_D const BvhView& range_map_bvh()
{
    const DeviceParams& p = c_params;
    return RangeMode<kMode>::beams ? p.beam_map.bvh : p.med_map.bvh;
}

constexpr int kSearchWarps = 4;
constexpr unsigned kNoQuery = 0xffffffffu;  // no more queries in this round
constexpr unsigned kCandRing = 128;  // > 31 waiting + 64 new pairs per step

// The top kSmemStack entries of each lane's traversal stack live in shared
// memory (column per lane, so lanes never share a bank); deeper entries go
// to local memory.  Local memory competes with the photon maps for L1.
constexpr int kSmemStack = 16;

// A waiting pair names the lane whose query it belongs to in the top bits of
// its leaf word (leaf indices stay below 2^kLeafShift).  With shared_geo the
// lane's query geometry sits in shared memory, so a pair test reads only the
// map's record from global memory; a lane then overwrites its geometry only
// when no pair is waiting.
constexpr unsigned kPairLeafMask = (1u << kLeafShift) - 1u;

struct SearchWarp {
    uint2 cand[kCandRing];  // (query record, map leaf | owner lane << kLeafShift)
    uint2 hit_qb[64];
    int stack[kSmemStack][32];
};
struct SearchWarpGeo : SearchWarp {
    float4 qgeo[2][32];     // per lane: (origin, tmin), (direction, tmax)
};
template <int kMode>
using SearchWarpOf = std::conditional_t<RangeMode<kMode>::shared_geo, SearchWarpGeo, SearchWarp>;
static_assert(kLeafShift + 5 <= 32, "owner lane bits");

// The estimate of one accepted (query, neighbour) pair: the predicate's
// geometry recomputed, the estimator with its MIS weight, added into the
// camera image.  fq(i) and fn(i) return float4 i of the query's record
// (segment query, or a point query's camera vertex) and of the neighbour's
// (beam or light vertex).
template <int kMode, bool kGuided, class FQ, class FN>
UPBP_D void eval_range_hit(uint2 qb, FQ&& fq, FN&& fn)
{
    using M = RangeMode<kMode>;
    const DeviceParams& p = c_params;
    if constexpr (M::seg) {
        QuerySeg q;
        StateWeights cw;
        float3 weight;
        unsigned pk, path, key;
        read_seg_query(fq, q, cw, weight, pk, path, key);
        if (!event_kept(path, key)) return;
        float3 est;
        if constexpr (kMode == kModeBb1d) {
            Beam lb;
            read_beam(fn, lb);
            float dist, sin_theta, t1, t2;
            if (!pred_beam_beam(q.o, q.d, q.dmin, q.dmax, lb.o, lb.d, lb.length, p.radius_bb1d_2, dist, sin_theta,
                                t1, t2))
                return;
            float w = -1.f;
            est = p.bb1d_normalization * eval_bb1d(q, cw, lb, dist, sin_theta, t1, t2, &w, kGuided);
            UPBP_MISDBG(if (w >= 0.f) {
                MisEvent e{kMisBb1d, path, q.cam_path_length, lb.path_idx, lb.path_length, 0u, w,
                           lb.o + lb.d * t2, q.o + q.d * t1, lb.origin_offset + t2, t1, lb.origin_offset};
                mis_event(e, nullptr, 0);
            });
        } else {
            LightVertex lv;
            read_vertex(fn, lv);
            float dist, rad2;
            if (!pred_ray_disc(q.o, q.d, q.dmin, q.dmax, lv.hit, p.radius_pb2d_2, dist, rad2)) return;
            float w = -1.f;
            est = p.pb2d_normalization * eval_pb2d(q, cw, lv, dist, rad2, &w, kGuided);
            UPBP_MISDBG(if (w >= 0.f) {
                MisEvent e{kMisPb2d, path, q.cam_path_length, qb.y / p.slots_per_path, lv.path_length, 0u, w,
                           lv.hit, q.o + q.d * dist, 0.f, dist};
                mis_event(e, nullptr, 0);
            });
        }
        splat_camera(pk >> 8, weight * est);
    } else {
        const float4 q8 = __ldg(&p.pt_queue[qb.x].q8);
        LightVertex cv;
        read_vertex(fq, cv);
        if (!kGuided) cv.bsdf.gcell = -1;  // the unguided instantiation has no proposal code
        Beam lb;
        read_beam(fn, lb);
        float dist, rad2;
        if (!pred_ray_disc(lb.o, lb.d, 0.f, lb.length, cv.hit, p.radius_bp2d_2, dist, rad2)) return;
        float w = -1.f;
        splat_camera(fbits(q8.x),
                     cv.thr * p.bp2d_normalization * eval_bp2d(lb, cv.path_length, cv.w, cv.bsdf, dist, rad2, &w));
        UPBP_MISDBG(if (w >= 0.f) {
            MisEvent e{kMisBp2d, fbits(q8.z), cv.path_length, lb.path_idx, lb.path_length, 0u, w,
                       lb.o + lb.d * dist, cv.hit, lb.origin_offset + dist, 0.f, lb.origin_offset};
            mis_event(e, nullptr, 0);
        });
    }
}

// Leaf tests of the 32 (or, at the end, fewer) oldest waiting pairs, one per
// lane; accepted pairs go to the hit buffer, which is flushed by 32.  A hit
// is (query record, beam) or (query record, light-vertex slot).
template <int kMode>
UPBP_D void search_test_pairs(SearchWarpOf<kMode>& w, unsigned& head, unsigned count, unsigned& hfill, unsigned lane,
                              unsigned& cand, unsigned& hits, unsigned long long& seen)
{
    const DeviceParams& p = c_params;
    const unsigned below = (1u << lane) - 1u;
    __syncwarp();
    bool hit = false;
    uint2 pr = make_uint2(0u, 0u);
    unsigned id = 0;
    if (lane < count) {
        pr = w.cand[(head + lane) % kCandRing];
        const unsigned leaf = pr.y & kPairLeafMask, owner = pr.y >> kLeafShift;
        if constexpr (RangeMode<kMode>::seg) {
            const float4* r = p.seg_queue[pr.x].q;
            float4 q0, q1;
            if constexpr (RangeMode<kMode>::shared_geo) {
                q0 = w.qgeo[0][owner];
                q1 = w.qgeo[1][owner];
            } else {
                q0 = __ldg(&r[0]);
                q1 = __ldg(&r[1]);
            }
            if constexpr (kMode == kModeBb1d) {
                BeamSegHit h;
                hit = beam_chunk_vs_segment(p.beam_map, (int)leaf, xyz(q0), xyz(q1), q0.w, q1.w, p.radius_bb1d_2,
                                            false, p.do_bp2d != 0, -1, &r[2], cand, h);
                id = h.beam;
            } else {
                const float4 pp = __ldg(&p.med_map.pos[leaf]);
                float dist, rad2;
                cand++;
                hit = pred_ray_disc(xyz(q0), xyz(q1), q0.w, q1.w, xyz(pp), p.radius_pb2d_2, dist, rad2);
                id = fbits(pp.w);
            }
        } else {
            // BP2D: beams_near_point's leaf test, the chunk holding the
            // beam's closest point reports it
            const float3 x = xyz(__ldg(&p.pt_queue[pr.x].v.q[0]));
            const float4 s0 = __ldg(&p.beam_map.seg[3 * leaf]), s1 = __ldg(&p.beam_map.seg[3 * leaf + 1]);
            float dist, rad2;
            cand++;
            if (pred_ray_disc(xyz(s0), xyz(s1), 0.f, s0.w, x, p.radius_bp2d_2, dist, rad2)) {
                const float4 s2 = __ldg(&p.beam_map.seg[3 * leaf + 2]);  // the chunk's range, for accepted pairs only
                hit = dist >= s2.x && dist < s2.y;
            }
            id = fbits(s1.w) & 0x7fffffffu;
        }
    }
    head += count;
    const unsigned hm = __ballot_sync(~0u, hit);
    if (hit) {
        const unsigned pos = hfill + __popc(hm & below);
        w.hit_qb[pos] = make_uint2(pr.x, id);
        hits++;
    }
    hfill += __popc(hm);
    if (hfill >= 32) {
        __syncwarp();
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&p.hit_state->total, 32ull);
        base = __shfl_sync(~0u, base, 0);
        seen = base + 32;
        if (base + lane < p.hit_capacity) p.hit_qb[base + lane] = w.hit_qb[lane];
        __syncwarp();
        if (lane + 32 < hfill) w.hit_qb[lane] = w.hit_qb[lane + 32];
        hfill -= 32;
    }
    __syncwarp();
}

template <int kMode>
__global__ void __launch_bounds__(128) range_search_kernel(int slot)
{
    using M = RangeMode<kMode>;
    begin_kernel(M::kern, slot);
    const DeviceParams& p = c_params;
    __shared__ SearchWarpOf<kMode> s_warp[kSearchWarps];
    SearchWarpOf<kMode>& w = s_warp[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    // this round's range of the processing order, within the queue
    const unsigned nq = M::seg ? min(p.queue_count[0], p.seg_capacity) : min(p.queue_count[1], p.pt_capacity);
    const unsigned n = min(p.query_end, nq) - min(p.query_begin, min(p.query_end, nq));
    unsigned long long seen = 0;  // hit total after this warp's last flush
    const BvhView bvh = range_map_bvh<kMode>();
    int node = kWalkDone, sp = 0;
    int deep[kStackDepth - kSmemStack];
    float3 inv = v3(0.f), oinv = v3(0.f), x = v3(0.f);
    float tmin = 0.f, tmax = 0.f;
    unsigned qk = 0;
    bool exhausted = false;  // no queries left for this warp (the same in every lane)
    bool overflow = false;
    unsigned head = 0, tail = 0, hfill = 0;  // same values in every lane
    unsigned visits = 0, cand = 0, hits = 0;
    for (;;) {
        // primitives of the leaf children reached this step (a compressed
        // node's leaves hold one primitive each), -1 for none
        int leaf0 = -1, leaf1 = -1;
        const unsigned idle = __ballot_sync(~0u, node == kWalkDone);
        if (exhausted && idle == ~0u) break;
        const unsigned want = exhausted ? 0u : idle;
        if (want) {
            // a lane that takes a new query overwrites its geometry: test the
            // pairs still waiting first
            if (M::shared_geo && tail != head)
                search_test_pairs<kMode>(w, head, tail - head, hfill, lane, cand, hits, seen);
            // no new queries once the hit list is 3/4 full, as far as this
            // warp saw at its last flush of hits (no extra load of the
            // counter, which every flush and request updates)
            const int leader = __ffs(want) - 1;
            unsigned base = kNoQuery;
            if ((int)lane == leader && seen < p.hit_soft_limit)
                base = atomicAdd(&p.hit_state->fetched, (unsigned)__popc(want));
            base = __shfl_sync(~0u, base, leader);
            // the queue is used up once a lane's index falls past its end
            if (base == kNoQuery || base + (unsigned)__popc(want) > n) exhausted = true;
            if ((want >> lane) & 1u) {
                const unsigned r = base + __popc(want & below);
                bool take = base != kNoQuery && r < n;
                const unsigned j = p.query_begin + r;
                if (take) {
                    if constexpr (M::seg) {
                        qk = p.seg_order ? __ldg(&p.seg_order[j]) : j;
                        const float4* r = p.seg_queue[qk].q;
                        const float4 q0 = __ldg(&r[0]), q1 = __ldg(&r[1]);
                        tmin = q0.w;
                        tmax = q1.w;
                        inv = safe_inv(xyz(q1));
                        oinv = oinv_of(xyz(q0), inv);
                        if constexpr (M::shared_geo) {
                            w.qgeo[0][lane] = q0;
                            w.qgeo[1][lane] = q1;
                        }
                    } else {
                        // point queries of other estimators, or of camera paths
                        // that failed earlier, are skipped
                        qk = p.pt_order ? __ldg(&p.pt_order[j]) : j;
                        const float4 q8 = __ldg(&p.pt_queue[qk].q8);
                        take = (fbits(q8.y) & kQueryBp2d) && event_kept(fbits(q8.z), fbits(q8.w));
                        x = xyz(__ldg(&p.pt_queue[qk].v.q[0]));
                    }
                }
                if (take) {
                    sp = 0;
                    node = bvh.count > 1 ? 0 : kWalkDone;
                    if (bvh.count == 1) {  // a one-leaf map
                        leaf0 = 0;
                    }
                }
            }
        }
        if (node != kWalkDone) {
            // one internal node: leaf children become pairs, internal ones are visited
            visits++;
            bool hl, hr;
            int cl, cr;
            if constexpr (M::seg) {
                qnode_slab(bvh.qnodes, node, inv, oinv, tmin, tmax, hl, hr, cl, cr);
            } else {
                const NodeBoxes nb = load_qnode(bvh.qnodes, node);
                hl = inside(nb.llo, nb.lhi, x);
                hr = inside(nb.rlo, nb.rhi, x);
                cl = nb.l;
                cr = nb.r;
            }
            int next = -1, other = -1;
            if (hl) {
                if (cl < 0) {
                    leaf0 = leaf_first(cl);
                } else {
                    next = cl;
                }
            }
            if (hr) {
                if (cr < 0) {
                    leaf1 = leaf_first(cr);
                } else if (next < 0) {
                    next = cr;
                } else {
                    other = cr;
                }
            }
            if (other >= 0) {
                if (sp < kSmemStack)
                    w.stack[sp++][lane] = other;
                else if (sp < kStackDepth)
                    deep[sp++ - kSmemStack] = other;
                else
                    overflow = true;
            }
            if (next >= 0) {
                node = next;
            } else if (sp > 0) {
                --sp;
                node = sp < kSmemStack ? w.stack[sp][lane] : deep[sp - kSmemStack];
            } else {
                node = kWalkDone;
            }
        }
        // each reached leaf becomes a waiting pair (a lane adds up to two,
        // next to each other); 32 waiting pairs are tested at once.  The
        // walk tests compressed boxes, which contain the exact ones: the leaf
        // test re-checks a chunk's own box where it matters.
        {
            const unsigned m0 = __ballot_sync(~0u, leaf0 >= 0), m1 = __ballot_sync(~0u, leaf1 >= 0);
            unsigned at = tail + __popc(m0 & below) + __popc(m1 & below);
            if (leaf0 >= 0) w.cand[at++ % kCandRing] = make_uint2(qk, (unsigned)leaf0 | (lane << kLeafShift));
            if (leaf1 >= 0) w.cand[at % kCandRing] = make_uint2(qk, (unsigned)leaf1 | (lane << kLeafShift));
            tail += __popc(m0) + __popc(m1);
#pragma unroll 1
            while (tail - head >= 32) search_test_pairs<kMode>(w, head, 32, hfill, lane, cand, hits, seen);
        }
    }
    if (tail != head) search_test_pairs<kMode>(w, head, tail - head, hfill, lane, cand, hits, seen);
    __syncwarp();
    if (hfill) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&p.hit_state->total, (unsigned long long)hfill);
        base = __shfl_sync(~0u, base, 0);
        if (lane < hfill && base + lane < p.hit_capacity) p.hit_qb[base + lane] = w.hit_qb[lane];
    }
    count_work(kCtrNodes, visits);
    count_work(M::beams ? kCtrBeamCand : kCtrPointCand, cand);
    count_work(M::beams ? kCtrBeamHit : kCtrPointHit, hits);
    if (overflow) flag_status(kErrTraversalStack);
}

// The 128-byte records of a warp's 32 hits, read together: eight lanes load
// one record as consecutive 16-byte pieces (four records per instruction, a
// coalesced access each, instead of eight lookups per lane at unrelated
// addresses, which kept the L1 busy), then every lane takes its own record
// from shared memory (rows padded to 144 bytes, so the eight lanes of a
// quarter-warp read different banks).  rec is this lane's record.
constexpr int kEvalWarps = 4;
UPBP_D void gather_records(const float4* rec, float4 (&out)[8], float4 (*s)[9], unsigned lane)
{
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const unsigned r = 4u * k + (lane >> 3);
        const auto rp = reinterpret_cast<const float4*>(
            __shfl_sync(~0u, reinterpret_cast<unsigned long long>(rec), (int)r));
        s[r][lane & 7u] = __ldg(rp + (lane & 7u));
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = s[lane][i];
}

// One warp per 32 consecutive hits; lanes past the end read the warp's
// first hit's records and evaluate nothing.
// kGuided: a learned-proposal table is in use (the unguided instantiation,
// the common case, contains none of the proposal's code).
template <int kMode, bool kGuided>
__global__ void __launch_bounds__(128, 7) range_eval_kernel(int slot)
{
    using M = RangeMode<kMode>;
    begin_kernel(M::kern, slot);
    const DeviceParams& p = c_params;
    __shared__ float4 s_rec[kEvalWarps][32][9];
    float4(*s)[9] = s_rec[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned n = (unsigned)min(p.hit_state->total, (unsigned long long)p.hit_capacity);
    for (unsigned base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x) {
        const unsigned j = base + lane;
        const uint2 qb = __ldg(&p.hit_qb[j < n ? j : base]);
        const float4* qrec;
        const float4* nrec;
        if constexpr (M::seg)
            qrec = p.seg_queue[qb.x].q;
        else
            qrec = p.pt_queue[qb.x].v.q;
        if constexpr (M::beams)
            nrec = p.beams[qb.y].q;
        else
            nrec = p.vertices[qb.y].q;
        float4 qa[8], na[8];
        gather_records(qrec, qa, s, lane);
        gather_records(nrec, na, s, lane);
        if (j < n) eval_range_hit<kMode, kGuided>(qb, [&](int i) { return qa[i]; }, [&](int i) { return na[i]; });
    }
}

// SURF and PP3D for one point-query record per thread, evaluated inline:
// their walks are short and their hits few, so the search / evaluation split
// (kept for PB2D, BB1D and BP2D) costs more than it saves here.
template <bool medium, bool kGuided>
__global__ void __launch_bounds__(128) point_merge_kernel(int slot)
{
    begin_kernel(medium ? kKernPp3d : kKernSurf, slot);
    const DeviceParams& p = c_params;
    const PointMap& map = medium ? p.med_map : p.surf_map;
    const float r2 = medium ? p.radius_pp3d_2 : p.radius_surf_2;
    const unsigned n = min(p.queue_count[1], p.pt_capacity);
    for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const unsigned k = p.pt_order ? __ldg(&p.pt_order[j]) : j;
        const float4 q8 = __ldg(&p.pt_queue[k].q8);
        if (!(fbits(q8.y) & (medium ? kQueryPp3d : kQuerySurf)) || !event_kept(fbits(q8.z), fbits(q8.w))) continue;
        LightVertex cv;
        load_vertex(&p.pt_queue[k].v, cv);
        if (!kGuided) cv.bsdf.gcell = -1;  // the unguided instantiation has no proposal code
        float3 acc = v3(0.f);
        points_in_radius(map, cv.hit, r2, [&](unsigned slot) {
            LightVertex lv;
            load_vertex(p.vertices + slot, lv);
            float w = -1.f;
            acc += eval_point_merge(lv, cv.path_length, cv.w, cv.bsdf, medium, &w);
            UPBP_MISDBG(if (w >= 0.f) {
                MisEvent e{medium ? kMisPp3d : kMisSurf, fbits(q8.z), cv.path_length, slot / p.slots_per_path,
                           lv.path_length, 0u, w, lv.hit, cv.hit, 0.f, 0.f};
                mis_event(e, nullptr, 0);
            });
        });
        splat_camera(fbits(q8.x), cv.thr * (medium ? p.pp3d_normalization : p.surf_normalization) * acc);
    }
}

// State of one camera subpath between bounces.
struct CameraLane {
    PathState s;
    Rng rng;
    float3 color;
    unsigned path;    // the pixel the path was generated for (its random stream)
    unsigned target;  // pixel the sample lands in, kNoPixel if off screen
    unsigned ret;     // status of a failed step (0: none)
    bool origin_in_medium;
    bool only_spec_surf;
};

constexpr unsigned kNoPixel = 0xffffffu;

// Appends the camera vertex of deferred connections; returns its record
// index (past the capacity the record is counted but not written, and the
// host grows the queue and repeats the camera pass).
UPBP_D unsigned store_conn_vertex(float3 hit, const PathState& s, const Bsdf& bsdf, float3 frame_src, bool behind,
                                  unsigned pixel, unsigned path)
{
    const DeviceParams& p = c_params;
    const unsigned k = warp_reserve1(&p.queue_count[3]);
    if (k >= p.conn_capacity) return k;
    ConnVertexRec* r = p.conn_vertices + k;
    store_vertex(&r->v, hit, s.throughput, s.path_length, bsdf.in_medium(), behind, bsdf, frame_src, s.sw.w);
    r->q8 = make_float4(ubits(pixel), ubits((unsigned)s.stack.size), ubits(path), ubits(s.path_length));
    for (int i = 0; i < s.stack.size; i++) r->stack[i] = make_int2(s.stack.el[i].mat, s.stack.el[i].med);
    return k;
}

// The boundary stack of a connection vertex (priorities from the materials,
// as every push computes them).
UPBP_D void load_conn_stack(const ConnVertexRec* r, unsigned size, BoundaryStack& st)
{
    for (unsigned i = 0; i < size; i++) {
        const int2 e = r->stack[i];
        st.el[i] = Boundary{e.x, e.y};
        st.pri[i] = boundary_priority(e.x);
    }
    st.size = (int)size;
}

// Starts the camera subpath of `pixel`; false if it ended already.
UPBP_D bool camera_path_begin(CameraLane& c, unsigned pixel)
{
    const DeviceParams& p = c_params;
    c.path = pixel;
    c.rng.init(p.iteration + p.iteration_offset, pixel, 1u);
    float2 screen;
    c.ret = generate_camera_sample(screen, pixel, c.s, c.rng);
    c.color = v3(0.f);
    // add_color (frame_buffer.cuh:36-45) targets the pixel of the jittered
    // sample, which float rounding can move to the next pixel or off screen
    c.target = kNoPixel;
    if (!(screen.x < 0.f || screen.x >= (float)p.res_x || screen.y < 0.f || screen.y >= (float)p.res_y))
        c.target = (unsigned)int(screen.x) + (unsigned)int(screen.y) * p.res_x;
    c.origin_in_medium = false;
    c.only_spec_surf = (p.estimator_techniques & (kPrevious | kCompatible)) != 0;
    return c.ret == 0;
}

// One bounce of a camera subpath (one iteration of the path loop of
// __raygen__trace_camera, trace_camera.cu:79-381); false when the path ends.
UPBP_D bool camera_path_bounce(CameraLane& c, VolSeg* segs, LiteSeg* lsegs)
{
    const DeviceParams& p = c_params;
    PathState& s = c.s;
    Rng& rng = c.rng;
    float3& color = c.color;
    const unsigned target = c.target;
    bool& origin_in_medium = c.origin_in_medium;
    bool& only_spec_surf = c.only_spec_surf;
    unsigned& ret = c.ret;
    const float3 ro = s.origin, rd = s.dir;
    Isect isect;
    isect.dist = kInfinity;
    isect.mat = isect.med = isect.light = -1;
    isect.normal = v3(0.f);
    isect.enter = false;
    int nseg = 0, nlseg = 0;
    bool hit;
    ret = intersect_scene(hit, ro, rd, isect, s.stack, kSampleScattering, origin_in_medium ? kOriginInMedium : 0u,
                          segs, nseg, lsegs, nlseg, rng);
    if (ret) return false;
    UPBP_MISDBG(mis_ray(false, c.path, s.path_length, rd, hit ? isect.dist : kInfinity,
                        origin_in_medium ? kOriginInMedium : 0u, lsegs, nlseg));
    if ((p.build_pb2d && p.n_medium > 0) || (p.build_bb1d && p.n_beams > 0)) {
        const unsigned qflags = origin_in_medium ? kOriginInMedium : 0u;
        const bool use_lite = !(isect.on_surface() || p.camera_beam_type == kShortBeam || !hit);
        emit_segment_queries(ro, rd, segs, nseg, lsegs, nlseg, use_lite, qflags, s.path_length, s.sw, s.throughput,
                             target, c.path);
    }
    if (!hit) {
        if (s.path_length < p.min_path_length) return false;
        if (p.background_light < 0) return false;
        if (p.media[p.global_medium].has_attenuation) return false;
    }
    float rs_for = 1.f, rs_rev = 1.f;
    if (nseg > 0) {
        rs_for = seg_for_pdf(segs, nseg);
        rs_rev = seg_rev_pdf(segs, nseg);
        s.throughput *= seg_attenuation(segs, nseg) / rs_for;
    }
    if (is_black_or_negative(s.throughput)) return false;
    VertexWeights& w = s.sw.w;
    if (s.path_length > 1u) {
        const float f_i = pde_factor(w.prev_in_medium, w.prev_specular, 1.f / rs_rev, w.rev_ratio, w.for_inv,
                                     w.for_ratio, s.sw.last_sin_theta);
        w.d_bpt = s.sw.d_bpt_a * f_i + s.sw.d_bpt_b;
        w.d_pde = s.sw.d_pde_a * f_i + s.sw.d_pde_b;
    }
    w.d_shared /= rs_for;
    w.d_bpt /= rs_for;
    w.d_pde /= rs_for;
    if (!hit) {
        color += s.throughput * light_hit_radiance(p.lights[p.background_light], s, rs_rev);
        return false;
    }
    Bsdf bsdf;
    if (isect.on_surface())
        bsdf_setup_surface(bsdf, rd, isect.normal, isect.shading_normal, isect.mat, false, relative_ior(isect, s.stack));
    else
        bsdf_setup_medium(bsdf, rd, isect.med, false, ro + rd * isect.dist);
    if (!bsdf.valid()) return false;
    float ratio = 0.f;
    if (bsdf.in_medium()) ratio = 1.f / p.media[bsdf.id].min_pos_att;
    const float3 hitpoint = ro + rd * isect.dist;
    origin_in_medium = isect.in_medium();
    UPBP_MISDBG(mis_hit(false, c.path, s.path_length, hitpoint, isect.in_medium(),
                        isect.in_medium() ? isect.med : isect.mat, isect.in_medium() ? v3(0.f) : isect.shading_normal,
                        isect.in_medium() ? v3(0.f) : isect.normal, bsdf.delta(), bsdf.cont_prob));
    {
        const float d = bsdf.d_factor();
        w.d_shared *= isect.dist * isect.dist;
        w.d_shared /= d;
        w.d_bpt /= d;
        w.d_pde /= d;
        w.for_inv = 1.f / rs_for;
        w.rev_inv = 1.f / rs_rev;
        w.for_ratio = ratio;
        w.rev_ratio = ratio;
    }
    if (isect.light >= 0) {
        if (s.path_length < p.min_path_length) return false;
        float wl = -1.f;
        color += s.throughput * light_hit_radiance(p.lights[isect.light], s, rs_rev, &wl);
        UPBP_MISDBG({
            mis_hit_light(c.path, s.path_length, hitpoint, isect.light, isect.normal);
            if (wl >= 0.f) {
                MisEvent e{kMisEmitterHit, c.path, s.path_length, 0u, 0u, (unsigned)isect.light, wl, hitpoint, hitpoint,
                           0.f, 0.f};
                mis_event(e, nullptr, 0);
            }
        });
        return false;
    }
    if (s.path_length >= p.max_path_length) return false;
    // NEE and BPT connections: the samples are drawn here, from this path's
    // random stream and in the reference's order; their occlusion rays are
    // traced by nee_connect_kernel and bpt_connect_kernel, one per thread.
    const bool connect = p.do_bpt && !bsdf.delta() && (bsdf.in_medium() || !only_spec_surf);
    NeeSample ns;
    bool nee = false;
    if (connect && s.path_length + 1 >= p.min_path_length && p.light_count > 0)
        nee = nee_sample(ns, hitpoint, bsdf, rng);
    unsigned nv = 0, lp = 0;
    bool behind = false;
    if (connect) {
        if (bsdf.in_medium() && s.stack.size > 0) {
            const int mid = s.stack.top().mat;
            if (mid >= 0 && p.materials[mid].real) behind = true;
        }
        lp = (unsigned)int(rng.uniform() * p.light_subpath_count);
        nv = p.path_vertex_count[lp];
    }
    if ((nee || nv > 0) && target != kNoPixel) {
        const float3 frame_src = bsdf.on_surface() ? isect.shading_normal : rd;
        const unsigned v = store_conn_vertex(hitpoint, s, bsdf, frame_src, behind, target, c.path);
        if (nee) {
            const unsigned k = warp_reserve1(&p.queue_count[4]);
            if (k < p.nee_capacity && v < p.conn_capacity) {
                float4* q = p.nee_queue[k].q;
                q[0] = make_float4(hitpoint.x, hitpoint.y, hitpoint.z, ns.dist);
                q[1] = make_float4(ns.dir.x, ns.dir.y, ns.dir.z, ubits(v));
                q[2] = make_float4(ns.rad.x, ns.rad.y, ns.rad.z, ns.k);
                q[3] = make_float4(ns.f.x, ns.f.y, ns.f.z, ns.w_light);
                q[4] = make_float4(ns.a, ns.rpdf, ns.sin_theta,
                                   ubits((bsdf.in_medium() ? 1u : 0u) UPBP_MISDBG(| ((unsigned)ns.light << 1))));
            }
        }
        if (nv > 0) {
            const unsigned k = warp_reserve(&p.queue_count[5], nv);
            if (v < p.conn_capacity)
                for (unsigned i = 0; i < nv && k + i < p.bpt_capacity; i++)
                    p.bpt_pairs[k + i] = make_uint2(v, lp * p.slots_per_path + i);
        }
    }
    {
        unsigned mask = 0;
        if (p.build_surf && p.n_surface > 0 && bsdf.on_surface() && !bsdf.delta() && !only_spec_surf)
            mask |= kQuerySurf;
        if (p.build_pp3d && p.n_medium > 0 && bsdf.in_medium() && !bsdf.delta()) mask |= kQueryPp3d;
        if (p.build_bp2d && p.n_beams > 0 && bsdf.in_medium()) mask |= kQueryBp2d;
        if (mask) {
            const unsigned k = warp_reserve1(&p.queue_count[1]);
            if (k < p.pt_capacity) {
                PointQueryRec* rec = p.pt_queue + k;
                const float3 frame_src = bsdf.on_surface() ? isect.shading_normal : rd;
                store_vertex(&rec->v, hitpoint, s.throughput, s.path_length, bsdf.in_medium(), false, bsdf,
                             frame_src, s.sw.w);
                rec->q8 = make_float4(ubits(target), ubits(mask), ubits(c.path),
                                      ubits(event_key(s.path_length, kEvPoint)));
            }
        }
    }
    bool cont;
    ret = sample_scattering(cont, bsdf, hitpoint, isect, s, rng);
    if (ret || !cont) return false;
    UPBP_MISDBG(if (s.sw.w.prev_specular) mis_specular(false, c.path, s.path_length));
    if (bsdf.on_surface()) {
        if (!s.sw.w.prev_specular && (only_spec_surf || (p.estimator_techniques & kSpecularOnly))) return false;
    } else {
        if (p.estimator_techniques & kSpecularOnly) return false;
        if (only_spec_surf) {
            if (p.estimator_techniques & kCompatible)
                only_spec_surf = false;
            else
                return false;
        }
    }
    s.path_length++;
    return true;
}

// Ends a camera subpath: its status and its emitter-hit colour, which
// k_resolve_camera adds once the deferred connections of the path are done.
UPBP_D void camera_path_end(const CameraLane& c)
{
    if (c.ret) flag_status(c.ret);
    c_params.path_color[c.path] = make_float4(c.color.x, c.color.y, c.color.z, ubits(c.target));
}

// Camera pass (extend): persistent warps, one camera subpath per lane.  Path
// lengths differ widely (an escaping ray ends after one bounce, a ray in a
// dense medium scatters up to the maximum), so a lane whose path ended takes
// the next pixel from a global counter instead of idling until the longest
// path of its warp is done.  Each pixel's random stream depends on the pixel
// alone, so the assignment of pixels to lanes does not change any path.
__global__ void __launch_bounds__(128, 8) camera_pass_kernel(int slot)
{
    begin_kernel(kKernCameraExtend, slot);
    const DeviceParams& p = c_params;
    VolSeg segs[kMaxVolSegments];
    LiteSeg lsegs[kMaxVolSegments];
    CameraLane c;
    const unsigned lane = threadIdx.x & 31;
    const unsigned n = p.screen_pixel_count;
    bool active = false, exhausted = false;
    for (;;) {
        const unsigned want = __ballot_sync(~0u, !active && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned base = 0;
            if ((int)lane == leader) base = atomicAdd(&p.queue_count[2], (unsigned)__popc(want));
            base = __shfl_sync(~0u, base, leader);
            if (!active && !exhausted) {
                const unsigned j = base + __popc(want & ((1u << lane) - 1u));
                if (j < n) {
                    active = camera_path_begin(c, j);
                    if (!active) camera_path_end(c);
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(~0u, exhausted && !active)) break;
        if (active && !camera_path_bounce(c, segs, lsegs)) {
            camera_path_end(c);
            active = false;
        }
    }
}

// Deferred NEE: one light sample per thread -- occlusion ray through the
// media, MIS weight, throughput.  The contribution is kept per sample until
// k_resolve_camera knows whether an earlier step of the path failed.
__global__ void __launch_bounds__(128, 8) nee_connect_kernel(int slot)
{
    begin_kernel(kKernNee, slot);
    const DeviceParams& p = c_params;
    const unsigned n = min(p.queue_count[4], p.nee_capacity);
    VolSeg segs[kMaxVolSegments];
    BoundaryStack st;
    for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const float4* q = p.nee_queue[j].q;
        const float4 q0 = __ldg(&q[0]), q1 = __ldg(&q[1]), q2 = __ldg(&q[2]), q3 = __ldg(&q[3]), q4 = __ldg(&q[4]);
        NeeSample ns;
        const float3 hit = xyz(q0);
        ns.dist = q0.w;
        ns.dir = xyz(q1);
        ns.rad = xyz(q2);
        ns.k = q2.w;
        ns.f = xyz(q3);
        ns.w_light = q3.w;
        ns.a = q4.x;
        ns.rpdf = q4.y;
        ns.sin_theta = q4.z;
        const bool in_medium = (fbits(q4.w) & 1u) != 0;
        const ConnVertexRec* cr = p.conn_vertices + fbits(q1.w);
        const float4 thr = __ldg(&cr->v.q[1]), w2 = __ldg(&cr->v.q[2]), w3 = __ldg(&cr->v.q[3]);
        const float4 q8 = __ldg(&cr->q8);
        VertexWeights wc;
        wc.d_shared = w2.x;
        wc.d_bpt = w2.y;
        wc.d_pde = w2.z;
        wc.for_inv = w2.w;
        wc.rev_inv = w3.x;
        wc.for_ratio = w3.y;
        wc.rev_ratio = w3.z;
        wc.prev_in_medium = (fbits(w3.w) >> 28) & 1u;
        wc.prev_specular = (fbits(w3.w) >> 29) & 1u;
        load_conn_stack(cr, fbits(q8.y), st);
        float3 c;
        float w = -1.f;
        int nseg = 0;
        const unsigned e = nee_finish(c, ns, hit, in_medium, st, wc, segs, &w, &nseg);
        UPBP_MISDBG(if (!e && w >= 0.f) {
            MisEvent ev{kMisNee, fbits(q8.z), fbits(q8.w), 0u, 0u, fbits(q4.w) >> 1, w, hit + ns.dir * ns.dist, hit,
                        0.f, 0.f};
            mis_event(ev, segs, nseg);
        });
        if (e) {
            // the reference ends the camera path at a failed step
            flag_status(e);
            atomicMin(&p.path_err[fbits(q8.z)], event_key(fbits(q8.w), kEvNee));
            c = v3(0.f);
        }
        const float3 col = xyz(thr) * c;
        p.nee_color[j] = make_float4(col.x, col.y, col.z, 0.f);
    }
}

// Deferred BPT: one (camera vertex, light vertex) pair per thread -- the
// path-length and media checks of the connection loop, then the connection
// with its occlusion ray; the contribution is kept per pair like NEE's.
__global__ void __launch_bounds__(128, 8) bpt_connect_kernel(int slot)
{
    begin_kernel(kKernBpt, slot);
    const DeviceParams& p = c_params;
    const unsigned n = min(p.queue_count[5], p.bpt_capacity);
    VolSeg segs[kMaxVolSegments];
    PathState ps;
    unsigned loads = 0;
    for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint2 pr = __ldg(&p.bpt_pairs[j]);
        const ConnVertexRec* cr = p.conn_vertices + pr.x;
        p.bpt_color[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        LightVertex lv, cv;
        load_vertex(p.vertices + pr.y, lv);
        loads++;
        load_vertex(&cr->v, cv);
        const unsigned plen = lv.path_length + 1 + cv.path_length;
        if (plen > p.max_path_length || plen < p.min_path_length) continue;
        const bool diff_media = lv.bsdf.in_medium() && cv.bsdf.in_medium() && lv.bsdf.id != cv.bsdf.id &&
                                (lv.behind_surf || cv.behind_surf);
        if (diff_media) continue;
        const float4 q8 = __ldg(&cr->q8);
        load_conn_stack(cr, fbits(q8.y), ps.stack);
        ps.sw.w = cv.w;
        Rng unused;
        unused.state = unused.inc = 0;  // occlusion rays draw no random numbers
        float3 c;
        float w = -1.f;
        int nseg = 0;
        const unsigned e = connect_vertices(c, lv, cv.bsdf, cv.hit, ps, unused, segs, &w, &nseg);
        UPBP_MISDBG(if (!e && w >= 0.f) {
            MisEvent ev{kMisBpt, fbits(q8.z), fbits(q8.w), pr.y / p.slots_per_path, lv.path_length, 0u, w, lv.hit,
                        cv.hit, 0.f, 0.f};
            mis_event(ev, segs, nseg);
        });
        if (e) {
            // the reference ends the camera path at a failed connection
            flag_status(e);
            atomicMin(&p.path_err[fbits(q8.z)], event_key(fbits(q8.w), bpt_step(pr.y % p.slots_per_path)));
            continue;
        }
        const float3 col = cv.thr * lv.thr * c;
        p.bpt_color[j] = make_float4(col.x, col.y, col.z, 0.f);
    }
    count_work(kCtrVertexLoads, loads);
}

// Adds the deferred connections and the emitter-hit colours into the camera
// image, each only if no earlier step of its camera path failed: NEE samples,
// then BPT pairs, then one colour per camera path.
__global__ void __launch_bounds__(256) k_resolve_camera(int slot)
{
    begin_kernel(kKernCameraExtend, slot);
    const DeviceParams& p = c_params;
    const unsigned nn = min(p.queue_count[4], p.nee_capacity);
    const unsigned nb = min(p.queue_count[5], p.bpt_capacity);
    const unsigned total = nn + nb + p.screen_pixel_count;
    for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        if (j < nn) {
            const float4 c = p.nee_color[j];
            if (c.x == 0.f && c.y == 0.f && c.z == 0.f) continue;
            const float4 q8 = __ldg(&p.conn_vertices[fbits(__ldg(&p.nee_queue[j].q[1]).w)].q8);
            if (event_kept(fbits(q8.z), event_key(fbits(q8.w), kEvNee))) splat_camera(fbits(q8.x), xyz(c));
        } else if (j < nn + nb) {
            const unsigned k = j - nn;
            const float4 c = p.bpt_color[k];
            if (c.x == 0.f && c.y == 0.f && c.z == 0.f) continue;
            const uint2 pr = __ldg(&p.bpt_pairs[k]);
            const float4 q8 = __ldg(&p.conn_vertices[pr.x].q8);
            if (event_kept(fbits(q8.z), event_key(fbits(q8.w), bpt_step(pr.y % p.slots_per_path))))
                splat_camera(fbits(q8.x), xyz(c));
        } else {
            const unsigned path = j - nn - nb;
            const float4 c = p.path_color[path];
            // an emitter hit ends its path, after every connection of the path
            if (p.path_err[path] == ~0u) splat_camera(fbits(c.w), xyz(c));
        }
    }
}

// Morton keys of the query records (segment midpoint / vertex position in
// the scene's bounding cube), so the query kernels walk spatially coherent
// warps through the photon maps.
template <bool kSeg>
__global__ void k_query_keys(int slot, unsigned n, unsigned* keys, unsigned* vals)
{
    begin_kernel(kKernCameraExtend, slot);
    const DeviceParams& p = c_params;
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float3 x;
    if (kSeg) {
        const float4 q0 = p.seg_queue[k].q[0], q1 = p.seg_queue[k].q[1];
        const float t = q1.w < 1e30f ? .5f * (q0.w + q1.w) : q0.w;
        x = xyz(q0) + xyz(q1) * t;
    } else {
        x = xyz(p.pt_queue[k].v.q[0]);
    }
    const float inv = .5f / p.scene_radius;
    const float3 u = (x - p.scene_center) * inv + v3(.5f);
    keys[k] = morton3(u);
    vals[k] = k;
}

// Adds the camera image into the iteration image (which holds the light
// tracer's splats) and the iteration image into the accumulation.
__global__ void k_finish_iteration(float* fb, const float* cam_fb, double* acc, unsigned n)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = fb[i] + cam_fb[i];
    fb[i] = v;
    acc[i] += (double)v;
}

}  // namespace upbp
