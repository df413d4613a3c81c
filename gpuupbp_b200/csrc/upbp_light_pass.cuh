// Light pass: one thread per light subpath.  Emission, tracing through media,
// photon-beam and light-vertex records, light-to-camera splats.
// Follows __raygen__trace_light (gpuupbp/kernel/trace_light.cu:42-325) and
// generate_light_sample / add_beams / connect_to_camera
// (gpuupbp/kernel/functs_light.cuh:86-388).
#pragma once

#include "upbp_paths.cuh"

namespace upbp {

UPBP_D unsigned generate_light_sample(PathState& s, Rng& rng, unsigned path_idx)
{
    const DeviceParams& p = c_params;
    const float lc = (float)p.light_count;
    const int lid = int(rng.uniform() * lc);
    const float d0 = rng.uniform(), d1 = rng.uniform(), p0 = rng.uniform(), p1 = rng.uniform();
    const DLight& l = p.lights[lid];
    float emission_pdf_w, direct_pdf_a, cos_light;
    s.throughput = light_emit(l, d0, d1, p0, p1, s.origin, s.dir, emission_pdf_w, direct_pdf_a, cos_light);
    emission_pdf_w /= lc;
    direct_pdf_a /= lc;
    s.throughput /= emission_pdf_w;
    UPBP_MISDBG(mis_origin(true, path_idx, s.origin, l.frame.z, (unsigned)lid));
    s.path_length = 1;
    s.is_infinite_light = !light_is_finite(l);
    s.is_specular_path = false;
    VertexWeights& w = s.sw.w;
    w.d_shared = direct_pdf_a / emission_pdf_w;
    if (!light_is_delta(l)) {
        const float used_cos = light_is_finite(l) ? cos_light : 1.f;
        w.d_bpt = used_cos / emission_pdf_w;
    } else {
        w.d_bpt = 0.f;
    }
    w.d_pde = w.d_bpt * p.subpath_count_bpt;
    w.prev_specular = false;
    w.prev_in_medium = false;
    if (!init_boundary_stack(s.stack)) return kErrBoundaryStack;
    if (l.mat_id != -1 && l.med_id != -1) {
        if (!s.stack.push(Boundary{l.mat_id, l.med_id}, boundary_priority(l.mat_id))) return kErrBoundaryStack;
    }
    return 0;
}

// Photon beams along the traced ray (functs_light.cuh:159-247).
UPBP_D void add_beams(float3 ro, float3 rd, float3 throughput, unsigned path_length, unsigned sflags,
                      const VolSeg* segs, int nseg, const LiteSeg* lsegs, int nlseg, unsigned path_idx,
                      const PathState& s)
{
    const DeviceParams& p = c_params;
    float3 thr = throughput;
    float fpdf = 1.f, rpdf = 1.f;
    Beam b;
    b.d = rd;
    b.path_idx = path_idx;
    b.sw = s.sw;
    b.path_length = path_length;
    b.infinite = s.is_infinite_light;
    const bool short_beams = p.photon_beam_type == kShortBeam;
    const int n = short_beams ? nseg : nlseg;
    for (int i = 0; i < n; i++) {
        const float dmin = short_beams ? segs[i].dmin : lsegs[i].dmin;
        const float dmax = short_beams ? segs[i].dmax : lsegs[i].dmax;
        const int med = short_beams ? segs[i].med : lsegs[i].med;
        const DMedium& m = p.media[med];
        if (m.has_scattering) {
            b.med = med;
            b.o = ro + rd * dmin;
            b.length = fminf(dmax - dmin, m.max_beam_length);
            b.origin_offset = dmin;
            b.for_pdf = fpdf;
            b.rev_pdf = rpdf;
            b.flags = kEndInMedium | (i == 0 ? sflags : 0u);
            b.thr = thr;
            const unsigned idx = atomicAdd(&p.counters[3], 1u);
            if (idx < p.beam_capacity)
                store_beam(p.beams + idx, b);
            else
                flag_status(kErrBeamCapacity);
        }
        if (short_beams) {
            thr *= segs[i].att / segs[i].pdf_for;
            fpdf *= segs[i].pdf_for;
            rpdf *= segs[i].pdf_rev;
        } else {
            thr *= attenuation(m, dmax - dmin);
            float sr;
            const float sf = distance_pdf(m, dmin, dmax, i == 0 ? sflags : 0u, sr);
            fpdf *= sf;
            rpdf *= sr;
        }
    }
}

// Light tracing splat to the image plane (functs_light.cuh:251-388, Eq D.38).
UPBP_D unsigned connect_to_camera(const PathState& s, float3 hit, const Bsdf& bsdf, Rng& rng, VolSeg* segs,
                                  unsigned path_idx)
{
    const DeviceParams& p = c_params;
    const DCamera& cam = p.camera;
    float3 to_cam = cam.origin - hit;
    if (dot(cam.direction, -to_cam) <= 0.f) return 0;
    const float2 ip = world_to_raster(cam, hit);
    if (!raster_inside(cam, ip)) return 0;
    const float d2 = dot(to_cam, to_cam);
    const float dist = sqrtf(d2);
    to_cam /= dist;
    float cos_to_cam, fpdf, rpdf, sin_theta;
    const float3 f = bsdf_eval(bsdf, to_cam, cos_to_cam, &fpdf, &rpdf, &sin_theta);
    if (is_black_or_negative(f)) return 0;
    rpdf *= bsdf.cont_prob;
    const float cos_at_cam = dot(cam.direction, -to_cam);
    const float ip_dist = cam.image_plane_dist / cos_at_cam;
    const float i2sa = ip_dist * ip_dist / cos_at_cam;
    const float i2s = i2sa * fabsf(cos_to_cam) / (dist * dist);
    const float camera_pdf_a = i2s;
    int nseg = 0;
    bool occ;
    const unsigned st = occluded(occ, hit, to_cam, dist, s.stack, bsdf.in_medium() ? kOriginInMedium : 0u, segs, nseg, rng);
    if (st) return st;
    if (occ) return 0;
    float rs_rev = 1.f;
    float3 att = v3(1.f);
    if (nseg > 0) {
        rs_rev = seg_rev_pdf(segs, nseg);
        att = seg_attenuation(segs, nseg);
        if (!is_positive(att)) return 0;
    }
    const VertexWeights& wl = s.sw.w;
    const float f_s = pde_factor(bsdf.in_medium(), false, wl.for_inv, wl.for_ratio, 1.f / rs_rev, wl.rev_ratio, sin_theta);
    const float bpt_s_sub_1 = !wl.prev_specular;
    const float w_light = (camera_pdf_a / p.light_subpath_count) * rs_rev *
                          (f_s + bpt_s_sub_1 * wl.d_shared + (rpdf / wl.rev_inv) * wl.d_bpt);
    const float mis = 1.f / (w_light + 1.f);
    UPBP_MISDBG({
        MisEvent e{kMisLightTrace, 0u, 0u, path_idx, s.path_length, 0u, mis, hit, cam.origin, 0.f, 0.f};
        mis_event(e, segs, nseg);
    });
    const float s2i = 1.f / i2s;
    const float3 contrib = mis * s.throughput * f * att / (p.light_subpath_count * s2i);
    if (is_black_or_negative(contrib)) return 0;
    if (ip.x < 0.f || ip.x >= (float)p.res_x || ip.y < 0.f || ip.y >= (float)p.res_y) return 0;
    const unsigned px = (unsigned)int(ip.x) + (unsigned)int(ip.y) * p.res_x;
    atomicAdd(&p.framebuffer[3 * px + 0], contrib.x);
    atomicAdd(&p.framebuffer[3 * px + 1], contrib.y);
    atomicAdd(&p.framebuffer[3 * px + 2], contrib.z);
    return 0;
}

// State of one light subpath between bounces.
struct LightLane {
    PathState s;
    Rng rng;
    LightVertexRec* my_slots;
    unsigned path_idx, stored, ret;
    bool store_beams, origin_in_medium;
};

// Starts light subpath path_idx; false if it ended already.
UPBP_D bool light_path_begin(LightLane& l, unsigned path_idx)
{
    const DeviceParams& p = c_params;
    l.rng.init(p.iteration + p.iteration_offset, path_idx, 0u);
    l.path_idx = path_idx;
    l.store_beams = (p.do_bb1d && path_idx < p.bb1d_used_light_subpath_count) || p.do_bp2d;
    l.stored = 0;
    l.my_slots = p.vertices + (size_t)path_idx * p.slots_per_path;
    l.origin_in_medium = false;
    if (p.light_count == 0) {
        // A scene without lights (an emitting medium only): no light subpaths.
        // The reference samples lights[0] of its empty light array here
        // (functs_light.cuh:93).
        l.ret = 0;
        return false;
    }
    l.ret = generate_light_sample(l.s, l.rng, path_idx);
    if (l.s.is_infinite_light && p.media[p.global_medium].has_attenuation) {
        // the reference ends such a path before tracing it, without an error
        l.ret = 0;
        return false;
    }
    return l.ret == 0;
}

// One bounce of a light subpath (one iteration of the path loop of
// __raygen__trace_light, trace_light.cu:84-320); false when the path ends.
UPBP_D bool light_path_bounce(LightLane& l, VolSeg* segs, LiteSeg* lsegs)
{
    const DeviceParams& p = c_params;
    PathState& s = l.s;
    Rng& rng = l.rng;
    const unsigned path_idx = l.path_idx;
    const bool store_beams = l.store_beams;
    unsigned& stored = l.stored;
    LightVertexRec* my_slots = l.my_slots;
    bool& origin_in_medium = l.origin_in_medium;
    unsigned& ret = l.ret;
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
    UPBP_MISDBG(mis_ray(true, path_idx, s.path_length, rd, hit ? isect.dist : kInfinity,
                        origin_in_medium ? kOriginInMedium : 0u, lsegs, nlseg));
    if (store_beams)
        add_beams(ro, rd, s.throughput, s.path_length, origin_in_medium ? kOriginInMedium : 0u, segs, nseg, lsegs,
                  nlseg, path_idx, s);
    if (!hit) return false;

    float rs_for = 1.f, rs_rev = 1.f;
    if (nseg > 0) {
        rs_for = seg_for_pdf(segs, nseg);
        rs_rev = seg_rev_pdf(segs, nseg);
        s.throughput *= seg_attenuation(segs, nseg) / rs_for;
    }
    if (is_black_or_negative(s.throughput)) return false;

    VertexWeights& w = s.sw.w;
    if (s.path_length > 1u) {
        const float f_i = pde_factor(w.prev_in_medium, w.prev_specular, w.for_inv, w.for_ratio, 1.f / rs_rev,
                                     w.rev_ratio, s.sw.last_sin_theta);
        w.d_bpt = s.sw.d_bpt_a * f_i + s.sw.d_bpt_b;
        w.d_pde = s.sw.d_pde_a * f_i + s.sw.d_pde_b;
    }
    w.d_shared /= rs_for;
    w.d_bpt /= rs_for;
    w.d_pde /= rs_for;

    Bsdf bsdf;
    float3 frame_src;
    if (isect.on_surface()) {
        frame_src = isect.shading_normal;
        bsdf_setup_surface(bsdf, rd, isect.normal, isect.shading_normal, isect.mat, true, relative_ior(isect, s.stack));
    } else {
        frame_src = rd;
        bsdf_setup_medium(bsdf, rd, isect.med, true, ro + rd * isect.dist);
    }
    if (!bsdf.valid()) return false;
    float ratio = 0.f;
    if (bsdf.in_medium()) ratio = 1.f / p.media[bsdf.id].min_pos_att;
    const float3 hitpoint = ro + rd * isect.dist;
    origin_in_medium = isect.in_medium();
    UPBP_MISDBG(mis_hit(true, path_idx, s.path_length, hitpoint, isect.in_medium(),
                        isect.in_medium() ? isect.med : isect.mat, isect.in_medium() ? v3(0.f) : isect.shading_normal,
                        isect.in_medium() ? v3(0.f) : isect.normal, bsdf.delta(), bsdf.cont_prob));
    {
        const float d = bsdf.d_factor();
        if (!(s.path_length == 1 && s.is_infinite_light)) w.d_shared *= isect.dist * isect.dist;
        w.d_shared /= d;
        w.d_bpt /= d;
        w.d_pde /= d;
        w.for_inv = 1.f / rs_for;
        w.rev_inv = 1.f / rs_rev;
        w.for_ratio = ratio;
        w.rev_ratio = ratio;
    }
    if (!bsdf.delta()) {
        bool behind = false;
        if (origin_in_medium && s.stack.size > 0) {
            const int mid = s.stack.top().mat;
            if (mid >= 0 && p.materials[mid].real) behind = true;
        }
        if (stored < p.slots_per_path) {
            const unsigned slot = path_idx * p.slots_per_path + stored;
            store_vertex(my_slots + stored, hitpoint, s.throughput, s.path_length, origin_in_medium, behind, bsdf,
                         frame_src, w);
            stored++;
            atomicAdd(&p.counters[0], 1u);
            if (origin_in_medium) {
                const unsigned k = atomicAdd(&p.counters[2], 1u);
                p.idx_medium[k] = slot;
            } else {
                const unsigned k = atomicAdd(&p.counters[1], 1u);
                p.idx_surface[k] = slot;
            }
        }
    }
    if (p.guide_collect && bsdf.in_medium()) {
        // a training record of the learned proposal: where light arrives in
        // the medium, from which direction, with how much throughput
        const unsigned k = warp_reserve1(p.guide_rec_count);
        if (k < p.guide_rec_capacity)
            p.guide_recs[k] = GuideRecord{make_float4(hitpoint.x, hitpoint.y, hitpoint.z, ubits((unsigned)bsdf.id)),
                                          make_float4(rd.x, rd.y, rd.z, luminance(s.throughput))};
    }
    if (p.do_bpt && !bsdf.delta() && (bsdf.in_medium() || p.connect_to_camera_from_surf)) {
        if (s.path_length + 1 >= p.min_path_length) {
            ret = connect_to_camera(s, hitpoint, bsdf, rng, segs, path_idx);
            if (ret) return false;
        }
    }
    if (s.path_length + 2 > p.max_path_length) return false;
    bool cont;
    ret = sample_scattering(cont, bsdf, hitpoint, isect, s, rng);
    if (ret || !cont) return false;
    UPBP_MISDBG(if (s.sw.w.prev_specular) mis_specular(true, path_idx, s.path_length));
    s.path_length++;
    return true;
}

// Ends a light subpath: its status and its stored-vertex count.
UPBP_D void light_path_end(const LightLane& l)
{
    if (l.ret) flag_status(l.ret);
    c_params.path_vertex_count[l.path_idx] = l.stored;
}

// Light pass: persistent warps, one light subpath per lane; a lane whose
// path ended takes the next path index from a global counter (counters[4]),
// as the camera pass does with pixels.  Each path's random stream and
// vertex slots depend on its index alone.
__global__ void __launch_bounds__(128, 8) light_pass_kernel(int slot)
{
    begin_kernel(kKernLight, slot);
    const DeviceParams& p = c_params;
    VolSeg segs[kMaxVolSegments];
    LiteSeg lsegs[kMaxVolSegments];
    LightLane l;
    const unsigned lane = threadIdx.x & 31;
    const unsigned n = p.light_subpath_count;
    bool active = false, exhausted = false;
    for (;;) {
        const unsigned want = __ballot_sync(~0u, !active && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned base = 0;
            if ((int)lane == leader) base = atomicAdd(&p.counters[4], (unsigned)__popc(want));
            base = __shfl_sync(~0u, base, leader);
            if (!active && !exhausted) {
                const unsigned j = base + __popc(want & ((1u << lane) - 1u));
                if (j < n) {
                    active = light_path_begin(l, j);
                    if (!active) light_path_end(l);
                } else {
                    exhausted = true;
                }
            }
        }
        if (__all_sync(~0u, exhausted && !active)) break;
        if (active && !light_path_bounce(l, segs, lsegs)) {
            light_path_end(l);
            active = false;
        }
    }
}

}  // namespace upbp
