// Oracle translation unit 1: the reference's own OptiX device programs
// (gpuupbp/kernel/*.cu), compiled in place as host C++, plus
//   * an emulation of the OptiX device API they call (optixTrace over scalar
//     CPU BVHs, payload/attribute/SBT intrinsics), and
//   * a restatement of the reference's host-side iteration loop
//     (Renderer::init, gpuupbp/renderer/renderer_init.cpp:675-929, and
//     Renderer::run_iteration, gpuupbp/renderer/renderer.cpp:37-418) that
//     replaces the accel-structure builds with CPU BVHs and the two optixLaunch
//     calls with std::thread loops over the launch index.
// The result, oracle/_ref/libupbp_ref_cpu.so, is the reference renderer
// running on host cores.  It is the parity oracle for the B200 path and the
// timed CPU baseline.  Test infrastructure only: nothing in the product links it.
#include "kernel/trace_light.cu"
#include "kernel/trace_camera.cu"
#include "kernel/intersector.cu"
#include "kernel/pde/program_bb1d.cu"
#include "kernel/pde/program_bp2d.cu"
#include "kernel/pde/program_pb2d.cu"
#include "kernel/pde/program_pp3d.cu"
#include "kernel/pde/program_surf.cu"

#include "ref_bvh.h"
#include "ref_setup.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

////////////////////////////////////////////////////////////////////////////////
// RNG pass selection (read by the curand stand-in)

thread_local int g_oracle_rng_pass = 0;
unsigned long long g_oracle_rng_paths_per_iter = 0;

////////////////////////////////////////////////////////////////////////////////
// OptiX emulation

namespace {

enum : unsigned long long { kHandleScene = 1, kHandlePoints = 2, kHandleBeams = 3, kHandleCylinder = 4 };

struct Geometry {
    OracleBvh bvh_real;  // real triangles then real spheres
    OracleBvh bvh_imag;  // imaginary triangles then imaginary spheres
    unsigned int n_real_tri = 0, n_imag_tri = 0;
    std::vector<HitgroupData> sbt;  // one per record
    OracleBvh bvh_surface, bvh_medium, bvh_beams;
    unsigned int beam_count = 0;
};

Geometry g_geo;

struct TraceState {
    float3 o, d;
    float tmin, tmax;
    unsigned int* p0;
    unsigned int* p1;
    unsigned int prim, inst;
    bool tri;
    float2 bary;
    unsigned int attr[3];
    const HitgroupData* sbt;
    float ah_t;        // hit distance seen by an any-hit program
    bool in_anyhit;
    bool terminated;
    bool ignored;
    int mode;          // 0: closest-hit search, 1: any-hit collection, 2: IS only
    // closest-hit candidate found so far
    bool have_best;
    unsigned int best_prim;
    bool best_tri;
    float best_t;
    float2 best_bary;
    unsigned int best_attr[3];
};

thread_local TraceState ts;
thread_local uint3 g_launch_index;

std::atomic<unsigned long long> g_exceptions[8];

inline bool tri_hit(const float4* v, unsigned int prim, const float3& o, const float3& d, float& t, float2& bary)
{
    // Moller-Trumbore, double sided
    const float3 v0 = make_float3(v[3 * prim].x, v[3 * prim].y, v[3 * prim].z);
    const float3 v1 = make_float3(v[3 * prim + 1].x, v[3 * prim + 1].y, v[3 * prim + 1].z);
    const float3 v2 = make_float3(v[3 * prim + 2].x, v[3 * prim + 2].y, v[3 * prim + 2].z);
    const float3 e1 = v1 - v0, e2 = v2 - v0;
    const float3 p = cross(d, e2);
    const float det = dot(e1, p);
    if (det == 0.f) return false;
    const float inv = 1.f / det;
    const float3 s = o - v0;
    const float u = dot(s, p) * inv;
    if (u < 0.f || u > 1.f) return false;
    const float3 q = cross(s, e1);
    const float w = dot(d, q) * inv;
    if (w < 0.f || u + w > 1.f) return false;
    t = dot(e2, q) * inv;
    bary = make_float2(u, w);
    return true;
}

inline OracleBox box_of_tri(const float4* v, unsigned int i)
{
    OracleBox b;
    for (int a = 0; a < 3; a++) {
        float c0 = (&v[3 * i].x)[a], c1 = (&v[3 * i + 1].x)[a], c2 = (&v[3 * i + 2].x)[a];
        b.lo[a] = std::min(c0, std::min(c1, c2));
        b.hi[a] = std::max(c0, std::max(c1, c2));
    }
    return b;
}

inline OracleBox box_of_aabb(const OptixAabb& a)
{
    OracleBox b;
    b.lo[0] = a.minX;
    b.lo[1] = a.minY;
    b.lo[2] = a.minZ;
    b.hi[0] = a.maxX;
    b.hi[1] = a.maxY;
    b.hi[2] = a.maxZ;
    return b;
}

void trace_scene_real()
{
    const Scene& sc = params.scene;
    const float o[3] = {ts.o.x, ts.o.y, ts.o.z}, d[3] = {ts.d.x, ts.d.y, ts.d.z};
    ts.have_best = false;
    ts.mode = 0;
    float tmax = ts.tmax;
    g_geo.bvh_real.traverse(o, d, ts.tmin, tmax, [&](uint32_t p, float& tm) {
        if (p < g_geo.n_real_tri) {
            float t;
            float2 b;
            if (tri_hit(sc.triangles_real.verts, p, ts.o, ts.d, t, b) && t >= ts.tmin && t <= tm) {
                tm = t;
                ts.have_best = true;
                ts.best_prim = p;
                ts.best_tri = true;
                ts.best_t = t;
                ts.best_bary = b;
            }
        } else {
            ts.prim = p - g_geo.n_real_tri;
            ts.tmax = tm;
            __intersection__sphere_real();
            tm = ts.tmax;
        }
        return true;
    });
    if (!ts.have_best) return;
    ts.prim = ts.best_prim;
    ts.tri = ts.best_tri;
    ts.tmax = ts.best_t;
    ts.bary = ts.best_bary;
    for (int i = 0; i < 3; i++) ts.attr[i] = ts.best_attr[i];
    unsigned int rec = ts.tri ? sc.triangles_real.records[ts.prim] : sc.spheres_real.records[ts.prim];
    ts.sbt = &g_geo.sbt[rec];
    __closesthit__closest();
}

void trace_scene_imag()
{
    const Scene& sc = params.scene;
    const float o[3] = {ts.o.x, ts.o.y, ts.o.z}, d[3] = {ts.d.x, ts.d.y, ts.d.z};
    ts.mode = 1;
    ts.terminated = false;
    float tmax = ts.tmax;
    g_geo.bvh_imag.traverse(o, d, ts.tmin, tmax, [&](uint32_t p, float&) {
        if (p < g_geo.n_imag_tri) {
            float t;
            float2 b;
            if (tri_hit(sc.triangles_imag.verts, p, ts.o, ts.d, t, b) && t >= ts.tmin && t <= ts.tmax) {
                ts.prim = p;
                ts.tri = true;
                ts.bary = b;
                ts.ah_t = t;
                ts.in_anyhit = true;
                ts.sbt = &g_geo.sbt[sc.triangles_imag.records[p]];
                __anyhit__all();
                ts.in_anyhit = false;
            }
        } else {
            ts.prim = p - g_geo.n_imag_tri;
            __intersection__sphere_imag();
        }
        return !ts.terminated;
    });
}

void trace_points(unsigned int mask, unsigned int sbt_offset)
{
    const float o[3] = {ts.o.x, ts.o.y, ts.o.z}, d[3] = {ts.d.x, ts.d.y, ts.d.z};
    ts.mode = 2;
    float tmax = ts.tmax;
    auto run = [&](const OracleBvh& bvh, void (*prog)()) {
        bvh.traverse(o, d, ts.tmin, tmax, [&](uint32_t p, float&) {
            ts.prim = p;
            prog();
            return true;
        });
    };
    if ((mask & GEOM_MASK_PP2D) && sbt_offset == RAY_TYPE2_PP2D) run(g_geo.bvh_surface, __intersection__surf);
    if (mask & GEOM_MASK_POINT_MEDIUM) {
        if (sbt_offset == RAY_TYPE2_PP3D) run(g_geo.bvh_medium, __intersection__pp3d);
        if (sbt_offset == RAY_TYPE2_PB2D) run(g_geo.bvh_medium, __intersection__pb2d);
    }
}

void trace_beams(unsigned int mask, unsigned int sbt_offset)
{
    const float o[3] = {ts.o.x, ts.o.y, ts.o.z}, d[3] = {ts.d.x, ts.d.y, ts.d.z};
    ts.mode = 2;
    float tmax = ts.tmax;
    g_geo.bvh_beams.traverse(o, d, ts.tmin, tmax, [&](uint32_t b, float&) {
        if ((params.instances_beam[b].visibilityMask & mask) == 0) return true;
        ts.inst = b;
        ts.prim = 0;
        if (sbt_offset == RAY_TYPE2_BB1D) __intersection__bb1d();
        if (sbt_offset == RAY_TYPE2_BP2D) __intersection__bp2d();
        return true;
    });
}

}  // namespace

uint3 optixGetLaunchIndex() { return g_launch_index; }

void optixTrace(OptixTraversableHandle handle,
                float3 ray_origin,
                float3 ray_direction,
                float tmin,
                float tmax,
                float,
                unsigned int visibility_mask,
                unsigned int,
                unsigned int sbt_offset,
                unsigned int,
                unsigned int,
                unsigned int& p0,
                unsigned int& p1)
{
    TraceState saved = ts;
    ts.o = ray_origin;
    ts.d = ray_direction;
    ts.tmin = tmin;
    ts.tmax = tmax;
    ts.p0 = &p0;
    ts.p1 = &p1;
    ts.terminated = false;
    ts.in_anyhit = false;
    if (handle == kHandleScene) {
        if (sbt_offset == RAY_TYPE_SCENE_REAL)
            trace_scene_real();
        else
            trace_scene_imag();
    } else if (handle == kHandlePoints) {
        trace_points(visibility_mask, sbt_offset);
    } else if (handle == kHandleBeams) {
        trace_beams(visibility_mask, sbt_offset);
    }
    ts = saved;
}

unsigned int optixGetPayload_0() { return *ts.p0; }
unsigned int optixGetPayload_1() { return *ts.p1; }
void optixSetPayload_0(unsigned int v) { *ts.p0 = v; }
void optixSetPayload_1(unsigned int v) { *ts.p1 = v; }
void optixTerminateRay() { ts.terminated = true; }
void optixIgnoreIntersection() { ts.ignored = true; }
float3 optixGetWorldRayOrigin() { return ts.o; }
float3 optixGetWorldRayDirection() { return ts.d; }
float optixGetRayTmin() { return ts.tmin; }
float optixGetRayTmax() { return ts.in_anyhit ? ts.ah_t : ts.tmax; }
unsigned int optixGetPrimitiveIndex() { return ts.prim; }
unsigned int optixGetInstanceIndex() { return ts.inst; }
bool optixIsTriangleHit() { return ts.tri; }
float2 optixGetTriangleBarycentrics() { return ts.bary; }
unsigned int optixGetAttribute_0() { return ts.attr[0]; }
unsigned int optixGetAttribute_1() { return ts.attr[1]; }
unsigned int optixGetAttribute_2() { return ts.attr[2]; }
void* optixGetSbtDataPointer() { return (void*)ts.sbt; }
int optixGetExceptionCode() { return 0; }

void optixThrowException(int code)
{
    // exceptions are disabled in the reference unless -assert is given; count them
    g_exceptions[(code >= 0 && code < 8) ? code : 7]++;
}

bool optixReportIntersection(float t, unsigned int, unsigned int a0, unsigned int a1, unsigned int a2)
{
    if (!(t >= ts.tmin && t <= ts.tmax)) return false;
    if (ts.mode == 0) {  // closest-hit search over real spheres: accept and shrink
        ts.have_best = true;
        ts.best_prim = ts.prim;
        ts.best_tri = false;
        ts.best_t = t;
        ts.best_attr[0] = a0;
        ts.best_attr[1] = a1;
        ts.best_attr[2] = a2;
        ts.tmax = t;
        return true;
    }
    if (ts.mode == 1) {  // imaginary spheres: run the any-hit program
        ts.tri = false;
        ts.attr[0] = a0;
        ts.attr[1] = a1;
        ts.attr[2] = a2;
        ts.ah_t = t;
        ts.ignored = false;
        ts.in_anyhit = true;
        ts.sbt = &g_geo.sbt[params.scene.spheres_imag.records[ts.prim]];
        __anyhit__all();
        ts.in_anyhit = false;
        return !ts.ignored && !ts.terminated;
    }
    return false;
}

////////////////////////////////////////////////////////////////////////////////
// Host iteration loop (restated from the reference's Renderer)

struct RefCtx {
    OracleSetup setup;
    float bb1d_r0, bp2d_r0, pb2d_r0, pp3d_r0, surf_r0;
    unsigned int light_subpath_count, screen_pixel_count;
    float bb1d_used;
    bool build_bb1d, build_bp2d, build_pb2d, build_pp3d, build_surf;
    std::vector<LightVertex> verts;
    std::vector<OptixAabb> aabb_surface, aabb_medium;
    std::vector<unsigned int> idx_surface, idx_medium;
    std::vector<LightBeam> beams;
    std::vector<OptixInstance> instances;
    std::vector<unsigned int> starts;
    unsigned int counters[4];
    std::vector<float3> fb;
    int threads;
    double t_light, t_build, t_camera;
    unsigned int last_vertices, last_surface, last_medium, last_beams;
};

static void run_parallel(unsigned int n, int threads, int pass, void (*prog)())
{
    std::atomic<unsigned int> next{0};
    auto worker = [&]() {
        g_oracle_rng_pass = pass;
        const unsigned int chunk = 64;
        for (;;) {
            unsigned int b = next.fetch_add(chunk);
            if (b >= n) break;
            unsigned int e = std::min(n, b + chunk);
            for (unsigned int i = b; i < e; i++) {
                g_launch_index = make_uint3(i, 0, 0);
                prog();
            }
        }
    };
    if (threads <= 1) {
        worker();
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
}

static float relative_radius(float r, float scene_radius) { return r < 0.f ? -r * scene_radius : r; }

extern "C" {

// Creates the oracle from the reference's own command line.  Only one context
// may exist at a time (the reference keeps its launch parameters in a global).
int upbp_ref_create(int argc, const char** argv, int threads, RefCtx** out)
{
    RefCtx* c = new RefCtx{};
    int rc = oracle_parse_and_load(argc, argv, &c->setup);
    if (rc != 0) {
        delete c;
        return rc;
    }
    c->threads = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    const OracleSetup& s = c->setup;
    const float scene_radius = s.scene.scene_sphere.radius;
    c->bb1d_r0 = relative_radius(s.bb1d_radius_initial, scene_radius);
    c->bp2d_r0 = relative_radius(s.bp2d_radius_initial, scene_radius);
    c->pb2d_r0 = relative_radius(s.pb2d_radius_initial, scene_radius);
    c->pp3d_r0 = relative_radius(s.pp3d_radius_initial, scene_radius);
    c->surf_r0 = relative_radius(s.surf_radius_initial, scene_radius);

    LaunchParams& p = params;
    p = LaunchParams{};
    const unsigned int flags = s.algorithm_flags;
    p.trace_light_paths = flags != 0;
    p.trace_camera_paths = flags != 0;
    p.do_bpt = flags & BPT;
    p.do_bb1d = flags & BB1D;
    p.do_bp2d = flags & BP2D;
    p.do_pb2d = flags & PB2D;
    p.do_pp3d = flags & PP3D;
    p.do_surf = flags & SURF;
    if (flags & SPECULAR_ONLY) {
        p.trace_light_paths = false;
        p.trace_camera_paths = true;
        p.do_bpt = p.do_bb1d = p.do_bp2d = p.do_pb2d = p.do_pp3d = p.do_surf = false;
    }
    p.connect_to_camera_from_surf = (flags & (PREVIOUS | COMPATIBLE)) == 0;
    c->screen_pixel_count = s.res_x * s.res_y;
    c->light_subpath_count = (unsigned int)s.path_count_per_iter;
    c->bb1d_used = s.bb1d_used_light_subpath_count;
    if (c->bb1d_used < 0.f) c->bb1d_used = std::floor(-c->bb1d_used * (float)c->light_subpath_count);
    p.scene = s.scene;

    // scene geometry: BVHs and hit-group records
    const Scene& sc = s.scene;
    g_geo = Geometry{};
    g_geo.sbt.resize(s.record_count);
    for (unsigned int i = 0; i < s.record_count; i++) g_geo.sbt[i].gpu_mat = s.records[i];
    {
        std::vector<OracleBox> boxes;
        for (unsigned int i = 0; i < sc.triangles_real.count; i++) boxes.push_back(box_of_tri(sc.triangles_real.verts, i));
        for (unsigned int i = 0; i < sc.spheres_real.count; i++) boxes.push_back(box_of_aabb(sc.spheres_real.aabbs[i]));
        g_geo.n_real_tri = sc.triangles_real.count;
        g_geo.bvh_real.build(boxes);
        boxes.clear();
        for (unsigned int i = 0; i < sc.triangles_imag.count; i++) boxes.push_back(box_of_tri(sc.triangles_imag.verts, i));
        for (unsigned int i = 0; i < sc.spheres_imag.count; i++) boxes.push_back(box_of_aabb(sc.spheres_imag.aabbs[i]));
        g_geo.n_imag_tri = sc.triangles_imag.count;
        g_geo.bvh_imag.build(boxes);
    }

    const unsigned int L = c->light_subpath_count;
    const unsigned int max_verts_per_path = s.max_path_length - 1;
    const unsigned int max_beams_per_path = (max_verts_per_path - 1) * 1u;
    const unsigned int vertex_max = L * max_verts_per_path;
    unsigned int beam_paths = 0;
    if (p.do_bb1d) beam_paths = std::max(beam_paths, (unsigned int)c->bb1d_used);
    if (p.do_bp2d) beam_paths = std::max(beam_paths, L);
    const unsigned int beam_max = beam_paths * max_beams_per_path;
    c->verts.resize(std::max(1u, vertex_max));
    c->aabb_surface.resize(std::max(1u, vertex_max));
    c->aabb_medium.resize(std::max(1u, vertex_max));
    c->idx_surface.resize(std::max(1u, vertex_max));
    c->idx_medium.resize(std::max(1u, vertex_max));
    c->beams.resize(std::max(1u, beam_max));
    c->instances.resize(std::max(1u, beam_max));
    c->starts.resize(std::max(1u, L));
    c->fb.resize(c->screen_pixel_count);
    p.light_vertex_count = vertex_max;
    p.light_beam_count = beam_max;
    p.light_vertices = c->verts.data();
    p.aabb_surface = c->aabb_surface.data();
    p.aabb_medium = c->aabb_medium.data();
    p.indices_surface = c->idx_surface.data();
    p.indices_medium = c->idx_medium.data();
    p.light_beams = c->beams.data();
    p.instances_beam = c->instances.data();
    p.light_subpath_starts = c->starts.data();
    p.light_vertex_counter = &c->counters[0];
    p.light_vertex_surface_counter = &c->counters[1];
    p.light_vertex_medium_counter = &c->counters[2];
    p.light_beam_counter = &c->counters[3];
    p.framebuffer.color = c->fb.data();
    p.framebuffer.resolution = make_uint2(s.res_x, s.res_y);

    const bool do_merging = s.max_path_length > 1;
    c->build_bb1d = p.trace_light_paths && do_merging && p.do_bb1d;
    c->build_bp2d = p.trace_light_paths && do_merging && p.do_bp2d;
    c->build_pb2d = p.trace_light_paths && do_merging && p.do_pb2d;
    c->build_pp3d = p.trace_light_paths && do_merging && p.do_pp3d;
    c->build_surf = p.trace_light_paths && do_merging && p.do_surf;

    p.rng_offset = s.iteration_offset * L;
    g_oracle_rng_paths_per_iter = L;
    p.min_path_length = s.min_path_length;
    p.max_path_length = s.max_path_length;
    p.photon_beam_type = (BeamType)s.photon_beam_type;
    p.camera_beam_type = (BeamType)s.query_beam_type;
    p.subpath_count_bpt = float(p.do_bpt);
    p.subpath_count_bb1d = float(p.do_bb1d) * c->bb1d_used;
    p.subpath_count_bp2d = float(p.do_bp2d) * L;
    p.subpath_count_pb2d = float(p.do_pb2d) * L;
    p.subpath_count_pp3d = float(p.do_pp3d) * L;
    p.subpath_count_surf = float(p.do_surf) * L;
    p.build_bb1d = c->build_bb1d;
    p.build_bp2d = c->build_bp2d;
    p.build_pb2d = c->build_pb2d;
    p.build_pp3d = c->build_pp3d;
    p.build_surf = c->build_surf;
    p.ignore_fully_spec_paths = s.ignore_fully_spec_paths;
    p.screen_pixel_count = c->screen_pixel_count;
    p.light_subpath_count = L;
    p.estimator_techniques = flags;
    p.bb1d_used_light_sub_path_count = (unsigned int)c->bb1d_used;
    p.use_shading_normal = s.use_shading_normal;
    p.handle_gas_beam = kHandleCylinder;
    p.sbt_offset = s.record_count * RAY_TYPE_COUNT;
    p.handle = kHandleScene;
    *out = c;
    return 0;
}

// One iteration of the reference's render loop; writes this iteration's
// framebuffer (W*H RGB float) to rgb (not accumulated).
int upbp_ref_run_iteration(RefCtx* c, int iteration, float* rgb)
{
    using clk = std::chrono::steady_clock;
    auto t0 = clk::now();
    LaunchParams& p = params;
    const OracleSetup& s = c->setup;
    std::fill(c->fb.begin(), c->fb.end(), make_float3(0.f));
    unsigned int found_v = 0, found_s = 0, found_m = 0, found_b = 0;
    const unsigned int L = c->light_subpath_count;
    if (p.trace_light_paths) {
        const float eff = 1.f + (float)iteration;
        float r_bb1d = c->bb1d_r0 * powf(1.f + (float)iteration * c->bb1d_used / (float)L, s.bb1d_radius_alpha - 1.f);
        r_bb1d = fmaxf(r_bb1d, 1e-7f);
        float r_bp2d = c->bp2d_r0 * powf(eff, (s.bp2d_radius_alpha - 1.f) * .5f);
        r_bp2d = fmaxf(r_bp2d, 1e-7f);
        float r_pb2d = c->pb2d_r0 * powf(eff, (s.pb2d_radius_alpha - 1.f) * .5f);
        r_pb2d = fmaxf(r_pb2d, 1e-7f);
        float r_pp3d = c->pp3d_r0 * powf(eff, (s.pp3d_radius_alpha - 1.f) * (1.f / 3.f));
        r_pp3d = fmaxf(r_pp3d, 1e-7f);
        float r_surf = c->surf_r0 * powf(eff, (s.surf_radius_alpha - 1.f) * .5f);
        r_surf = fmaxf(r_surf, 1e-7f);
        p.mis_factor_bb1d = .5f * r_bb1d * p.subpath_count_bb1d;
        p.mis_factor_bp2d = (PI_F * r_bp2d * r_bp2d) * p.subpath_count_bp2d;
        p.mis_factor_pb2d = (PI_F * r_pb2d * r_pb2d) * p.subpath_count_pb2d;
        p.mis_factor_pp3d = (4.f / 3.f) * (PI_F * r_pp3d * r_pp3d * r_pp3d) * p.subpath_count_pp3d;
        p.mis_factor_surf = (PI_F * r_surf * r_surf) * p.subpath_count_surf;
        p.bb1d_normalization = 1.f / c->bb1d_used;
        p.bp2d_normalization = 1.f / (float)L;
        p.pb2d_normalization = 1.f / (float)L;
        p.pp3d_normalization = 1.f / p.mis_factor_pp3d;
        p.surf_normalization = 1.f / p.mis_factor_surf;
        p.radius_bb1d = r_bb1d;
        p.radius_pb2d = r_pb2d;
        p.radius_surf = r_surf;
        p.radius_pp3d = r_pp3d;
        p.radius_bp2d = r_bp2d;
        p.rad_point_med = 0.f;
        if (p.do_pp3d) p.rad_point_med = std::max(p.rad_point_med, r_pp3d);
        if (p.do_pb2d) p.rad_point_med = std::max(p.rad_point_med, r_pb2d);
        p.rad_beam = 0.f;
        if (p.do_bb1d) p.rad_beam = std::max(p.rad_beam, r_bb1d);
        if (p.do_bp2d) p.rad_beam = std::max(p.rad_beam, r_bp2d);
        p.radius_bb1d_2 = r_bb1d * r_bb1d;
        p.radius_bp2d_2 = r_bp2d * r_bp2d;
        p.radius_pb2d_2 = r_pb2d * r_pb2d;
        p.radius_pp3d_2 = r_pp3d * r_pp3d;
        p.radius_surf_2 = r_surf * r_surf;
        p.iteration = iteration;
        c->counters[0] = c->counters[1] = c->counters[2] = c->counters[3] = 0;

        run_parallel(L, c->threads, 0, __raygen__trace_light);

        found_v = c->counters[0];
        found_s = c->counters[1];
        found_m = c->counters[2];
        found_b = c->counters[3];
        if (found_v > p.light_vertex_count) fprintf(stderr, "error: device finds more vertices than memory allocated");
        if (found_b > p.light_beam_count) fprintf(stderr, "error: device finds more beams than memory allocated");
    }
    auto t1 = clk::now();

    // photon maps: CPU BVHs over the same boxes OptiX would get
    const unsigned int nb = std::min(found_b, p.light_beam_count);
    const unsigned int nm = std::min(found_m, p.light_vertex_count);
    const unsigned int ns = std::min(found_s, p.light_vertex_count);
    {
        std::vector<OracleBox> boxes;
        if ((c->build_bb1d || c->build_bp2d) && nb > 0) {
            for (unsigned int i = 0; i < nb; i++) {
                const LightBeam& b = c->beams[i];
                const float3 a = b.ray.origin, e = b.ray.origin + b.ray.direction * b.beam_length;
                OracleBox bx;
                for (int k = 0; k < 3; k++) {
                    float ak = (&a.x)[k], ek = (&e.x)[k];
                    bx.lo[k] = std::min(ak, ek) - p.rad_beam;
                    bx.hi[k] = std::max(ak, ek) + p.rad_beam;
                }
                boxes.push_back(bx);
            }
            g_geo.bvh_beams.build(boxes);
            p.handle_beams = kHandleBeams;
        } else {
            g_geo.bvh_beams.build({});
            p.handle_beams = 0;
        }
        boxes.clear();
        for (unsigned int i = 0; i < (c->build_surf ? ns : 0u); i++) boxes.push_back(box_of_aabb(c->aabb_surface[i]));
        g_geo.bvh_surface.build(boxes);
        boxes.clear();
        for (unsigned int i = 0; i < ((c->build_pb2d || c->build_pp3d) ? nm : 0u); i++)
            boxes.push_back(box_of_aabb(c->aabb_medium[i]));
        g_geo.bvh_medium.build(boxes);
        p.handle_points = kHandlePoints;
    }
    auto t2 = clk::now();

    if (p.trace_camera_paths) run_parallel(c->screen_pixel_count, c->threads, 1, __raygen__trace_camera);
    auto t3 = clk::now();

    if (rgb) std::memcpy(rgb, c->fb.data(), sizeof(float) * 3 * c->screen_pixel_count);
    c->t_light = std::chrono::duration<double>(t1 - t0).count();
    c->t_build = std::chrono::duration<double>(t2 - t1).count();
    c->t_camera = std::chrono::duration<double>(t3 - t2).count();
    c->last_vertices = found_v;
    c->last_surface = found_s;
    c->last_medium = found_m;
    c->last_beams = found_b;
    return 0;
}

// Statistics of the last iteration: [vertices, surface, medium, beams,
// light paths, pixels, width, height] and [t_light, t_build, t_camera] seconds.
int upbp_ref_get_stats(RefCtx* c, unsigned int* u8, double* t3)
{
    if (u8) {
        u8[0] = c->last_vertices;
        u8[1] = c->last_surface;
        u8[2] = c->last_medium;
        u8[3] = c->last_beams;
        u8[4] = c->light_subpath_count;
        u8[5] = c->screen_pixel_count;
        u8[6] = c->setup.res_x;
        u8[7] = c->setup.res_y;
    }
    if (t3) {
        t3[0] = c->t_light;
        t3[1] = c->t_build;
        t3[2] = c->t_camera;
    }
    return 0;
}

// Counts of OptiX exceptions the reference's programs raised (code 0 is a
// failed GPU_ASSERT, 1-4 are capacity overflows).
void upbp_ref_exception_counts(unsigned long long* out8)
{
    for (int i = 0; i < 8; i++) out8[i] = g_exceptions[i].load();
}

const char* upbp_ref_output_name(RefCtx* c) { return c->setup.output_name; }

// JSON summary of the parsed configuration and the loaded scene, for the
// command-line and loader parity tests.
int upbp_ref_describe(RefCtx* c, char* buf, int cap)
{
    const OracleSetup& s = c->setup;
    const Scene& sc = s.scene;
    const Camera& cam = sc.camera;
    return snprintf(
        buf, (size_t)cap,
        "{\"algorithm_flags\": %u, \"iteration_count\": %d, \"res\": [%u, %u], \"max_path_length\": %u, "
        "\"min_path_length\": %u, \"path_count_per_iter\": %.9g, \"query_beam_type\": %d, "
        "\"photon_beam_type\": %d, \"radius_initial\": [%.9g, %.9g, %.9g, %.9g, %.9g], "
        "\"radius_alpha\": [%.9g, %.9g, %.9g, %.9g, %.9g], \"bb1d_used\": %.9g, \"ignore_spec\": %d, "
        "\"ioff\": %llu, \"shading_normal\": %d, \"output_name\": \"%s\", "
        "\"tri_real\": %u, \"tri_imag\": %u, \"lights\": %u, \"materials\": %u, \"media\": %u, "
        "\"global_medium\": %u, \"background\": %d, \"records\": %u, "
        "\"camera_origin\": [%.9g, %.9g, %.9g], \"camera_dir\": [%.9g, %.9g, %.9g], "
        "\"image_plane_dist\": %.9g, \"scene_center\": [%.9g, %.9g, %.9g], \"scene_radius\": %.9g}",
        s.algorithm_flags, s.iteration_count, s.res_x, s.res_y, s.max_path_length, s.min_path_length,
        s.path_count_per_iter, s.query_beam_type, s.photon_beam_type, s.surf_radius_initial, s.pp3d_radius_initial,
        s.pb2d_radius_initial, s.bb1d_radius_initial, s.bp2d_radius_initial, s.surf_radius_alpha, s.pp3d_radius_alpha,
        s.pb2d_radius_alpha, s.bb1d_radius_alpha, s.bp2d_radius_alpha, s.bb1d_used_light_subpath_count,
        (int)s.ignore_fully_spec_paths, (unsigned long long)s.iteration_offset, (int)s.use_shading_normal,
        s.output_name, sc.triangles_real.count, sc.triangles_imag.count, sc.light_count, sc.mat_count,
        sc.med_count, sc.global_medium_idx, sc.background_light_idx == UINT32_MAX ? -1 : (int)sc.background_light_idx,
        s.record_count, cam.origin.x, cam.origin.y, cam.origin.z, cam.direction.x, cam.direction.y,
        cam.direction.z, cam.image_plane_dist, sc.scene_sphere.center.x, sc.scene_sphere.center.y,
        sc.scene_sphere.center.z, sc.scene_sphere.radius);
}

// JSON dump of every record of the loaded scene (triangles with their face
// normals, sphere boxes, primitive records, materials, media, lights), for
// the loader parity tests.  Returns the length the dump needs; writes it when
// it fits in `cap` bytes.
int upbp_ref_scene_json(RefCtx* c, char* buf, int cap)
{
    const OracleSetup& s = c->setup;
    const Scene& sc = s.scene;
    std::string o = "{";
    auto num = [&](double v) {
        char t[40];
        snprintf(t, sizeof(t), "%.9g", v);
        o += t;
    };
    auto f3 = [&](float3 v) {
        o += "[";
        num(v.x);
        o += ",";
        num(v.y);
        o += ",";
        num(v.z);
        o += "]";
    };
    auto rec = [&](unsigned r) {
        o += "[";
        num(s.records[r].id_material);
        o += ",";
        num(s.records[r].id_light);
        o += "]";
    };
    auto tris = [&](const char* name, const Triangles& t) {
        o += std::string("\"") + name + "\": [";
        for (unsigned i = 0; i < t.count; i++) {
            if (i) o += ",";
            o += "[";
            for (int k = 0; k < 3; k++) {
                f3(make_float3(t.verts[3 * i + k].x, t.verts[3 * i + k].y, t.verts[3 * i + k].z));
                o += ",";
            }
            f3(t.norms[4 * i + 3]);
            o += ",";
            rec(t.records[i]);
            o += "]";
        }
        o += "], ";
    };
    auto sphs = [&](const char* name, const Spheres& t) {
        o += std::string("\"") + name + "\": [";
        for (unsigned i = 0; i < t.count; i++) {
            if (i) o += ",";
            const OptixAabb& b = t.aabbs[i];
            o += "[";
            f3(make_float3(b.minX, b.minY, b.minZ));
            o += ",";
            f3(make_float3(b.maxX, b.maxY, b.maxZ));
            o += ",";
            rec(t.records[i]);
            o += "]";
        }
        o += "], ";
    };
    tris("tri_real", sc.triangles_real);
    tris("tri_imag", sc.triangles_imag);
    sphs("sph_real", sc.spheres_real);
    sphs("sph_imag", sc.spheres_imag);
    o += "\"materials\": [";
    for (unsigned i = 0; i < sc.mat_count; i++) {
        const Material& m = sc.materials[i];
        if (i) o += ",";
        o += "[";
        f3(m.diffuse_reflectance);
        o += ",";
        f3(m.phong_reflectance);
        o += ",";
        num(m.phong_exponent);
        o += ",";
        f3(m.mirror_reflectance);
        o += ",";
        num(m.ior);
        o += ",";
        num(m.priority);
        o += ",";
        num(m.real ? 1 : 0);
        o += ",";
        num(m.med_idx);
        o += "]";
    }
    o += "], \"media\": [";
    for (unsigned i = 0; i < sc.med_count; i++) {
        const Medium& m = sc.media[i];
        if (i) o += ",";
        o += "[";
        f3(m.absorption_coeff);
        o += ",";
        f3(m.emission_coeff);
        o += ",";
        f3(m.scattering_coeff);
        o += ",";
        num(m.continuation_prob);
        o += ",";
        num(m.mean_cosine);
        o += "]";
    }
    // per light: type, material, medium, then (area) p0, e1, e2, intensity;
    // (background) colour, scale; (directional) frame z, intensity; (point)
    // position, intensity
    o += "], \"lights\": [";
    for (unsigned i = 0; i < sc.light_count; i++) {
        const AbstractLight& l = sc.lights[i];
        if (i) o += ",";
        o += "[";
        num((int)l.type);
        o += ",";
        num(l.mat_id);
        o += ",";
        num(l.med_id);
        o += ",";
        if (l.type == AREA) {
            f3(l.area.p0);
            o += ",";
            f3(l.area.e1);
            o += ",";
            f3(l.area.e2);
            o += ",";
            f3(l.area.intensity);
        } else if (l.type == BACKGROUND) {
            f3(l.background.background_color);
            o += ",";
            num(l.background.scale);
        } else if (l.type == DIRECTIONAL) {
            f3(l.directional.frame.z);
            o += ",";
            f3(l.directional.intensity);
        } else {
            f3(l.point.position);
            o += ",";
            f3(l.point.intensity);
        }
        o += "]";
    }
    o += "], \"global_medium\": ";
    num(sc.global_medium_idx);
    o += ", \"background\": ";
    num(sc.background_light_idx == UINT32_MAX ? -1 : (int)sc.background_light_idx);
    o += ", \"scene_center\": ";
    f3(sc.scene_sphere.center);
    o += ", \"scene_radius\": ";
    num(sc.scene_sphere.radius);
    if (sc.has_env_map) {  // the environment map image as the loader left it
        const Image& im = sc.env_map.img;
        o += ", \"env\": [";
        num(im.width);
        o += ",";
        num(im.height);
        o += ",[";
        for (int i = 0; i < im.width * im.height; i++) {
            if (i) o += ",";
            f3(im.data[i]);
        }
        o += "]]";
    }
    o += "}";
    if ((int)o.size() < cap) std::memcpy(buf, o.c_str(), o.size() + 1);
    return (int)o.size() + 1;
}

int upbp_ref_iteration_count(RefCtx* c) { return c->setup.iteration_count; }

void upbp_ref_destroy(RefCtx* c)
{
    if (!c) return;
    oracle_free_setup(&c->setup);
    g_geo = Geometry{};
    delete c;
}

}  // extern "C"
