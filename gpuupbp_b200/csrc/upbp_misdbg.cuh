// MIS recording for the FP64 full-path weight check (compiled into the
// separate library libupbp_b200_misdbg.so with -DUPBP_MIS_DEBUG; the
// production library contains none of it).
//
// For every light and camera subpath the recording build keeps each vertex
// with the media segments of the ray that reached it; for every contribution
// it keeps the technique, the FP32 MIS weight the renderer applied and the
// points where the two subpaths meet.  The FP64 oracle (oracle/mis_fp64.py)
// rebuilds each contribution's full path from these and evaluates the weight
// over all of its vertices and techniques.
#pragma once

#include "upbp_trace.cuh"

namespace upbp {

// Vertex record: kMisVtxWords float4 per vertex, slot path * max_verts + k
// (k = 0 the subpath's origin on the light or the camera, k >= 1 the vertex
// the k-th ray reached).
//   w0: position.xyz, flags bits (kMisValid | kMisMedium | kMisSpecular | kMisDelta | kMisLight | kMisCamera | kMisMiss)
//   w1: frame normal.xyz (shading normal; light normal at a light vertex), id bits (material / medium / light)
//   w2: geometric normal.xyz, segment count bits
//   w3: ray length to this vertex, trace flags bits (origin in medium), continuation probability, 0
//   w4: direction of that ray.xyz, 0
//   w5..: media segments of that ray (dmin, dmax, medium id bits, 0), up to kMisSegs, to the ray's real hit
constexpr int kMisSegs = 10;
constexpr int kMisVtxWords = 5 + kMisSegs;
enum : unsigned {
    kMisValid = 1u, kMisMedium = 2u, kMisSpecular = 4u, kMisDelta = 8u, kMisLight = 16u, kMisCamera = 32u,
    kMisMiss = 64u
};

// Contribution record: kMisEvWords float4.
//   e0: technique bits, weight, camera path bits, camera vertex index bits
//   e1: light path bits, light vertex index bits, light id bits (NEE), photon beam's origin offset from its vertex
//   e2: light-side point.xyz, distance along the photon beam from its vertex (beams)
//   e3: camera-side point.xyz, distance along the query ray from its vertex (query beams)
//   e4: connection-ray segment count bits, 0, 0, 0
//   e5..: segments of the connection ray (dmin, dmax, medium id bits, 0), traced from the camera-side end
//         (BPT, NEE) or from the light vertex (light tracing)
constexpr int kMisEvWords = 5 + kMisSegs;
enum : unsigned {
    kMisEmitterHit = 0u, kMisNee, kMisBpt, kMisLightTrace, kMisSurf, kMisPp3d, kMisPb2d, kMisBb1d, kMisBp2d
};

struct MisDebug {
    float4* light;          // light subpath vertices
    float4* camera;         // camera subpath vertices
    float4* events;         // contributions
    unsigned* event_count;
    unsigned event_capacity;
    unsigned max_verts;     // vertex slots per subpath
    unsigned light_paths, camera_paths;
};

#ifdef UPBP_MIS_DEBUG
__constant__ MisDebug c_misdbg;

UPBP_D float4* mis_vertex(bool light, unsigned path, unsigned k)
{
    const MisDebug& d = c_misdbg;
    if (k >= d.max_verts || path >= (light ? d.light_paths : d.camera_paths)) return nullptr;
    return (light ? d.light : d.camera) + ((size_t)path * d.max_verts + k) * kMisVtxWords;
}

// The origin of a subpath (light sample or camera).
UPBP_D void mis_origin(bool light, unsigned path, float3 pos, float3 n, unsigned id)
{
    float4* v = mis_vertex(light, path, 0);
    if (!v) return;
    v[0] = make_float4(pos.x, pos.y, pos.z, __uint_as_float(kMisValid | (light ? kMisLight : kMisCamera)));
    v[1] = make_float4(n.x, n.y, n.z, __uint_as_float(id));
    v[2] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
    v[3] = make_float4(0.f, 0.f, 1.f, 0.f);
}

// The ray that reaches vertex k: its media segments (up to the real hit) and
// its length to the vertex (the hit, a sampled scattering distance, or
// infinity for a miss).
UPBP_D void mis_ray(bool light, unsigned path, unsigned k, float3 dir, float dist, unsigned sflags,
                    const LiteSeg* lsegs, int nlseg)
{
    float4* v = mis_vertex(light, path, k);
    if (!v) return;
    const int n = min(nlseg, kMisSegs);
    v[0] = make_float4(0.f, 0.f, 0.f, __uint_as_float(kMisMiss));
    v[2] = make_float4(0.f, 0.f, 0.f, __uint_as_float((unsigned)n));
    v[3] = make_float4(dist, __uint_as_float(sflags), 1.f, 0.f);
    v[4] = make_float4(dir.x, dir.y, dir.z, 0.f);
    for (int i = 0; i < n; i++) v[5 + i] = make_float4(lsegs[i].dmin, lsegs[i].dmax, __uint_as_float((unsigned)lsegs[i].med), 0.f);
}

// The vertex the ray reached: position, frame, ids and its scattering function.
UPBP_D void mis_hit(bool light, unsigned path, unsigned k, float3 pos, bool in_medium, int id, float3 shading_n,
                    float3 geom_n, bool delta, float cont_prob)
{
    float4* v = mis_vertex(light, path, k);
    if (!v) return;
    unsigned f = kMisValid | (in_medium ? kMisMedium : 0u) | (delta ? kMisDelta : 0u);
    v[0] = make_float4(pos.x, pos.y, pos.z, __uint_as_float(f));
    v[1] = make_float4(shading_n.x, shading_n.y, shading_n.z, __uint_as_float((unsigned)id));
    v[2] = make_float4(geom_n.x, geom_n.y, geom_n.z, v[2].w);
    v[3].z = cont_prob;
}

// An emitter the ray reached (an emitter hit of a camera path).
UPBP_D void mis_hit_light(unsigned path, unsigned k, float3 pos, int light, float3 n)
{
    float4* v = mis_vertex(false, path, k);
    if (!v) return;
    v[0] = make_float4(pos.x, pos.y, pos.z, __uint_as_float(kMisValid | kMisLight));
    v[1] = make_float4(n.x, n.y, n.z, __uint_as_float((unsigned)light));
}

// Vertex k sampled a specular event (no connection or merge through it).
UPBP_D void mis_specular(bool light, unsigned path, unsigned k)
{
    float4* v = mis_vertex(light, path, k);
    if (v) v[0].w = __uint_as_float(__float_as_uint(v[0].w) | kMisSpecular);
}

struct MisEvent {
    unsigned tech, cam_path, cam_k, light_path, light_k, light_id;
    float weight;
    float3 pl, pc;
    float tl, tc;
    float offset;
};

UPBP_D void mis_event(const MisEvent& e, const VolSeg* segs, int nseg)
{
    const MisDebug& d = c_misdbg;
    const unsigned i = atomicAdd(d.event_count, 1u);
    if (i >= d.event_capacity) return;
    float4* r = d.events + (size_t)i * kMisEvWords;
    const int n = min(nseg, kMisSegs);
    r[0] = make_float4(__uint_as_float(e.tech), e.weight, __uint_as_float(e.cam_path), __uint_as_float(e.cam_k));
    r[1] = make_float4(__uint_as_float(e.light_path), __uint_as_float(e.light_k), __uint_as_float(e.light_id), e.offset);
    r[2] = make_float4(e.pl.x, e.pl.y, e.pl.z, e.tl);
    r[3] = make_float4(e.pc.x, e.pc.y, e.pc.z, e.tc);
    r[4] = make_float4(__uint_as_float((unsigned)n), 0.f, 0.f, 0.f);
    for (int j = 0; j < n; j++) r[5 + j] = make_float4(segs[j].dmin, segs[j].dmax, __uint_as_float((unsigned)segs[j].med), 0.f);
}
#define UPBP_MISDBG(...) __VA_ARGS__
#else
#define UPBP_MISDBG(...)
#endif

}  // namespace upbp
