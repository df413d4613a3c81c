// Device-side scene records, per-iteration parameters and the record layouts
// of light vertices and photon beams in HBM.
#pragma once

#include "upbp_math.cuh"

namespace upbp {

// Estimator bits (same values as the reference's shared/shared_enums.h).
enum : unsigned {
    kBpt = 1u << 2, kSurf = 1u << 3, kPp3d = 1u << 4, kPb2d = 1u << 5, kBb1d = 1u << 6, kBp2d = 1u << 7,
    kPrevious = 1u << 9, kCompatible = 1u << 10, kSpecularOnly = 1u << 12
};
enum : int { kShortBeam = 1, kLongBeam = 2 };
enum : int { kLightArea = 0, kLightBackground = 1, kLightDirectional = 2, kLightPoint = 3 };
enum : unsigned { kOriginInMedium = 1u << 0, kEndInMedium = 1u << 1 };

// Status bits written to the device status word (upbp.h UPBP_STATUS_*).
enum : unsigned {
    kErrBoundaryStack = 1u << 0, kErrIntersectionArray = 1u << 1, kErrVolSegmentArray = 1u << 2,
    kErrIntersectionStack = 1u << 3, kErrBeamCapacity = 1u << 4, kErrTraversalStack = 1u << 5
};

// Work counters per pass (warp-aggregated 64-bit atomics), the numerator of
// the algorithmic-bytes roofline: BVH node visits, triangle tests, rays cast,
// photon-point candidates / accepted merges, beam-chunk candidates / accepted
// merges, light-vertex records read by BPT connections.
enum : int {
    kCtrNodes = 0, kCtrTris, kCtrRays, kCtrPointCand, kCtrPointHit, kCtrBeamCand, kCtrBeamHit, kCtrVertexLoads,
    kCtrCount
};

struct DMaterial {
    float3 diffuse;
    float3 phong;
    float phong_exponent;
    float3 mirror;
    float ior;
    int priority;
    int real;
    int medium;
};

struct DMedium {
    float3 absorption, emission, scattering, attenuation;
    float min_pos_att;      // minimum positive attenuation component
    int min_pos_att_idx;
    float max_beam_length;
    int has_scattering;
    int has_attenuation;
    float cont_prob;
    float mean_cosine;
};

struct DLight {
    int type;
    int mat_id, med_id;
    float3 p0, e1, e2;      // area: triangle corner and edges
    Frame frame;            // area: frame from e1 x e2; directional: from direction
    float3 intensity;       // area/point/directional; background colour * scale
    float inv_area;
    float3 position;        // point light
    int env;                // background: radiance from the environment map
    float scale;            // background: scale of the environment map's radiance
};

// Environment map of the background light (gpuupbp/shared/env_map.h): the
// image and a piecewise-constant 2-D distribution over 2 * height columns x
// height rows, row r holding nu function values then nu + 1 cdf values,
// row nv the marginal over rows.
struct DEnvMap {
    const float4* img;      // width x height, rgb
    int width, height;
    const float* dist;      // (nv + 1) x (2 nu + 1)
    const float* row_int;   // integral of each row's function
    float marg_int;         // integral of the marginal
    int nu, nv;
    float norm;             // 1 / (2 pi^2)
};

struct DCamera {
    float3 origin, direction;
    float res_x, res_y;
    float raster_to_world[16];   // row-major 4x4
    float world_to_raster[16];
    float image_plane_dist;
    int mat_id, med_id;
};

// Two-wide BVH node: both children's boxes + child links.  A link >= 0 is an
// internal node, a link < 0 is a leaf: ~(first | (count - 1) << 27) for the
// `count` consecutive primitives (every tree here is built with one
// primitive per leaf; the walks accept longer leaves) from position `first`
// of the sorted order.  z and w count the primitives under the left and right
// child.
struct BvhNode {
    float4 a;   // left.lo.xyz, left.hi.x
    float4 b;   // left.hi.yz, right.lo.xy
    float4 c;   // right.lo.z, right.hi.xyz
    int4 link;  // left, right, left count, right count
};

constexpr int kLeafShift = 27;
constexpr unsigned kMaxBvhPrimitives = 1u << kLeafShift;
UPBP_HD int leaf_link(int first, int count) { return ~(first | ((count - 1) << kLeafShift)); }
UPBP_HD int leaf_first(int link) { return (~link) & ((1 << kLeafShift) - 1); }
UPBP_HD int leaf_count(int link) { return ((~link) >> kLeafShift) + 1; }

// Compressed two-wide node of a photon map, 32 bytes (half a BvhNode), for
// the range searches, which were bound by the L1's lookups (lanes of a warp
// read nodes at unrelated addresses and each lane's 16-byte part of a load is
// looked up separately; the path kernels, bound by divergence, stay on
// BvhNodes, where decoding cost more than it saved): the node's box
// origin and a power-of-two step per axis, both children's boxes as 8-bit
// multiples of the step (lower planes rounded down, upper planes up, with
// the decoder's own arithmetic, so each stored box contains the exact one),
// and the children of a Karras hierarchy of one-primitive leaves, which are
// always gamma and gamma + 1: link = gamma | left-is-leaf << 30 |
// right-is-leaf << 31.
struct __align__(32) QNode {
    float4 a;  // origin.xyz; w: biased step exponents x | y << 8 | z << 16
    uint4 b;   // plane bytes: left lo xyz, left hi xyz, right lo xyz, right hi xyz; w: link
};

// Step 2^(e - 127) of a biased exponent byte e in 1..254.
UPBP_D float qnode_step(unsigned e) { return __uint_as_float(e << 23); }

// Plane `byte` of a QNode word: origin + q * step with q the byte (the one
// rounding of the decoder; the encoder checks its bytes with it).
UPBP_D float qnode_plane(unsigned word, int byte, float step, float origin)
{
    return __fmaf_rn((float)((word >> (8 * byte)) & 0xffu), step, origin);
}

struct BvhView {
    const BvhNode* nodes;
    unsigned count;          // primitives
    const QNode* qnodes;     // the same hierarchy compressed (photon maps), or nullptr
};

// Triangles in BVH leaf order: v0 (w = original index bits), e1, e2.
struct TriView {
    BvhView bvh;
    const float4* tri;       // 3 float4 per triangle
    const float4* normals;   // 4 float4 per triangle (n0, n1, n2, face), original order
    const int2* record;      // (material, light) per triangle, original order
    // Analytic spheres of this class, tested one by one (the predefined
    // scenes have at most seven): centre and radius as the reference
    // recovers them from the sphere's box, and the material.
    const float4* spheres;
    const int* sph_mat;
    int sphere_count;
};

// Light vertex record: 8 x 16 B, one per stored light-subpath vertex, placed
// at slot path * slots_per_path + k so a subpath's vertices are contiguous.
//   q0: hitpoint.xyz, meta bits (path_length | flags << 8 | bsdf_flags << 16)
//   q1: throughput.xyz, continuation probability
//   q2: d_shared, d_bpt, d_pde, ray_sample_for_pdf_inv
//   q3: ray_sample_rev_pdf_inv, for_pdfs_ratio, rev_pdfs_ratio, id bits (mat or med id | prev bits << 24)
//   q4: frame z (shading normal or -world_dir_fix), ior or mean cosine
//   q5: local_dir_fix.xyz (surface) / world_dir_fix (medium), cos_theta_fix_geom
//   q6: local geometry normal.xyz, reflect coefficient
//   q7: diffuse / phong / reflect / refract probabilities
struct LightVertexRec {
    float4 q[8];
};

// Photon beam record: 8 x 16 B.
//   q0: origin.xyz, length        q1: direction.xyz, medium id bits
//   q2: throughput at origin.xyz, ray_sample_for_pdf
//   q3: ray_sample_rev_pdf, sampling flags bits, path index bits, path length bits
//   q4: d_shared, d_bpt, d_pde, ray_sample_for_pdf_inv
//   q5: ray_sample_rev_pdf_inv, for_pdfs_ratio, rev_pdfs_ratio, bits (prev_in_medium | prev_specular<<1 | infinite<<2)
//   q6: last_sin_theta, d_bpt_a, d_bpt_b, d_pde_a
//   q7: d_pde_b, distance from the light vertex that traced the ray to the origin, 0, 0
struct BeamRec {
    float4 q[8];
};

// Camera-pass query records (wavefront camera pass).
// Segment query (PB2D / BB1D along one medium segment of a camera ray):
//   q0: origin.xyz, dmin   q1: direction.xyz, dmax
//   q2: weight.xyz (path throughput x attenuation before the segment), medium id bits
//   q3: ray_sample_for_pdf, ray_sample_rev_pdf, sampling flags bits, pixel << 8 | camera path length
//   q4..q7: camera StateWeights in the beam record layout (BeamRec q4..q7);
//   q7.y camera path bits, q7.z event key bits
struct SegQueryRec {
    float4 q[8];
};
// Point query (SURF / PP3D / BP2D at one camera vertex): a LightVertexRec
// of the camera vertex (throughput, weights, BSDF) plus
//   q8: pixel bits, estimator mask bits (1 SURF, 2 PP3D, 4 BP2D), camera path bits, event key bits
struct PointQueryRec {
    LightVertexRec v;
    float4 q8;
};

// Camera vertex of deferred connections (NEE and BPT occlusion rays run in
// their own kernels): the vertex in the light-vertex layout (behind-surface
// bit included), then
//   q8: pixel bits, boundary-stack size bits, camera path bits, bounce bits
//   stack[i] = (material, medium) of the camera path's boundary stack at the
//   vertex, bottom first; the priorities follow from the materials.
constexpr int kConnStack = 20;
struct ConnVertexRec {
    LightVertexRec v;
    float4 q8;
    int2 stack[kConnStack];
};
// Next-event estimation sample whose occlusion ray is still to be traced:
//   q0: vertex position.xyz, distance to the light sample
//   q1: direction to the light.xyz, camera-vertex record index bits
//   q2: light radiance.xyz, cos_to_light / (pick * direct_pdf_w)
//   q3: BSDF value.xyz, w_light = bsdf pdf / (pick * direct_pdf_w)
//   q4: emission_pdf_w * cos_to_light / (direct_pdf_w * cos_at_light), reverse bsdf pdf, sin theta, flag bits
struct NeeRec {
    float4 q[5];
};

// Point map: BVH over light-vertex positions in leaf order.
//   pos[i] = (position.xyz, slot index bits)
struct PointMap {
    BvhView bvh;
    const float4* pos;
};

// Beam map: BVH over beam chunks (sub-segments of each beam) in leaf order.
//   seg[3i] = (origin.xyz, length), seg[3i+1] = (direction.xyz, beam index bits),
//   seg[3i+2] = (t0, t1) of the beam chunk this leaf covers, beam medium id
//   bits, chunk index | chunk count << 16 bits
struct BeamMap {
    BvhView bvh;
    const float4* seg;
    float dilate;  // the leaf boxes' dilation (BoxSource.dilate of the build)
};

// Parameter range [t0, t1) of chunk k of n along a beam of length len.  Both
// neighbours evaluate the shared boundary with the same expression, so the
// chunks partition [0, len) exactly.
UPBP_HD float chunk_t(float len, unsigned k, unsigned n) { return k >= n ? len : len * (float)k / (float)n; }

// Box of chunk k of n of the beam (o, d, len): the beam-map builder's leaf
// box, widened to cover the rounding of o + d t at both ends.  Written with
// round-to-nearest intrinsics (no fused multiply-add), so the build and the
// BB1D reporting rule compute the same box bit for bit.
UPBP_D float3 rn_axpy(float3 o, float3 d, float t)
{
    return make_float3(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)),
                       __fadd_rn(o.z, __fmul_rn(d.z, t)));
}

UPBP_D void chunk_box(float3 o, float3 d, float len, unsigned k, unsigned n, float3& lo, float3& hi)
{
    const float t0 = chunk_t(len, k, n), t1 = chunk_t(len, k + 1, n);
    const float3 a = rn_axpy(o, d, t0), e = rn_axpy(o, d, t1);
    lo = make_float3(fminf(a.x, e.x), fminf(a.y, e.y), fminf(a.z, e.z));
    hi = make_float3(fmaxf(a.x, e.x), fmaxf(a.y, e.y), fmaxf(a.z, e.z));
    const float m = __fmul_rn(1e-6f, __fadd_rn(__fadd_rn(__fadd_rn(fabsf(lo.x), fabsf(lo.y)), fabsf(lo.z)), 1e-3f));
    const float3 ext = make_float3(__fadd_rn(__fmul_rn(__fsub_rn(hi.x, lo.x), 1e-6f), m),
                                   __fadd_rn(__fmul_rn(__fsub_rn(hi.y, lo.y), 1e-6f), m),
                                   __fadd_rn(__fmul_rn(__fsub_rn(hi.z, lo.z), 1e-6f), m));
    lo = lo - ext;
    hi = hi + ext;
}

// A photon map's leaf box: the primitive's box dilated by the largest query
// radius (plus rounding margins) of the map, so the walks test boxes as
// they are.  The same expression builds the box and re-tests it.
UPBP_HD void dilate_box(float3& lo, float3& hi, float d)
{
    lo = lo - v3(d);
    hi = hi + v3(d);
}

// Chunk of n holding parameter t of a beam of length len (t in [0, len)).
UPBP_HD unsigned chunk_of(float t, float len, unsigned n)
{
    unsigned k = (unsigned)fminf(fmaxf(t / len * (float)n, 0.f), (float)(n - 1));
    while (k > 0 && t < chunk_t(len, k, n)) k--;
    while (k + 1 < n && t >= chunk_t(len, k + 1, n)) k++;
    return k;
}

// Counters of one range-search round: hits found (may exceed the hit list's
// capacity; 64-bit, a dense iteration finds billions) and queries handed out
// (may exceed the round's range by the last requests).
struct HitState {
    unsigned long long total;
    unsigned fetched;
    unsigned pad;
};

// Learned proposal table (upbp_guide.cuh): entries over cells^3 x dir_res^2
// directions of travel x media slots; entries == nullptr: no guiding.
struct GuideTable {
    const float4* entries;
    float3 lo, inv_cell;     // scene box and grid step
    int cells, dir_res;      // cells per axis, direction bins per octahedral axis
    int slots;               // media slots in the table
    const int* medium_slot;  // medium id -> slot, -1 if not guided
};

// Training record of the learned proposal, one per medium vertex of a light
// subpath.
struct GuideRecord {
    float4 a;  // position.xyz, medium bits
    float4 b;  // direction of travel of the light subpath.xyz, throughput luminance
};

struct DeviceParams {
    // scene
    const DMaterial* materials;
    int material_count;
    const DMedium* media;
    int medium_count;
    int global_medium;
    const DLight* lights;
    int light_count;
    int background_light;
    DEnvMap env;
    DCamera camera;
    float3 scene_center;
    float scene_radius, inv_radius_sqr;
    // Margins of the photon maps' box dilation beyond the radius: cull_eps
    // covers the rounding of box tests at the scene's coordinate magnitude;
    // beam_cull_eps (beam map) also covers the BB1D predicate's error in t1:
    // for 1 - dd^2 >= 1e-5 (the predicate rejects flatter pairs) t1 is off by
    // at most ~2.4e-7 |coordinates| / (1 - dd^2), so the query point at the
    // computed t1 can lie up to ~8e-5 |coordinates| farther from the beam than
    // the line distance.
    float cull_eps, beam_cull_eps;
    TriView real;
    TriView imag;

    // configuration (fixed for the context)
    unsigned min_path_length, max_path_length;
    int photon_beam_type, camera_beam_type;
    float subpath_count_bpt, subpath_count_bb1d, subpath_count_bp2d, subpath_count_pb2d, subpath_count_pp3d,
        subpath_count_surf;
    int trace_light_paths, trace_camera_paths;
    int do_bpt, do_bb1d, do_bp2d, do_pb2d, do_pp3d, do_surf;
    int build_bb1d, build_bp2d, build_pb2d, build_pp3d, build_surf;
    int connect_to_camera_from_surf, ignore_fully_spec_paths, use_shading_normal;
    unsigned estimator_techniques;
    unsigned screen_pixel_count, light_subpath_count, bb1d_used_light_subpath_count;
    // 0: the reference's MIS weights; 1: weights equal to the full-path
    // balance heuristic where the reference's recursion departs from it
    // (photon-beam merges measure the light-side distance from the light
    // vertex, first-segment BB1D beams of finite lights include it, and the
    // NEE weight includes the media on the camera side of the light ray)
    int mis_exact;
    unsigned res_x, res_y;
    unsigned long long iteration_offset;

    // per iteration
    unsigned iteration;
    float bb1d_normalization, bp2d_normalization, pb2d_normalization, pp3d_normalization, surf_normalization;
    float mis_factor_bb1d, mis_factor_bp2d, mis_factor_pb2d, mis_factor_pp3d, mis_factor_surf;
    float radius_bb1d, radius_bp2d, radius_pb2d, radius_pp3d, radius_surf;
    float radius_bb1d_2, radius_bp2d_2, radius_pb2d_2, radius_pp3d_2, radius_surf_2;
    float rad_point_med, rad_beam;

    // light-pass records
    LightVertexRec* vertices;
    unsigned slots_per_path;
    unsigned* path_vertex_count;      // stored vertices per light subpath
    unsigned* counters;               // [0] vertices [1] surface [2] medium [3] beams [4] next light path
    unsigned* idx_surface;            // vertex slots of surface vertices (append order)
    unsigned* idx_medium;
    BeamRec* beams;
    unsigned beam_capacity;
    float* framebuffer;               // W*H*3
    unsigned* status;
    unsigned* assert_counts;  // -assert: failed assertions, then one count per status bit; null without it
    unsigned long long* work;         // kCtrCount counters of the running pass

    // photon maps built after the light pass
    PointMap surf_map, med_map;
    BeamMap beam_map;
    unsigned n_surface, n_medium, n_beams;   // host-side copies of the light-pass counters

    // wavefront camera pass
    SegQueryRec* seg_queue;
    unsigned seg_capacity;
    PointQueryRec* pt_queue;
    unsigned pt_capacity;
    unsigned* queue_count;            // [0] segment queries [1] point queries [2] next camera pixel
                                      // [3] connection vertices [4] NEE samples [5] BPT pairs
    const unsigned* seg_order;        // processing order of segment queries (Morton order of the midpoint)
    const unsigned* pt_order;         // processing order of point queries (Morton order of the position)
    float* cam_fb;                    // camera-pass image, W*H*3

    // Range-query hit list (PB2D, BB1D, BP2D): a search round appends every
    // (query, neighbour) pair the predicate accepts for the queries
    // [query_begin, query_end) of the processing order; the evaluation kernel
    // consumes the list.  A round stops handing out queries once
    // hit_soft_limit hits were found, so that the queries in flight still
    // fit; the host runs rounds until every query was handed out.
    uint2* hit_qb;                    // (query record index, beam index or light-vertex slot)
    unsigned hit_capacity;
    unsigned query_begin, query_end;
    unsigned long long hit_soft_limit;
    HitState* hit_state;

    // deferred camera-side connections; counts in queue_count[3..5]
    ConnVertexRec* conn_vertices;
    unsigned conn_capacity;
    NeeRec* nee_queue;
    unsigned nee_capacity;
    uint2* bpt_pairs;                 // (camera-vertex record, light-vertex slot)
    unsigned bpt_capacity;
    float4* nee_color;                // contribution of each NEE sample (after its occlusion ray)
    float4* bpt_color;                // contribution of each BPT pair
    // Per camera path (index = the pixel it was generated for): the first
    // event key at which a deferred connection failed (~0: none), and the
    // emitter-hit colour of the path with its target pixel.  A failed step
    // ends a path in the reference, so contributions with a later key drop.
    unsigned* path_err;
    float4* path_color;

    // learned proposal: the table camera subpaths sample and every
    // camera-direction pdf reads; the light pass appends training records
    // while guide_collect is set
    GuideTable guide;
    GuideRecord* guide_recs;
    unsigned* guide_rec_count;
    unsigned guide_rec_capacity;
    int guide_collect;
};

// Event keys order the contributions of a camera path as the reference's
// path loop makes them: bounce * 256 + step, step = 1 segment merges (PB2D,
// BB1D), 2 NEE, 3 + k BPT connection k, 255 point merges (SURF, PP3D, BP2D).
enum : unsigned { kEvSegment = 1u, kEvNee = 2u, kEvBpt = 3u, kEvPoint = 255u };
UPBP_HD unsigned event_key(unsigned bounce, unsigned step) { return bounce * 256u + step; }

// Launch parameters: one slot per context (kParamSlots per device), each
// uploaded by its context before its launches on its own stream.  Every
// kernel that reads them takes its context's slot as an argument and records
// it in shared memory at entry; device code names the running kernel's
// parameters c_params.  Contexts therefore run concurrently, each on its own
// slot and stream.
//
// The hot kernels are also compiled a second time (upbp_slot0.cu, its own
// namespace) against a bank of one fixed slot: reading c_slots[s_slot] is
// a constant-bank load of its own at every access, reading a fixed bank an
// operand of the instruction that uses it (3% of an iteration).  Slot 0 --
// the slot of a context running alone -- launches that copy; its
// parameters are uploaded to both banks.
constexpr int kParamSlots = 48;
__shared__ int s_slot;
__shared__ int s_kernel_kind;
#ifdef UPBP_SLOT0_BANK
__constant__ DeviceParams c_slot0;
#define c_params (c_slot0)
#else
__constant__ DeviceParams c_slots[kParamSlots];
#define c_params (c_slots[s_slot])
#endif

// Records the running kernel's parameter slot and kind (for its work
// counters); every thread of the block calls it first, before any early
// return.
UPBP_D void begin_kernel(int kind, int slot)
{
    if (threadIdx.x == 0) {
        s_kernel_kind = kind;
        s_slot = slot;
    }
    __syncthreads();
}

// Work counters of every kernel kind (kKernRows sets of kCtrCount at
// c_params.work): the running kernel's set.
UPBP_D unsigned long long* c_work_ptr() { return c_params.work + (size_t)s_kernel_kind * kCtrCount; }

// Kernel kinds of an iteration, for work counters and timing.  The
// diagnostic neighbour queries count into a row of their own after the
// iteration's rows (kKernDebug), so they never change an iteration's figures.
enum : int {
    kKernLight = 0, kKernCameraExtend, kKernPb2d, kKernBb1d, kKernSurf, kKernPp3d, kKernBp2d, kKernNee, kKernBpt,
    kKernCount, kKernDebug = kKernCount, kKernRows
};

}  // namespace upbp
