// C ABI of libupbp_b200.so: context creation (scene upload, scene BVHs,
// record buffers) and the per-iteration schedule (radius reduction, light
// pass, photon-map builds, camera pass, accumulation).  Mirrors
// Renderer::init (gpuupbp/renderer/renderer_init.cpp:675-929) and
// Renderer::run_iteration (gpuupbp/renderer/renderer.cpp:37-418).
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "host/upbp_scene.h"
#include "upbp_build.cuh"
#include "upbp_camera_pass.cuh"
#include "upbp_ploc.cuh"
#include "upbp_light_pass.cuh"
#include "upbp_scene_bvh.cuh"
#include "upbp_kernel_table.h"

using namespace upbp;

constexpr int kEventRing = 64;
// Events per iteration: 0 start, 1 light pass done, 2 photon maps done, 3
// extend, 4 NEE, 5 BPT + resolve, 6 query sort, 7 SURF, 8 PP3D, 9 BP2D,
// 10 PB2D, 11 BB1D, 12 iteration done.  Each kernel kind's time is one
// interval.
constexpr int kEvPerIter = 14;  // [13]: end of the light pass, start of the proposal's training
struct EvInterval {
    int kind, from, to;
};
constexpr EvInterval kKindInterval[kKernCount] = {
    {kKernLight, 0, 1}, {kKernCameraExtend, 2, 3}, {kKernNee, 3, 4},   {kKernBpt, 4, 5},  {kKernSurf, 6, 7},
    {kKernPp3d, 7, 8},  {kKernBp2d, 8, 9},         {kKernPb2d, 9, 10}, {kKernBb1d, 10, 11}};

namespace {

#define UPBP_CK(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            upbp_host::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));              \
            return UPBP_ERR_CUDA;                                                                  \
        }                                                                                          \
    } while (0)

// Makes device `dev` current for the scope of an entry point and restores
// the caller's device after it: every call works on the device its context
// was created on, whichever device the calling thread has current.
class DeviceGuard {
  public:
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != dev) err_ = cudaSetDevice(dev);
        else prev_ = dev;
        dev_ = dev;
    }
    ~DeviceGuard()
    {
        if (prev_ != dev_) cudaSetDevice(prev_);
    }
    cudaError_t error() const { return err_; }

  private:
    int prev_ = 0, dev_ = 0;
    cudaError_t err_ = cudaSuccess;
};

// Parameter slots (c_slots) of each device.  A call that launches
// parameter-reading kernels leases the lowest free slot for its duration
// (every such call ends with a synchronisation of the context's stream, so
// no kernel of it still reads the slot afterwards); any number of contexts
// may exist, and up to kParamSlots of them run at once -- a further call
// waits for a slot.
constexpr int kMaxDevices = 64;
constexpr int kAssertCounts = 7;  // -assert: failed assertions + the six UPBP_STATUS_* bits
struct SlotTable {
    std::mutex mu;
    std::condition_variable freed;
    bool used[kParamSlots] = {};
};
SlotTable g_slots[kMaxDevices];

class SlotLease {
  public:
    SlotLease(int dev, int& slot, cudaStream_t st) : t_(g_slots[dev]), slot_(slot), st_(st)
    {
        std::unique_lock<std::mutex> lk(t_.mu);
        for (;;) {
            for (int i = 0; i < kParamSlots; i++)
                if (!t_.used[i]) {
                    t_.used[i] = true;
                    slot_ = i;
                    return;
                }
            t_.freed.wait(lk);
        }
    }
    ~SlotLease()
    {
        // no kernel of the call may still read the slot (an error return
        // skips the call's own final synchronisation)
        cudaStreamSynchronize(st_);
        {
            std::lock_guard<std::mutex> lk(t_.mu);
            t_.used[slot_] = false;
            slot_ = -1;
        }
        t_.freed.notify_one();
    }

  private:
    SlotTable& t_;
    int& slot_;
    cudaStream_t st_;
};

// Range-query hit lists are needed only while an iteration's searches run.
// Contexts of a device borrow them from a pool for the duration of
// upbp_run_iteration, so contexts driven by W threads at once hold at most W
// lists (a 64-job batch would otherwise keep 64, each grown to its job's
// largest iteration); a returned list keeps its size for the next borrower.
// The pool's idle lists are freed with the device's last context, or to make
// room when a list cannot grow.
struct HitPool {
    std::mutex mu;
    std::vector<std::pair<uint2*, unsigned>> idle;  // (list, capacity in entries)
    int contexts = 0;
};
HitPool g_hit_pool[kMaxDevices];

// Frees the device's idle hit lists (the device must be current).
void hit_pool_release_idle(int dev)
{
    HitPool& p = g_hit_pool[dev];
    std::lock_guard<std::mutex> lk(p.mu);
    for (auto& h : p.idle) cudaFree(h.first);
    p.idle.clear();
}

template <class T>
cudaError_t dalloc(T** p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
}

// Reallocates *p for at least n elements (n + n/4) when n exceeds cap;
// the old contents are dropped.
template <class T>
cudaError_t grow(T** p, unsigned& cap, unsigned n)
{
    if (n <= cap) return cudaSuccess;
    cudaFree(*p);
    cap = n + n / 4;
    return dalloc(p, cap);
}

template <class T>
cudaError_t dupload(T** p, const T* h, size_t n, cudaStream_t st)
{
    cudaError_t e = dalloc(p, n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(*p, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
}

// Neighbour sets of n queries through the estimators' range-query walkers.
// Query record: x y z dx dy dz tmin tmax (points use x y z only).
__global__ void k_debug_query(int slot, int kind, const float* q, unsigned n, unsigned* counts, unsigned* ids,
                              unsigned cap)
{
    begin_kernel(kKernDebug, slot);
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DeviceParams& p = c_params;
    const float* r = q + 8 * (size_t)i;
    const float3 x = make_float3(r[0], r[1], r[2]), d = make_float3(r[3], r[4], r[5]);
    unsigned k = 0;
    auto rec = [&](unsigned id) {
        if (k < cap) ids[(size_t)i * cap + k] = id;
        k++;
    };
    switch (kind) {
    case 0:
        points_in_radius(p.surf_map, x, p.radius_surf_2, [&](unsigned s) { rec(s); });
        break;
    case 1:
        points_in_radius(p.med_map, x, p.radius_pp3d_2, [&](unsigned s) { rec(s); });
        break;
    case 2:
        points_near_segment(p.med_map, x, d, r[6], r[7], p.radius_pb2d_2,
                            [&](unsigned s, float, float) { rec(s); });
        break;
    case 3:
        beams_near_segment(p.beam_map, x, d, r[6], r[7], p.radius_bb1d_2, p.do_bp2d != 0, -1,
                           [&](unsigned b, float, float, float, float) { rec(b); });
        break;
    default:
        beams_near_point(p.beam_map, x, p.radius_bp2d_2, [&](unsigned b, float, float) { rec(b); });
        break;
    }
    counts[i] = k;
}

}  // namespace

#include "upbp_guide_train.cuh"

namespace {

struct Geometry {
    BvhNode* nodes = nullptr;
    float4* tri = nullptr;
    float4* normals = nullptr;
    int2* record = nullptr;
    unsigned count = 0;
    float4* spheres = nullptr;  // centre, radius
    int* sph_mat = nullptr;
    unsigned sph_count = 0;
};

}  // namespace

struct upbp_ctx {
    upbp_config cfg{};
    DeviceParams P{};
    int dev = 0;                              // device the context was created on
    int slot = -1;                            // its launch-parameter slot during a call (SlotLease)
    cudaStream_t st = nullptr;
    unsigned* h_status = nullptr;             // page-locked copy of the iteration's status word
    unsigned status_seen = 0;                 // OR of every iteration's status bits
    unsigned char* static_scratch = nullptr;  // device address of the no-allocation query array
    cudaEvent_t ev_ring[kEventRing][kEvPerIter] = {};
    unsigned ev_pending = 0;                   // iterations recorded since the last stats read
    DMaterial* d_mat = nullptr;
    DMedium* d_med = nullptr;
    float4* d_env_img = nullptr;   // environment map and its sampling distribution
    float* d_env_dist = nullptr;
    float* d_env_row_int = nullptr;
    DLight* d_lights = nullptr;
    Geometry real, imag;
    LightVertexRec* d_vertices = nullptr;
    unsigned* d_path_count = nullptr;
    unsigned* d_counters = nullptr;
    unsigned* d_idx_s = nullptr;
    unsigned* d_idx_m = nullptr;
    BeamRec* d_beams = nullptr;
    float* d_fb = nullptr;
    double* d_acc = nullptr;
    unsigned* d_status = nullptr;
    BvhNode *d_surf_nodes = nullptr, *d_med_nodes = nullptr, *d_beam_nodes = nullptr;
    QNode *d_med_qnodes = nullptr, *d_beam_qnodes = nullptr;  // compressed copies for the range searches
    float4 *d_surf_pos = nullptr, *d_med_pos = nullptr, *d_beam_seg = nullptr;
    unsigned *d_chunk_counts = nullptr, *d_chunk_offsets = nullptr;
    uint2* d_chunks = nullptr;
    unsigned chunk_capacity = 0;
    PlocScratch ploc;  // the beam map's clustering (sized with the chunks)
    unsigned beam_map_passes = 0;  // clustering passes of the last beam map (0: LBVH)
    unsigned* h_ploc = nullptr;    // page-locked outcome of the last clustering (kPcWords)
    bool ploc_pending = false;     // its outcome is not read yet
    BoxSource ploc_src{};          // the build's source and size, to replace the tree
    unsigned ploc_n = 0;
    int ploc_budget = kPlocPasses;  // passes launched for the next beam map
    int ploc_cap = kPlocPasses;     // UPBP_PLOC_PASSES: at most this many
    int ploc_failures = 0;          // builds that ran out with every pass allowed
    bool ploc_off = false;  // UPBP_BEAM_MAP=lbvh: the beam map as a Morton-split LBVH
    void* d_scan_temp = nullptr;
    size_t scan_temp_bytes = 0;
    unsigned last_chunks = 0;
    unsigned long long* d_work = nullptr;   // kKernCount x kCtrCount
    unsigned launches = 0;
    size_t h2d_iter = 0, d2h_iter = 0;
    SegQueryRec* d_seg_queue = nullptr;
    PointQueryRec* d_pt_queue = nullptr;
    unsigned seg_capacity = 0, pt_capacity = 0;
    unsigned* d_qcount = nullptr;
    float* d_cam_fb = nullptr;
    unsigned h_qcount[6] = {0, 0, 0, 0, 0, 0};
    // deferred NEE / BPT connections of the camera pass
    ConnVertexRec* d_conn = nullptr;
    NeeRec* d_nee = nullptr;
    uint2* d_bpt = nullptr;
    float4 *d_nee_color = nullptr, *d_bpt_color = nullptr;
    unsigned conn_capacity = 0, nee_capacity = 0, bpt_capacity = 0;
    unsigned* d_path_err = nullptr;
    float4* d_path_color = nullptr;
    // range-query hit list (search -> evaluation), round counters, and a
    // copy of one kernel kind's work counters for a round that is repeated
    uint2* d_hit_qb = nullptr;
    unsigned hit_capacity = 0;
    size_t hit_want = 0;  // list size the last growth asked for (the pool's best fit)
    double ms_scene_bvh = 0;  // device time of the scene BVH builds in upbp_create
    uint64_t render_hash = 0;  // configuration + scene fingerprint a checkpoint must match
    unsigned* d_assert = nullptr;  // -assert: event counts (assertions, then one per status bit)
    size_t max_hits = 0;  // largest list: kMaxHits, or UPBP_MAX_HITS entries when that is smaller
    HitState* d_hit_state = nullptr;
    HitState h_hit_state = {};
    unsigned long long* d_work_saved = nullptr;
    int search_grid[kRangeModes] = {};  // per range-query mode (kModePb2d ...)
    int eval_grid[kRangeModes] = {};    // resident blocks of each evaluation kernel
    int camera_grid = 0;   // resident blocks of the persistent camera pass
    int light_grid = 0;    // resident blocks of the persistent light pass
    unsigned grid_limit = 0;  // cap on any launch's blocks (0: none), so that concurrent contexts share the SMs
    // Morton sort of the query records: keys/values and their alternates per queue
    unsigned* d_sort[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
    unsigned sort_capacity[2] = {0, 0};
    void* d_sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    BuildScratch sc;
    float r0[5] = {0, 0, 0, 0, 0};  // bb1d bp2d pb2d pp3d surf
    float bb1d_used = 0.f;
    unsigned vertex_capacity = 0, beam_capacity = 0;
    unsigned h_counters[4] = {0, 0, 0, 0};
    unsigned iterations = 0;
    uint64_t triangles = 0;
    MisDebug mis{};  // MIS recording buffers (recording build only)
    GuideState guide;  // learned proposal (guide.train_iterations > 0)
    float3 bbox_lo{}, bbox_hi{};
};

namespace {

// Blocks of a launch under the context's grid limit (at least one).
// Borrows the largest idle hit list of the context's device for one call
// and returns it (after the call's kernels are done) at the end.
class HitLease {
  public:
    explicit HitLease(upbp_ctx* c);
    ~HitLease();

  private:
    upbp_ctx* c_;
};

unsigned cap_grid(const upbp_ctx* c, unsigned blocks)
{
    return c->grid_limit ? std::max(1u, std::min(blocks, c->grid_limit)) : blocks;
}

// This compilation's parameter-reading kernels (the indexed slot bank).
const upbp_kernels::ParamKernels& slotted_kernels()
{
    static const upbp_kernels::ParamKernels k = {
        light_pass_kernel,
        camera_pass_kernel,
        nee_connect_kernel,
        bpt_connect_kernel,
        k_resolve_camera,
        {k_query_keys<false>, k_query_keys<true>},
        {range_search_kernel<kModePb2d>, range_search_kernel<kModeBb1d>, range_search_kernel<kModeBp2d>},
        {{range_eval_kernel<kModePb2d, false>, range_eval_kernel<kModePb2d, true>},
         {range_eval_kernel<kModeBb1d, false>, range_eval_kernel<kModeBb1d, true>},
         {range_eval_kernel<kModeBp2d, false>, range_eval_kernel<kModeBp2d, true>}},
        {{point_merge_kernel<false, false>, point_merge_kernel<false, true>},
         {point_merge_kernel<true, false>, point_merge_kernel<true, true>}},
    };
    return k;
}

// The kernels a call of context c launches: the fixed-bank copy (built
// without analytic spheres) on slot 0 for a scene without spheres.
const upbp_kernels::ParamKernels& PK(const upbp_ctx* c)
{
    const bool spheres = c->real.sph_count + c->imag.sph_count > 0;
    return c->slot == 0 && !spheres ? upbp_kernels::slot0_kernels() : slotted_kernels();
}

HitLease::HitLease(upbp_ctx* c) : c_(c)
{
    // the smallest idle list that holds what the context's last iteration
    // needed, else the largest (which then grows): a list is not freed and
    // reallocated (a device-wide synchronisation) while one of the right
    // size sits idle
    HitPool& p = g_hit_pool[c->dev];
    std::lock_guard<std::mutex> lk(p.mu);
    if (p.idle.empty()) return;
    auto pick = p.idle.end(), largest = p.idle.begin();
    for (auto it = p.idle.begin(); it != p.idle.end(); ++it) {
        if (it->second > largest->second) largest = it;
        if (it->second >= c->hit_want && (pick == p.idle.end() || it->second < pick->second)) pick = it;
    }
    if (pick == p.idle.end()) pick = largest;
    c->d_hit_qb = pick->first;
    c->hit_capacity = pick->second;
    p.idle.erase(pick);
}

HitLease::~HitLease()
{
    if (!c_->d_hit_qb) return;
    cudaStreamSynchronize(c_->st);  // an error return skips the call's own final synchronisation
    HitPool& p = g_hit_pool[c_->dev];
    std::lock_guard<std::mutex> lk(p.mu);
    p.idle.emplace_back(c_->d_hit_qb, c_->hit_capacity);
    c_->d_hit_qb = nullptr;
    c_->hit_capacity = 0;
}

// Uploads the context's launch parameters into its slot (stream-ordered
// before the launches that read them).
cudaError_t upload_params(upbp_ctx* c)
{
    const cudaError_t e = cudaMemcpyToSymbolAsync(c_slots, &c->P, sizeof(DeviceParams), sizeof(DeviceParams) * (size_t)c->slot,
                                   cudaMemcpyHostToDevice, c->st);
    if (e != cudaSuccess || c->slot != 0) return e;
    return upbp_kernels::slot0_upload_params(&c->P, sizeof(DeviceParams), c->st);
}

void init_medium(DMedium& m, const upbp_medium& in)
{
    m.absorption = make_float3(fabsf(in.absorption[0]), fabsf(in.absorption[1]), fabsf(in.absorption[2]));
    m.emission = make_float3(fabsf(in.emission[0]), fabsf(in.emission[1]), fabsf(in.emission[2]));
    m.scattering = make_float3(fabsf(in.scattering[0]), fabsf(in.scattering[1]), fabsf(in.scattering[2]));
    m.attenuation = m.absorption + m.scattering;
    m.cont_prob = in.continuation_prob;
    m.mean_cosine = in.mean_cosine;
    m.min_pos_att = m.attenuation.x;
    m.min_pos_att_idx = 0;
    if (m.attenuation.y > 0.f && (m.min_pos_att == 0.f || m.attenuation.y < m.min_pos_att)) {
        m.min_pos_att = m.attenuation.y;
        m.min_pos_att_idx = 1;
    }
    if (m.attenuation.z > 0.f && (m.min_pos_att == 0.f || m.attenuation.z < m.min_pos_att)) {
        m.min_pos_att = m.attenuation.z;
        m.min_pos_att_idx = 2;
    }
    m.has_scattering = (m.scattering.x > 0.f || m.scattering.y > 0.f || m.scattering.z > 0.f) ? 1 : 0;
    if (m.attenuation.x > 0.f || m.attenuation.y > 0.f || m.attenuation.z > 0.f) {
        m.has_attenuation = 1;
        m.max_beam_length = -logf(1e-9f) / max_component(m.attenuation);
    } else {
        m.has_attenuation = 0;
        m.max_beam_length = kInfinity;
    }
}

void init_light(DLight& l, const upbp_light& in)
{
    std::memset(&l, 0, sizeof(l));
    l.type = in.type;
    l.mat_id = in.mat_id;
    l.med_id = in.med_id;
    const float3 I = make_float3(in.intensity[0], in.intensity[1], in.intensity[2]);
    if (in.type == UPBP_LIGHT_AREA) {
        const float3 p0 = make_float3(in.p0[0], in.p0[1], in.p0[2]);
        const float3 p1 = make_float3(in.p1[0], in.p1[1], in.p1[2]);
        const float3 p2 = make_float3(in.p2[0], in.p2[1], in.p2[2]);
        l.p0 = p0;
        l.e1 = p1 - p0;
        l.e2 = p2 - p0;
        const float3 n = cross(l.e1, l.e2);
        l.inv_area = 2.f / length(n);
        l.frame.set_from_z(n);
        l.intensity = I;
    } else if (in.type == UPBP_LIGHT_BACKGROUND) {
        l.intensity = I * in.scale;
    } else if (in.type == UPBP_LIGHT_DIRECTIONAL) {
        l.frame.set_from_z(make_float3(in.position[0], in.position[1], in.position[2]));
        l.intensity = I;
    } else {
        l.position = make_float3(in.position[0], in.position[1], in.position[2]);
        l.intensity = I;
    }
}

// One piecewise-constant 1-D distribution over n values (init_distribution_1d,
// gpuupbp/host/env_map.hpp): the function, then its cdf normalised by the
// integral (uniform when the integral is 0); returns the integral.  Same
// float operations as the reference, so sampling decisions agree.
float env_distribution_1d(const float* f, int n, float* func, float* cdf)
{
    std::memcpy(func, f, (size_t)n * sizeof(float));
    cdf[0] = 0.f;
    for (int i = 1; i < n + 1; i++) cdf[i] = cdf[i - 1] + func[i - 1] / n;
    const float integral = cdf[n];
    if (integral == 0.f) {
        for (int i = 1; i < n + 1; i++) cdf[i] = float(i) / float(n);
    } else {
        for (int i = 1; i < n + 1; i++) cdf[i] /= integral;
    }
    return integral;
}

// The environment map's image and sampling distribution on the device
// (convert_image_to_pdf, gpuupbp/host/env_map.hpp): 2 * height columns x
// height rows of luminance times the sine of the row's polar angle.
int upload_env_map(upbp_ctx* c, const upbp_scene_desc* s)
{
    const int w = (int)s->env_width, h = (int)s->env_height;
    if (h <= 0 || w < 2 * h) {
        upbp_host::set_error("environment map must be at least twice as wide as high");
        return UPBP_ERR_SCENE;
    }
    const int nu = 2 * h, nv = h;
    std::vector<float4> img((size_t)w * h);
    for (size_t i = 0; i < img.size(); i++)
        img[i] = make_float4(s->env_rgb[3 * i], s->env_rgb[3 * i + 1], s->env_rgb[3 * i + 2], 0.f);
    std::vector<float> lum((size_t)nu * nv);
    for (int r = 0; r < nv; r++) {
        const float v = (float)(r + .5f) / (float)nv;
        const float st = std::sin(3.14159265358979323846f * v);
        for (int col = 0; col < nu; col++) {
            const float4 p = img[(size_t)r * w + col];
            lum[(size_t)r * nu + col] = st * (0.212671f * p.x + 0.715160f * p.y + 0.072169f * p.z);
        }
    }
    const size_t row = 2 * (size_t)nu + 1;
    std::vector<float> dist(row * (nv + 1), 0.f), row_int(nv), marg(nv);
    for (int r = 0; r < nv; r++)
        row_int[r] = env_distribution_1d(&lum[(size_t)r * nu], nu, &dist[row * r], &dist[row * r + nu]);
    for (int r = 0; r < nv; r++) marg[r] = row_int[r];
    const float marg_int = env_distribution_1d(marg.data(), nv, &dist[row * nv], &dist[row * nv + nu]);
    UPBP_CK(dupload(&c->d_env_img, img.data(), img.size(), c->st));
    UPBP_CK(dupload(&c->d_env_dist, dist.data(), dist.size(), c->st));
    UPBP_CK(dupload(&c->d_env_row_int, row_int.data(), row_int.size(), c->st));
    DEnvMap& m = c->P.env;
    m.img = c->d_env_img;
    m.width = w;
    m.height = h;
    m.dist = c->d_env_dist;
    m.row_int = c->d_env_row_int;
    m.marg_int = marg_int;
    m.nu = nu;
    m.nv = nv;
    m.norm = .5f * 0.318309886183790671538f * 0.318309886183790671538f;
    return UPBP_OK;
}

// Fingerprint of everything that decides a render's images: the
// configuration's render fields and the scene's records (FNV-1a over 8-byte
// words).  A checkpoint loads only into a context with the same one.
uint64_t hash_bytes(uint64_t h, const void* p, size_t bytes)
{
    const unsigned char* b = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 0x100000001b3ull;
    }
    for (; i < bytes; i++) h = (h ^ b[i]) * 0x100000001b3ull;
    return h;
}

template <class T>
uint64_t hash_value(uint64_t h, const T& v)
{
    return hash_bytes(h, &v, sizeof(v));
}

uint64_t render_fingerprint(const upbp_scene_desc* s, const upbp_config* c)
{
    uint64_t h = 0xcbf29ce484222325ull;
    const float radii[11] = {c->bb1d_radius_initial, c->bb1d_radius_alpha, c->bb1d_used_light_subpath_count,
                             c->bp2d_radius_initial, c->bp2d_radius_alpha, c->pb2d_radius_initial,
                             c->pb2d_radius_alpha,  c->pp3d_radius_initial, c->pp3d_radius_alpha,
                             c->surf_radius_initial, c->surf_radius_alpha};
    const int64_t ints[14] = {c->scene_id, c->algorithm_flags, c->res_x, c->res_y, c->max_path_length,
                              c->min_path_length, c->query_beam_type, c->photon_beam_type,
                              c->ignore_fully_spec_paths, (int64_t)c->iteration_offset, c->use_shading_normal,
                              c->mis_exact, c->guide_train_iterations, 0};
    h = hash_value(h, radii);
    h = hash_value(h, ints);
    h = hash_value(h, c->path_count_per_iter);
    const size_t n = s->triangle_count;
    h = hash_value(h, s->triangle_count);
    h = hash_bytes(h, s->verts, 9 * n * sizeof(float));
    h = hash_bytes(h, s->normals, 12 * n * sizeof(float));
    h = hash_bytes(h, s->tri_material, n * sizeof(int32_t));
    h = hash_bytes(h, s->tri_light, n * sizeof(int32_t));
    h = hash_bytes(h, s->materials, s->material_count * sizeof(upbp_material));
    h = hash_bytes(h, s->media, s->medium_count * sizeof(upbp_medium));
    h = hash_bytes(h, s->lights, s->light_count * sizeof(upbp_light));
    h = hash_value(h, s->camera);
    h = hash_value(h, s->global_medium);
    h = hash_value(h, s->background_light);
    h = hash_value(h, s->sphere_count);
    if (s->sphere_count) {
        h = hash_bytes(h, s->spheres, 4 * (size_t)s->sphere_count * sizeof(float));
        h = hash_bytes(h, s->sph_material, s->sphere_count * sizeof(int32_t));
    }
    h = hash_value(h, s->env_width);
    h = hash_value(h, s->env_height);
    if (s->env_rgb) h = hash_bytes(h, s->env_rgb, 3 * (size_t)s->env_width * s->env_height * sizeof(float));
    return h;
}

// Static scene: the binned-SAH tree of one class of triangles (original
// order in `tri`: v0, e1, e2), built on the device once per context
// (upbp_scene_bvh.cuh): g.nodes receives the n - 1 nodes, g.tri the
// triangles in leaf order with the original index in v0.w.  The host runs
// the levels of ranges above kSahSmall primitives (reading each level's
// split counts back to lay out the next); one launch finishes the rest.
cudaError_t build_scene_bvh(upbp_ctx* c, Geometry& g, const std::vector<float4>& tri)
{
    const unsigned n = g.count;
    cudaStream_t st = c->st;
    float4 *d_tri = nullptr, *blo = nullptr, *bhi = nullptr, *cen = nullptr;
    unsigned *perm = nullptr, *perm2 = nullptr;
    SahTask* d_tasks = nullptr;
    SahWork* d_work = nullptr;
    SahBins* d_bins = nullptr;
    SahSplit* d_splits = nullptr;
    unsigned *d_chunk_left = nullptr, *d_left_off = nullptr, *d_right_off = nullptr, *d_which = nullptr;
    unsigned task_cap = 0, work_cap = 0;
    auto run = [&]() -> cudaError_t {
        cudaError_t e;
#define SAH_CK(x)                               \
    do {                                        \
        if ((e = (x)) != cudaSuccess) return e; \
    } while (0)
        SAH_CK(dupload(&d_tri, tri.data(), tri.size(), st));
        SAH_CK(dalloc(&blo, n));
        SAH_CK(dalloc(&bhi, n));
        SAH_CK(dalloc(&cen, n));
        SAH_CK(dalloc(&perm, n));
        SAH_CK(dalloc(&perm2, n));
        k_sah_tri_boxes<<<(n + 255) / 256, 256, 0, st>>>(d_tri, n, blo, bhi, cen);
        {
            std::vector<unsigned> iota(n);
            for (unsigned i = 0; i < n; i++) iota[i] = i;
            SAH_CK(cudaMemcpyAsync(perm, iota.data(), n * sizeof(unsigned), cudaMemcpyHostToDevice, st));
            SAH_CK(cudaStreamSynchronize(st));
        }
        std::vector<SahTask> level, small;
        if (n >= 2) (n > kSahSmall ? level : small).push_back(SahTask{0, n, 0, 0});
        while (!level.empty()) {
            std::vector<SahWork> work;
            for (unsigned t = 0; t < level.size(); t++)
                for (unsigned a = level[t].a; a < level[t].e; a += kSahChunk)
                    work.push_back(SahWork{t, a, std::min(a + kSahChunk, level[t].e)});
            const unsigned nt = (unsigned)level.size(), nw = (unsigned)work.size();
            if (nt > task_cap) {
                cudaFree(d_tasks);
                cudaFree(d_bins);
                cudaFree(d_splits);
                cudaFree(d_which);
                d_tasks = nullptr;
                d_bins = nullptr;
                d_splits = nullptr;
                d_which = nullptr;
                task_cap = nt;
                SAH_CK(dalloc(&d_tasks, task_cap));
                SAH_CK(dalloc(&d_bins, task_cap));
                SAH_CK(dalloc(&d_splits, task_cap));
                SAH_CK(dalloc(&d_which, task_cap));
            }
            if (nw > work_cap) {
                cudaFree(d_work);
                cudaFree(d_chunk_left);
                cudaFree(d_left_off);
                cudaFree(d_right_off);
                d_work = nullptr;
                d_chunk_left = d_left_off = d_right_off = nullptr;
                work_cap = nw;
                SAH_CK(dalloc(&d_work, work_cap));
                SAH_CK(dalloc(&d_chunk_left, work_cap));
                SAH_CK(dalloc(&d_left_off, work_cap));
                SAH_CK(dalloc(&d_right_off, work_cap));
            }
            SAH_CK(cudaMemcpyAsync(d_tasks, level.data(), nt * sizeof(SahTask), cudaMemcpyHostToDevice, st));
            SAH_CK(cudaMemcpyAsync(d_work, work.data(), nw * sizeof(SahWork), cudaMemcpyHostToDevice, st));
            k_sah_init_bins<<<nt, 128, 0, st>>>(d_bins, nt);
            k_sah_centroid_bounds<<<nw, kSahThreads, 0, st>>>(d_work, perm, cen, d_bins);
            k_sah_bins<<<nw, kSahThreads, 0, st>>>(d_work, perm, cen, blo, bhi, d_bins);
            k_sah_choose<<<(nt + 127) / 128, 128, 0, st>>>(d_tasks, nt, d_bins, d_splits, g.nodes);
            k_sah_count_left<<<nw, kSahThreads, 0, st>>>(d_work, d_tasks, d_splits, perm, cen, d_chunk_left);
            SAH_CK(cudaGetLastError());
            std::vector<SahSplit> splits(nt);
            std::vector<unsigned> chunk_left(nw), left_off(nw), right_off(nw);
            SAH_CK(cudaMemcpyAsync(splits.data(), d_splits, nt * sizeof(SahSplit), cudaMemcpyDeviceToHost, st));
            SAH_CK(cudaMemcpyAsync(chunk_left.data(), d_chunk_left, nw * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
            SAH_CK(cudaStreamSynchronize(st));
            {
                unsigned task = ~0u, lsum = 0, rsum = 0;
                for (unsigned w = 0; w < nw; w++) {
                    if (work[w].task != task) {
                        task = work[w].task;
                        lsum = rsum = 0;
                    }
                    left_off[w] = lsum;
                    right_off[w] = rsum;
                    lsum += chunk_left[w];
                    rsum += (work[w].e - work[w].a) - chunk_left[w];
                }
            }
            SAH_CK(cudaMemcpyAsync(d_left_off, left_off.data(), nw * sizeof(unsigned), cudaMemcpyHostToDevice, st));
            SAH_CK(cudaMemcpyAsync(d_right_off, right_off.data(), nw * sizeof(unsigned), cudaMemcpyHostToDevice, st));
            SAH_CK(cudaMemcpyAsync(perm2, perm, n * sizeof(unsigned), cudaMemcpyDeviceToDevice, st));
            k_sah_scatter<<<nw, kSahThreads, 0, st>>>(d_work, d_tasks, d_splits, perm, cen, d_left_off, d_right_off,
                                                      perm2);
            std::swap(perm, perm2);
            std::vector<unsigned> middle;
            for (unsigned t = 0; t < nt; t++)
                if (splits[t].axis < 0) middle.push_back(t);
            if (!middle.empty()) {
                SAH_CK(cudaMemcpyAsync(d_which, middle.data(), middle.size() * sizeof(unsigned),
                                       cudaMemcpyHostToDevice, st));
                k_sah_middle_nodes<<<(unsigned)middle.size(), kSahThreads, 0, st>>>(d_tasks, d_which, d_splits, perm,
                                                                                   blo, bhi, g.nodes);
            }
            SAH_CK(cudaGetLastError());
            std::vector<SahTask> next;
            for (unsigned t = 0; t < nt; t++) {
                const SahTask& tk = level[t];
                const unsigned ml = splits[t].ml, mr = tk.e - tk.a - ml;
                const SahTask kids[2] = {SahTask{tk.a, tk.a + ml, tk.slot + 1, tk.depth + 1},
                                         SahTask{tk.a + ml, tk.e, tk.slot + ml, tk.depth + 1}};
                const unsigned counts[2] = {ml, mr};
                for (int k = 0; k < 2; k++)
                    if (counts[k] >= 2) (counts[k] > kSahSmall ? next : small).push_back(kids[k]);
            }
            SAH_CK(cudaStreamSynchronize(st));  // the host vectors of this level are read by the copies above
            level.swap(next);
        }
        if (!small.empty()) {
            SahTask* d_small = nullptr;
            SAH_CK(dupload(&d_small, small.data(), small.size(), st));
            const unsigned ns = (unsigned)small.size();
            k_sah_small<<<(ns + 127) / 128, 128, 0, st>>>(d_small, ns, perm, perm2, cen, blo, bhi, g.nodes);
            SAH_CK(cudaGetLastError());
            SAH_CK(cudaStreamSynchronize(st));
            cudaFree(d_small);
        }
        k_sah_leaf_tris<<<(n + 255) / 256, 256, 0, st>>>(d_tri, perm, n, g.tri);
        SAH_CK(cudaGetLastError());
        return cudaStreamSynchronize(st);
#undef SAH_CK
    };
    const cudaError_t e = run();
    cudaStreamSynchronize(st);
    void* bufs[] = {d_tri, blo, bhi, cen, perm, perm2, d_tasks, d_work, d_bins, d_splits, d_chunk_left,
                    d_left_off, d_right_off, d_which};
    for (void* b : bufs)
        if (b) cudaFree(b);
    return e;
}

int upload_geometry(upbp_ctx* c, const upbp_scene_desc* s, bool real, Geometry& g)
{
    std::vector<float4> tri, nrm;
    std::vector<int2> rec;
    for (uint32_t i = 0; i < s->triangle_count; i++) {
        const int m = s->tri_material[i];
        if ((s->materials[m].real != 0) != real) continue;
        const float* v = s->verts + 9 * (size_t)i;
        const float* n = s->normals + 12 * (size_t)i;
        tri.push_back(make_float4(v[0], v[1], v[2], 0.f));
        tri.push_back(make_float4(v[3] - v[0], v[4] - v[1], v[5] - v[2], 0.f));
        tri.push_back(make_float4(v[6] - v[0], v[7] - v[1], v[8] - v[2], 0.f));
        for (int k = 0; k < 4; k++) nrm.push_back(make_float4(n[3 * k], n[3 * k + 1], n[3 * k + 2], 0.f));
        rec.push_back(make_int2(m, s->tri_light[i]));
    }
    g.count = (unsigned)rec.size();
    // Spheres of this class.  The reference hands OptiX a box per sphere and
    // recovers centre and radius from it (intersector.cu:37-42); the same
    // round trip here gives the same floats.
    std::vector<float4> sph;
    std::vector<int> sph_mat;
    for (uint32_t i = 0; i < s->sphere_count; i++) {
        const int m = s->sph_material[i];
        if ((s->materials[m].real != 0) != real) continue;
        const float* q = s->spheres + 4 * (size_t)i;
        const float r = q[3];
        const float lo[3] = {q[0] - r, q[1] - r, q[2] - r}, hi[3] = {q[0] + r, q[1] + r, q[2] + r};
        float cen[3];
        for (int k = 0; k < 3; k++) cen[k] = lo[k] + .5f * (hi[k] - lo[k]);
        sph.push_back(make_float4(cen[0], cen[1], cen[2], (hi[0] - lo[0]) * .5f));
        sph_mat.push_back(m);
    }
    g.sph_count = (unsigned)sph.size();
    if (g.sph_count) {
        UPBP_CK(dupload(&g.spheres, sph.data(), sph.size(), c->st));
        UPBP_CK(dupload(&g.sph_mat, sph_mat.data(), sph_mat.size(), c->st));
    }
    UPBP_CK(dupload(&g.normals, nrm.data(), nrm.size(), c->st));
    UPBP_CK(dupload(&g.record, rec.data(), rec.size(), c->st));
    UPBP_CK(dalloc(&g.nodes, g.count > 1 ? g.count - 1 : 1));
    UPBP_CK(dalloc(&g.tri, 3 * (size_t)std::max(1u, g.count)));
    if (g.count > 0) {
        cudaEvent_t e0, e1;
        UPBP_CK(cudaEventCreate(&e0));
        UPBP_CK(cudaEventCreate(&e1));
        UPBP_CK(cudaEventRecord(e0, c->st));
        const cudaError_t be = build_scene_bvh(c, g, tri);
        float ms = 0.f;
        if (be == cudaSuccess && cudaEventRecord(e1, c->st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess)
            cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        UPBP_CK(be);
        c->ms_scene_bvh += ms;
    }
    UPBP_CK(cudaStreamSynchronize(c->st));
    return UPBP_OK;
}

int alloc_scratch(BuildScratch& sc, unsigned cap)
{
    cap = std::max(cap, 2u);
    sc.capacity = cap;
    UPBP_CK(dalloc(&sc.keys, cap));
    UPBP_CK(dalloc(&sc.keys_alt, cap));
    UPBP_CK(dalloc(&sc.vals, cap));
    UPBP_CK(dalloc(&sc.vals_alt, cap));
    UPBP_CK(dalloc(&sc.parent_internal, cap));
    UPBP_CK(dalloc(&sc.parent_leaf, cap));
    UPBP_CK(dalloc(&sc.flags, cap));
    UPBP_CK(dalloc(&sc.ord6, 6));
    cub::DoubleBuffer<unsigned> kb(sc.keys, sc.keys_alt), vb(sc.vals, sc.vals_alt);
    size_t bytes = 0;
    UPBP_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, (int)cap, 0, 30));
    sc.temp_bytes = bytes;
    UPBP_CK(cudaMalloc(&sc.temp, bytes));
    return UPBP_OK;
}

void free_ploc(PlocScratch& ps)
{
    if (ps.exec) cudaGraphExecDestroy(ps.exec);
    if (ps.capture) cudaStreamDestroy(ps.capture);
    void* b[] = {ps.cl[0], ps.cl[1], ps.leaf,       ps.nn,      ps.flag,    ps.tile_sum,
                 ps.node_box, ps.node_child, ps.node_place, ps.written, ps.order, ps.count};
    for (void* x : b)
        if (x) cudaFree(x);
    ps = PlocScratch{};
}

// Clustering scratch for cap leaves; on failure none (the beam map is then
// built as an LBVH).
void alloc_ploc(PlocScratch& ps, unsigned cap)
{
    free_ploc(ps);
    bool ok = dalloc(&ps.cl[0], 2 * (size_t)cap) == cudaSuccess && dalloc(&ps.cl[1], 2 * (size_t)cap) == cudaSuccess &&
              dalloc(&ps.leaf, 2 * (size_t)cap) == cudaSuccess &&
              dalloc(&ps.nn, cap) == cudaSuccess && dalloc(&ps.flag, cap) == cudaSuccess &&
              dalloc(&ps.tile_sum, cap / kPlocTile + 1) == cudaSuccess &&
              dalloc(&ps.node_box, 2 * (size_t)cap) == cudaSuccess && dalloc(&ps.node_child, cap) == cudaSuccess &&
              dalloc(&ps.node_place, cap) == cudaSuccess && dalloc(&ps.written, cap) == cudaSuccess &&
              dalloc(&ps.order, cap) == cudaSuccess && dalloc(&ps.count, kPcWords) == cudaSuccess;
    if (ok && cudaStreamCreateWithFlags(&ps.capture, cudaStreamNonBlocking) != cudaSuccess) ps.capture = nullptr;
    if (!ok) {
        cudaGetLastError();
        free_ploc(ps);
        return;
    }
    ps.capacity = cap;
}

void free_scratch(BuildScratch& sc)
{
    cudaFree(sc.keys);
    cudaFree(sc.keys_alt);
    cudaFree(sc.vals);
    cudaFree(sc.vals_alt);
    cudaFree(sc.parent_internal);
    cudaFree(sc.parent_leaf);
    cudaFree(sc.flags);
    cudaFree(sc.ord6);
    cudaFree(sc.temp);
    sc = BuildScratch{};
}

float relative_radius(float r, float scene_radius) { return r < 0.f ? -r * scene_radius : r; }

// Sort buffers for queue q (0 segment, 1 point) of at least n records.
int ensure_sort(upbp_ctx* c, int q, unsigned n)
{
    if (n <= c->sort_capacity[q]) return UPBP_OK;
    for (auto& b : c->d_sort[q]) {
        cudaFree(b);
        UPBP_CK(dalloc(&b, n));
    }
    c->sort_capacity[q] = n;
    cub::DoubleBuffer<unsigned> kb(c->d_sort[q][0], c->d_sort[q][1]), vb(c->d_sort[q][2], c->d_sort[q][3]);
    size_t bytes = 0;
    UPBP_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, (int)n, 0, 30));
    if (bytes > c->sort_temp_bytes) {
        cudaFree(c->d_sort_temp);
        UPBP_CK(cudaMalloc(&c->d_sort_temp, bytes));
        c->sort_temp_bytes = bytes;
    }
    return UPBP_OK;
}

// Sorts queue q's n records into Morton order; returns the order array.
int sort_queries(upbp_ctx* c, int q, unsigned n, const unsigned** order)
{
    *order = nullptr;
    if (n < 2) return UPBP_OK;
    if (ensure_sort(c, q, n) != UPBP_OK) return UPBP_ERR_CUDA;
    unsigned** b = c->d_sort[q];
    if (q == 0)
        PK(c).query_keys[1]<<<(n + 255) / 256, 256, 0, c->st>>>(c->slot, n, b[0], b[2]);
    else
        PK(c).query_keys[0]<<<(n + 255) / 256, 256, 0, c->st>>>(c->slot, n, b[0], b[2]);
    UPBP_CK(cudaGetLastError());
    cub::DoubleBuffer<unsigned> kb(b[0], b[1]), vb(b[2], b[3]);
    size_t tb = c->sort_temp_bytes;
    UPBP_CK(cub::DeviceRadixSort::SortPairs(c->d_sort_temp, tb, kb, vb, (int)n, 0, 30, c->st));
    *order = vb.Current();
    return UPBP_OK;
}

// Grows the chunked beam-map buffers (and the build scratch) to n chunks.
int ensure_chunks(upbp_ctx* c, unsigned n)
{
    if (n <= c->chunk_capacity && n <= c->sc.capacity) return UPBP_OK;
    const unsigned cap = std::max(n + n / 4, 1024u);
    if (cap > c->chunk_capacity) {
        cudaFree(c->d_chunks);
        cudaFree(c->d_beam_nodes);
        cudaFree(c->d_beam_qnodes);
        cudaFree(c->d_beam_seg);
        UPBP_CK(dalloc(&c->d_chunks, cap));
        UPBP_CK(dalloc(&c->d_beam_nodes, cap));
        UPBP_CK(dalloc(&c->d_beam_qnodes, cap));
        UPBP_CK(dalloc(&c->d_beam_seg, 3 * (size_t)cap));
        c->chunk_capacity = cap;
    }
    if (cap > c->sc.capacity) {
        UPBP_CK(cudaStreamSynchronize(c->st));
        free_scratch(c->sc);
        if (alloc_scratch(c->sc, cap) != UPBP_OK) return UPBP_ERR_CUDA;
    }
    return UPBP_OK;
}

// Largest range-query hit list (8 bytes per entry, 34 GB, allocated only
// when an iteration finds that many pairs); an iteration with more hits runs
// its searches in rounds, each ending with a drain of the longest queries
// in flight.  The evaluation's grid-stride index stays below 2^32.
constexpr size_t kMaxHits = (size_t(1) << 32) - (size_t(1) << 21);

// Room for n range-query hits (n + n/4, within 2^20 .. max_hits).  When
// the device has no room for that list, the pool's idle lists are freed and
// then ever smaller lists tried, down to 2^20 entries: the context's limit
// becomes the size obtained, and its searches run in more rounds.
int ensure_hits(upbp_ctx* c, size_t n)
{
    if (n <= c->hit_capacity || c->hit_capacity >= c->max_hits) return UPBP_OK;
    size_t cap = std::min<size_t>(std::max<size_t>(n + n / 4, 1u << 20), c->max_hits);
    c->hit_want = std::max(c->hit_want, cap);
    UPBP_CK(cudaStreamSynchronize(c->st));
    cudaFree(c->d_hit_qb);
    c->d_hit_qb = nullptr;
    c->hit_capacity = 0;
    bool pool_freed = false;
    for (;;) {
        const cudaError_t e = dalloc(&c->d_hit_qb, cap);
        if (e == cudaSuccess) break;
        if (e != cudaErrorMemoryAllocation) UPBP_CK(e);
        (void)cudaGetLastError();  // an allocation failure is not sticky
        if (!pool_freed) {
            hit_pool_release_idle(c->dev);
            pool_freed = true;
            continue;
        }
        if (cap <= (1u << 20)) UPBP_CK(e);
        cap = std::max<size_t>(cap / 2, 1u << 20);
        c->max_hits = cap;
    }
    c->hit_capacity = (unsigned)cap;
    return UPBP_OK;
}

}  // namespace

// ---- neighbour-set query without device allocation --------------------
// upbp_debug_query stages the queries, counts and ids in buffers it
// allocates and frees on every call.  Some callers cannot do that: a host
// application that gives the renderer a fixed device-memory budget at
// creation, or one whose other streams must not be stalled by the
// device-wide synchronisation cudaFree implies.  upbp_debug_query_static
// stages everything in one statically allocated device array instead.  The
// array is shared by every call in the process: two calls whose copies or
// kernels overlap on the GPU overwrite each other's data, so callers
// serialise them.
constexpr unsigned kStaticQueryMax = 4096;  // queries per call
constexpr unsigned kStaticIdsMax = 256;     // ids per query
constexpr size_t kStaticQueryBytes = (size_t)kStaticQueryMax * 8 * sizeof(float);
constexpr size_t kStaticCountBytes = (size_t)kStaticQueryMax * sizeof(unsigned);
constexpr size_t kStaticIdBytes = (size_t)kStaticQueryMax * kStaticIdsMax * sizeof(unsigned);
// About 4.2 MB; every GPU that loads the library holds it until exit.
static __device__ __align__(256) unsigned char g_query_scratch[kStaticQueryBytes + kStaticCountBytes + kStaticIdBytes];

extern "C" int upbp_create(const upbp_scene_desc* s, const upbp_config* cfg, upbp_ctx** out)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!s || !cfg || !out) return UPBP_ERR_ARGS;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            upbp_host::set_error("no CUDA device");
            return UPBP_ERR_NO_DEVICE;
        }
        if (s->material_count == 0 || s->medium_count == 0 || s->global_medium < 0 ||
            (uint32_t)s->global_medium >= s->medium_count) {
            upbp_host::set_error("scene has no materials or no valid global medium");
            return UPBP_ERR_SCENE;
        }
        for (uint32_t i = 0; i < s->triangle_count; i++)
            if (s->tri_material[i] < 0 || (uint32_t)s->tri_material[i] >= s->material_count) {
                upbp_host::set_error("triangle material index out of range");
                return UPBP_ERR_SCENE;
            }
        if (s->sphere_count > UPBP_MAX_SPHERES) {
            upbp_host::set_error("more than UPBP_MAX_SPHERES spheres");
            return UPBP_ERR_SCENE;
        }
        for (uint32_t i = 0; i < s->sphere_count; i++) {
            const float r = s->spheres[4 * (size_t)i + 3];
            if (s->sph_material[i] < 0 || (uint32_t)s->sph_material[i] >= s->material_count || !(r > 0.f) ||
                !std::isfinite(r)) {
                upbp_host::set_error("sphere with a material index out of range or a radius not positive");
                return UPBP_ERR_SCENE;
            }
        }
        int dev = 0;
        UPBP_CK(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) {
            upbp_host::set_error("device index beyond the library's limit of " + std::to_string(kMaxDevices));
            return UPBP_ERR_NO_DEVICE;
        }
        upbp_ctx* c = new upbp_ctx();
        c->cfg = *cfg;
        c->dev = dev;
        c->render_hash = render_fingerprint(s, cfg);
        {
            std::lock_guard<std::mutex> lk(g_hit_pool[dev].mu);
            g_hit_pool[dev].contexts++;
        }
        DeviceParams& P = c->P;
        UPBP_CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
        UPBP_CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_status), sizeof(unsigned)));
        *c->h_status = 0;
        UPBP_CK(cudaMallocHost(reinterpret_cast<void**>(&c->h_ploc), kPcWords * sizeof(unsigned)));
        {
            // Set-up of the no-allocation query (upbp_debug_query_static):
            // the static array's device address on this device.  Its host-side
            // symbol is only a stand-in and must never reach a kernel.
            void* ptr = nullptr;
            UPBP_CK(cudaGetSymbolAddress(&ptr, g_query_scratch));
            c->static_scratch = static_cast<unsigned char*>(ptr);
        }
        for (auto& slot : c->ev_ring)
            for (auto& e : slot) UPBP_CK(cudaEventCreate(&e));

        // scene records
        std::vector<DMaterial> mats(s->material_count);
        for (uint32_t i = 0; i < s->material_count; i++) {
            const upbp_material& m = s->materials[i];
            mats[i].diffuse = make_float3(m.diffuse[0], m.diffuse[1], m.diffuse[2]);
            mats[i].phong = make_float3(m.phong[0], m.phong[1], m.phong[2]);
            mats[i].phong_exponent = m.phong_exponent;
            mats[i].mirror = make_float3(m.mirror[0], m.mirror[1], m.mirror[2]);
            mats[i].ior = m.ior;
            mats[i].priority = m.priority;
            mats[i].real = m.real;
            mats[i].medium = m.medium;
        }
        std::vector<DMedium> meds(s->medium_count);
        for (uint32_t i = 0; i < s->medium_count; i++) init_medium(meds[i], s->media[i]);
        std::vector<DLight> lights(std::max(1u, s->light_count));
        for (uint32_t i = 0; i < s->light_count; i++) init_light(lights[i], s->lights[i]);
        if (s->env_rgb && s->background_light >= 0 && (uint32_t)s->background_light < s->light_count) {
            if (upload_env_map(c, s) != UPBP_OK) {
                upbp_destroy(c);
                return UPBP_ERR_CUDA;
            }
            lights[s->background_light].env = 1;
            lights[s->background_light].scale = s->lights[s->background_light].scale;
        }
        UPBP_CK(dupload(&c->d_mat, mats.data(), mats.size(), c->st));
        UPBP_CK(dupload(&c->d_med, meds.data(), meds.size(), c->st));
        UPBP_CK(dupload(&c->d_lights, lights.data(), lights.size(), c->st));
        P.materials = c->d_mat;
        P.material_count = (int)s->material_count;
        P.media = c->d_med;
        P.medium_count = (int)s->medium_count;
        P.global_medium = s->global_medium;
        P.lights = c->d_lights;
        P.light_count = (int)s->light_count;
        P.background_light = s->background_light;

        // camera and scene sphere (scene_loader.hpp:65-71)
        const upbp_host::CameraMatrices cm = upbp_host::camera_setup(s->camera, (float)cfg->res_x, (float)cfg->res_y);
        DCamera& cam = P.camera;
        cam.origin = make_float3(cm.origin[0], cm.origin[1], cm.origin[2]);
        cam.direction = make_float3(cm.direction[0], cm.direction[1], cm.direction[2]);
        cam.res_x = (float)cfg->res_x;
        cam.res_y = (float)cfg->res_y;
        std::memcpy(cam.raster_to_world, cm.raster_to_world, sizeof(cam.raster_to_world));
        std::memcpy(cam.world_to_raster, cm.world_to_raster, sizeof(cam.world_to_raster));
        cam.image_plane_dist = cm.image_plane_dist;
        cam.mat_id = s->camera.mat_id;
        cam.med_id = s->camera.med_id;
        {
            const float3 lo = make_float3(s->bbox_min[0], s->bbox_min[1], s->bbox_min[2]);
            const float3 hi = make_float3(s->bbox_max[0], s->bbox_max[1], s->bbox_max[2]);
            float r2 = dot(hi - lo, hi - lo);
            if (r2 == 0.f || r2 > kInfinity) r2 = 1.f;
            c->bbox_lo = lo;
            c->bbox_hi = hi;
            P.scene_center = (hi + lo) * .5f;
            P.scene_radius = std::sqrt(r2) * .5f;
            P.inv_radius_sqr = 1.f / (P.scene_radius * P.scene_radius);
            // largest coordinate magnitude the range queries see (scene and camera)
            const float3 co = cam.origin;
            const float mag = std::max(std::max(std::fabs(P.scene_center.x), std::fabs(P.scene_center.y)),
                                       std::fabs(P.scene_center.z)) + P.scene_radius;
            const float coord = std::max(mag, std::max(std::max(std::fabs(co.x), std::fabs(co.y)), std::fabs(co.z)));
            P.cull_eps = 1e-6f * coord;
            P.beam_cull_eps = 1e-4f * coord;
        }

        // configuration (renderer_init.cpp:681-925)
        const uint32_t flags = cfg->algorithm_flags;
        P.trace_light_paths = flags != 0;
        P.trace_camera_paths = flags != 0;
        P.do_bpt = (flags & kBpt) != 0;
        P.do_bb1d = (flags & kBb1d) != 0;
        P.do_bp2d = (flags & kBp2d) != 0;
        P.do_pb2d = (flags & kPb2d) != 0;
        P.do_pp3d = (flags & kPp3d) != 0;
        P.do_surf = (flags & kSurf) != 0;
        if (flags & kSpecularOnly) {
            P.trace_light_paths = 0;
            P.trace_camera_paths = 1;
            P.do_bpt = P.do_bb1d = P.do_bp2d = P.do_pb2d = P.do_pp3d = P.do_surf = 0;
        }
        P.connect_to_camera_from_surf = (flags & (kPrevious | kCompatible)) == 0;
        P.screen_pixel_count = cfg->res_x * cfg->res_y;
        const unsigned L = (unsigned)cfg->path_count_per_iter;
        P.light_subpath_count = L;
        c->bb1d_used = cfg->bb1d_used_light_subpath_count;
        if (c->bb1d_used < 0.f) c->bb1d_used = std::floor(-c->bb1d_used * (float)L);
        c->r0[0] = relative_radius(cfg->bb1d_radius_initial, P.scene_radius);
        c->r0[1] = relative_radius(cfg->bp2d_radius_initial, P.scene_radius);
        c->r0[2] = relative_radius(cfg->pb2d_radius_initial, P.scene_radius);
        c->r0[3] = relative_radius(cfg->pp3d_radius_initial, P.scene_radius);
        c->r0[4] = relative_radius(cfg->surf_radius_initial, P.scene_radius);

        const unsigned slots = cfg->max_path_length > 1 ? cfg->max_path_length - 1 : 1;
        const unsigned beams_per_path = cfg->max_path_length > 2 ? cfg->max_path_length - 2 : 0;
        unsigned beam_paths = 0;
        if (P.do_bb1d) beam_paths = std::max(beam_paths, (unsigned)c->bb1d_used);
        if (P.do_bp2d) beam_paths = std::max(beam_paths, L);
        c->vertex_capacity = L * slots;
        c->beam_capacity = beam_paths * beams_per_path;
        P.slots_per_path = slots;
        P.beam_capacity = c->beam_capacity;

        const bool merging = cfg->max_path_length > 1;
        P.build_bb1d = P.trace_light_paths && merging && P.do_bb1d;
        P.build_bp2d = P.trace_light_paths && merging && P.do_bp2d;
        P.build_pb2d = P.trace_light_paths && merging && P.do_pb2d;
        P.build_pp3d = P.trace_light_paths && merging && P.do_pp3d;
        P.build_surf = P.trace_light_paths && merging && P.do_surf;
        P.iteration_offset = cfg->iteration_offset;
        P.min_path_length = cfg->min_path_length;
        P.max_path_length = cfg->max_path_length;
        P.photon_beam_type = cfg->photon_beam_type;
        P.camera_beam_type = cfg->query_beam_type;
        P.subpath_count_bpt = float(P.do_bpt);
        P.subpath_count_bb1d = float(P.do_bb1d) * c->bb1d_used;
        P.subpath_count_bp2d = float(P.do_bp2d) * L;
        P.subpath_count_pb2d = float(P.do_pb2d) * L;
        P.subpath_count_pp3d = float(P.do_pp3d) * L;
        P.subpath_count_surf = float(P.do_surf) * L;
        P.ignore_fully_spec_paths = cfg->ignore_fully_spec_paths;
        P.estimator_techniques = flags;
        P.bb1d_used_light_subpath_count = (unsigned)c->bb1d_used;
        P.use_shading_normal = cfg->use_shading_normal;
        P.mis_exact = cfg->mis_exact != 0;
        P.res_x = cfg->res_x;
        P.res_y = cfg->res_y;

        // buffers
        unsigned n_real = 0, n_imag = 0;
        for (uint32_t i = 0; i < s->triangle_count; i++) (s->materials[s->tri_material[i]].real ? n_real : n_imag)++;
        c->triangles = s->triangle_count;
        if (alloc_scratch(c->sc, std::max({n_real, n_imag, c->vertex_capacity, c->beam_capacity})) != UPBP_OK) {
            upbp_destroy(c);
            return UPBP_ERR_CUDA;
        }
        if (upload_geometry(c, s, true, c->real) != UPBP_OK || upload_geometry(c, s, false, c->imag) != UPBP_OK) {
            upbp_destroy(c);
            return UPBP_ERR_CUDA;
        }
        P.real = TriView{BvhView{c->real.nodes, c->real.count}, c->real.tri, c->real.normals, c->real.record,
                         c->real.spheres, c->real.sph_mat, (int)c->real.sph_count};
        P.imag = TriView{BvhView{c->imag.nodes, c->imag.count}, c->imag.tri, c->imag.normals, c->imag.record,
                         c->imag.spheres, c->imag.sph_mat, (int)c->imag.sph_count};
        const size_t npx = (size_t)P.screen_pixel_count * 3;
        UPBP_CK(dalloc(&c->d_vertices, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_path_count, std::max(1u, L)));
        UPBP_CK(dalloc(&c->d_counters, 8));
        UPBP_CK(dalloc(&c->d_idx_s, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_idx_m, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_beams, c->beam_capacity));
        UPBP_CK(dalloc(&c->d_fb, npx));
        UPBP_CK(dalloc(&c->d_acc, npx));
        UPBP_CK(dalloc(&c->d_status, 1));
        if (cfg->gpu_assert) UPBP_CK(dalloc(&c->d_assert, kAssertCounts));
        UPBP_CK(dalloc(&c->d_work, (size_t)kKernRows * kCtrCount));
        UPBP_CK(dalloc(&c->d_qcount, 8));
        UPBP_CK(dalloc(&c->d_hit_state, 1));
        UPBP_CK(dalloc(&c->d_work_saved, kCtrCount));
        c->max_hits = kMaxHits;
        if (const char* e = std::getenv("UPBP_BEAM_MAP")) c->ploc_off = std::strcmp(e, "lbvh") == 0;
        if (const char* e = std::getenv("UPBP_PLOC_PASSES")) {
            const int v = std::atoi(e);
            if (v > 0) c->ploc_cap = std::min(v, kPlocPasses);
        }
        c->ploc_budget = c->ploc_cap;
        if (const char* e = std::getenv("UPBP_MAX_HITS")) {
            const long long v = std::atoll(e);
            if (v > 0) c->max_hits = std::min<size_t>((size_t)v, kMaxHits);
        }
        UPBP_CK(dalloc(&c->d_cam_fb, npx));
        {
            int sms = 0, per_sm = 0;
            UPBP_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const void* search[kRangeModes] = {(const void*)range_search_kernel<kModePb2d>,
                                               (const void*)range_search_kernel<kModeBb1d>,
                                               (const void*)range_search_kernel<kModeBp2d>};
            for (int m = 0; m < kRangeModes; m++) {
                UPBP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search[m], 128, 0));
                c->search_grid[m] = std::max(1, sms * std::max(1, per_sm));
            }
            const void* eval[kRangeModes] = {(const void*)range_eval_kernel<kModePb2d, false>,
                                             (const void*)range_eval_kernel<kModeBb1d, false>,
                                             (const void*)range_eval_kernel<kModeBp2d, false>};
            for (int m = 0; m < kRangeModes; m++) {
                UPBP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eval[m], 128, 0));
                c->eval_grid[m] = std::max(1, sms * std::max(1, per_sm));
            }
            UPBP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, camera_pass_kernel, 128, 0));
            c->camera_grid = std::max(1, sms * std::max(1, per_sm));
            UPBP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, light_pass_kernel, 128, 0));
            c->light_grid = std::max(1, sms * std::max(1, per_sm));
        }
        c->seg_capacity = std::max(1024u, 4 * P.screen_pixel_count);
        c->pt_capacity = std::max(1024u, 3 * P.screen_pixel_count);
        UPBP_CK(dalloc(&c->d_seg_queue, c->seg_capacity));
        UPBP_CK(dalloc(&c->d_pt_queue, c->pt_capacity));
        c->conn_capacity = std::max(1024u, 2 * P.screen_pixel_count);
        c->nee_capacity = std::max(1024u, 2 * P.screen_pixel_count);
        c->bpt_capacity = std::max(1024u, 2 * P.screen_pixel_count);
        UPBP_CK(dalloc(&c->d_conn, c->conn_capacity));
        UPBP_CK(dalloc(&c->d_nee, c->nee_capacity));
        UPBP_CK(dalloc(&c->d_bpt, c->bpt_capacity));
        UPBP_CK(dalloc(&c->d_nee_color, c->nee_capacity));
        UPBP_CK(dalloc(&c->d_bpt_color, c->bpt_capacity));
        UPBP_CK(dalloc(&c->d_path_err, P.screen_pixel_count));
        UPBP_CK(dalloc(&c->d_path_color, P.screen_pixel_count));
        UPBP_CK(dalloc(&c->d_surf_nodes, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_med_nodes, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_med_qnodes, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_surf_pos, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_med_pos, c->vertex_capacity));
        UPBP_CK(dalloc(&c->d_chunk_counts, c->beam_capacity));
        UPBP_CK(dalloc(&c->d_chunk_offsets, c->beam_capacity));
        {
            size_t bytes = 0;
            UPBP_CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, c->d_chunk_counts, c->d_chunk_offsets,
                                                  (int)std::max(1u, c->beam_capacity)));
            c->scan_temp_bytes = bytes;
            UPBP_CK(cudaMalloc(&c->d_scan_temp, std::max<size_t>(bytes, 16)));
        }
        if (ensure_chunks(c, std::max(1u, c->beam_capacity) * 4) != UPBP_OK) {
            upbp_destroy(c);
            return UPBP_ERR_CUDA;
        }
        UPBP_CK(cudaMemsetAsync(c->d_acc, 0, npx * sizeof(double), c->st));
        UPBP_CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->st));
        UPBP_CK(cudaMemsetAsync(c->d_path_count, 0, sizeof(unsigned) * std::max(1u, L), c->st));
        P.vertices = c->d_vertices;
        P.path_vertex_count = c->d_path_count;
        P.counters = c->d_counters;
        P.idx_surface = c->d_idx_s;
        P.idx_medium = c->d_idx_m;
        P.beams = c->d_beams;
        P.framebuffer = c->d_fb;
        P.status = c->d_status;
        P.assert_counts = c->d_assert;
        P.seg_queue = c->d_seg_queue;
        P.seg_capacity = c->seg_capacity;
        P.pt_queue = c->d_pt_queue;
        P.pt_capacity = c->pt_capacity;
        P.queue_count = c->d_qcount;
        P.conn_vertices = c->d_conn;
        P.conn_capacity = c->conn_capacity;
        P.nee_queue = c->d_nee;
        P.nee_capacity = c->nee_capacity;
        P.bpt_pairs = c->d_bpt;
        P.bpt_capacity = c->bpt_capacity;
        P.nee_color = c->d_nee_color;
        P.bpt_color = c->d_bpt_color;
        P.path_err = c->d_path_err;
        P.path_color = c->d_path_color;
        P.hit_state = c->d_hit_state;
        P.cam_fb = c->d_cam_fb;
        if (cfg->guide_train_iterations > 0) {
            GuideState& g = c->guide;
            g.train_iterations = cfg->guide_train_iterations;
            // media slots: every scattering medium, up to the one-hot width
            std::vector<int> slot(s->medium_count, -1);
            std::vector<float> med_g(s->medium_count, 0.f);
            for (uint32_t i = 0; i < s->medium_count; i++) {
                med_g[i] = meds[i].mean_cosine;
                if (meds[i].has_scattering && g.slots < kGuideMedia) slot[i] = g.slots++;
            }
            if (g.slots > 0) {
                const unsigned rows = 1u << 18;
                // cells per axis so that the table fits the batch buffers
                // (cells^3 x 64 direction bins x slots rows), at most 12
                g.cells = 12;
                while (g.cells > 2 && (unsigned)g.cells * g.cells * g.cells * g.dir_res * g.dir_res * g.slots > rows)
                    g.cells--;
                g.table_rows = (unsigned)g.cells * g.cells * g.cells * g.dir_res * g.dir_res * g.slots;
                const float3 ext = c->bbox_hi - c->bbox_lo;
                g.ext = make_float3(fmaxf(ext.x, 1e-3f), fmaxf(ext.y, 1e-3f), fmaxf(ext.z, 1e-3f));
                g.lo = c->bbox_lo;
                UPBP_CK(dupload(&g.medium_slot, slot.data(), slot.size(), c->st));
                UPBP_CK(dupload(&g.med_g, med_g.data(), med_g.size(), c->st));
                UPBP_CK(guide_alloc_net(g.net, c->st));
                std::vector<float> w0;
                guide_init_params(w0);
                UPBP_CK(guide_set_params(g.net, w0.data(), c->st));
                UPBP_CK(guide_alloc_batch(g.batch, rows, false));
                g.rec_capacity = 1u << 20;
                UPBP_CK(dalloc(&g.recs, g.rec_capacity));
                UPBP_CK(dalloc(&g.rec_count, 1));
                UPBP_CK(cudaMemsetAsync(g.rec_count, 0, sizeof(unsigned), c->st));
                for (auto& t : g.table) UPBP_CK(dalloc(&t, (size_t)g.table_rows * kGuideEntryWords));
                P.guide_recs = g.recs;
                P.guide_rec_count = g.rec_count;
                P.guide_rec_capacity = g.rec_capacity;
            } else {
                g.train_iterations = 0;  // no scattering medium to guide in
            }
        }
#ifdef UPBP_MIS_DEBUG
        {
            MisDebug& m = c->mis;
            m.max_verts = cfg->max_path_length + 1;
            m.light_paths = L;
            m.camera_paths = P.screen_pixel_count;
            m.event_capacity = 1u << 20;
            if (const char* e = std::getenv("UPBP_MIS_EVENTS")) m.event_capacity = (unsigned)std::max(1LL, std::atoll(e));
            UPBP_CK(dalloc(&m.light, (size_t)L * m.max_verts * kMisVtxWords));
            UPBP_CK(dalloc(&m.camera, (size_t)P.screen_pixel_count * m.max_verts * kMisVtxWords));
            UPBP_CK(dalloc(&m.events, (size_t)m.event_capacity * kMisEvWords));
            UPBP_CK(dalloc(&m.event_count, 1));
        }
#endif
        UPBP_CK(cudaStreamSynchronize(c->st));
        *out = c;
        return UPBP_OK;
    });
}

extern "C" int upbp_run_iteration(upbp_ctx* c, int iteration)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || iteration < 0) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        SlotLease lease(c->dev, c->slot, c->st);
        HitLease hits(c);
        DeviceParams& P = c->P;
        const upbp_config& cfg = c->cfg;
        const unsigned L = P.light_subpath_count;
        const size_t npx = (size_t)P.screen_pixel_count * 3;
        cudaEvent_t* ev = c->ev_ring[c->iterations % kEventRing];
        UPBP_CK(cudaEventRecord(ev[0], c->st));
        UPBP_CK(cudaMemsetAsync(c->d_fb, 0, npx * sizeof(float), c->st));
        UPBP_CK(cudaMemsetAsync(c->d_work, 0, (size_t)kKernCount * kCtrCount * sizeof(unsigned long long), c->st));
        UPBP_CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->st));  // this iteration's status bits
        if (c->d_assert) UPBP_CK(cudaMemsetAsync(c->d_assert, 0, kAssertCounts * sizeof(unsigned), c->st));
        unsigned launches = 0;
        size_t h2d = 0, d2h = 0;  // host<->device bytes of this iteration
        P.work = c->d_work;
#ifdef UPBP_MIS_DEBUG
        {
            const MisDebug& m = c->mis;
            UPBP_CK(cudaMemsetAsync(m.light, 0, (size_t)m.light_paths * m.max_verts * kMisVtxWords * sizeof(float4), c->st));
            UPBP_CK(cudaMemsetAsync(m.camera, 0, (size_t)m.camera_paths * m.max_verts * kMisVtxWords * sizeof(float4), c->st));
            UPBP_CK(cudaMemsetAsync(m.event_count, 0, sizeof(unsigned), c->st));
            UPBP_CK(cudaMemcpyToSymbolAsync(c_misdbg, &m, sizeof(m), 0, cudaMemcpyHostToDevice, c->st));
            UPBP_CK(upbp_kernels::slot0_upload_misdbg(&m, sizeof(m), c->st));
        }
#endif
        GuideState& gs = c->guide;
        const bool guide_training = gs.train_iterations > 0 && iteration < gs.train_iterations;
        {
            // the proposal table trained before this iteration began (none in
            // the first): both passes of the iteration read the same one
            GuideTable& t = P.guide;
            t = GuideTable{};
            if (gs.front >= 0) {
                const float3 cell = make_float3(gs.ext.x / gs.cells, gs.ext.y / gs.cells, gs.ext.z / gs.cells);
                t.entries = gs.table[gs.front];
                t.lo = gs.lo;
                t.inv_cell = make_float3(1.f / cell.x, 1.f / cell.y, 1.f / cell.z);
                t.cells = gs.cells;
                t.dir_res = gs.dir_res;
                t.slots = gs.slots;
                t.medium_slot = gs.medium_slot;
            }
            P.guide_collect = guide_training ? 1 : 0;
        }
        unsigned found[4] = {0, 0, 0, 0};
        if (P.trace_light_paths) {
            // radius schedule and MIS factors (renderer.cpp:57-119)
            const float eff = 1.f + (float)iteration;
            float r_bb1d = c->r0[0] * powf(1.f + (float)iteration * c->bb1d_used / (float)L, cfg.bb1d_radius_alpha - 1.f);
            r_bb1d = fmaxf(r_bb1d, 1e-7f);
            float r_bp2d = fmaxf(c->r0[1] * powf(eff, (cfg.bp2d_radius_alpha - 1.f) * .5f), 1e-7f);
            float r_pb2d = fmaxf(c->r0[2] * powf(eff, (cfg.pb2d_radius_alpha - 1.f) * .5f), 1e-7f);
            float r_pp3d = fmaxf(c->r0[3] * powf(eff, (cfg.pp3d_radius_alpha - 1.f) * (1.f / 3.f)), 1e-7f);
            float r_surf = fmaxf(c->r0[4] * powf(eff, (cfg.surf_radius_alpha - 1.f) * .5f), 1e-7f);
            P.mis_factor_bb1d = .5f * r_bb1d * P.subpath_count_bb1d;
            P.mis_factor_bp2d = (kPi * (r_bp2d * r_bp2d)) * P.subpath_count_bp2d;
            P.mis_factor_pb2d = (kPi * (r_pb2d * r_pb2d)) * P.subpath_count_pb2d;
            P.mis_factor_pp3d = (4.f / 3.f) * (kPi * (r_pp3d * r_pp3d * r_pp3d)) * P.subpath_count_pp3d;
            P.mis_factor_surf = (kPi * (r_surf * r_surf)) * P.subpath_count_surf;
            P.bb1d_normalization = 1.f / c->bb1d_used;
            P.bp2d_normalization = 1.f / (float)L;
            P.pb2d_normalization = 1.f / (float)L;
            P.pp3d_normalization = 1.f / P.mis_factor_pp3d;
            P.surf_normalization = 1.f / P.mis_factor_surf;
            P.radius_bb1d = r_bb1d;
            P.radius_bp2d = r_bp2d;
            P.radius_pb2d = r_pb2d;
            P.radius_pp3d = r_pp3d;
            P.radius_surf = r_surf;
            P.rad_point_med = 0.f;
            if (P.do_pp3d) P.rad_point_med = std::max(P.rad_point_med, r_pp3d);
            if (P.do_pb2d) P.rad_point_med = std::max(P.rad_point_med, r_pb2d);
            P.rad_beam = 0.f;
            if (P.do_bb1d) P.rad_beam = std::max(P.rad_beam, r_bb1d);
            if (P.do_bp2d) P.rad_beam = std::max(P.rad_beam, r_bp2d);
            P.radius_bb1d_2 = r_bb1d * r_bb1d;
            P.radius_bp2d_2 = r_bp2d * r_bp2d;
            P.radius_pb2d_2 = r_pb2d * r_pb2d;
            P.radius_pp3d_2 = r_pp3d * r_pp3d;
            P.radius_surf_2 = r_surf * r_surf;
            P.iteration = (unsigned)iteration;
            // [0] vertices [1] surface [2] medium [3] beams [4] next light path to hand out
            UPBP_CK(cudaMemsetAsync(c->d_counters, 0, 5 * sizeof(unsigned), c->st));
            h2d += sizeof(P);
            UPBP_CK(upload_params(c));
            if (L > 0) {
                PK(c).light_pass<<<cap_grid(c, std::min<unsigned>(c->light_grid, (L + 127) / 128)), 128, 0, c->st>>>(
                    c->slot);
                launches++;
            }
            UPBP_CK(cudaGetLastError());
            d2h += 4 * sizeof(unsigned);
            UPBP_CK(cudaMemcpyAsync(c->h_counters, c->d_counters, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
            UPBP_CK(cudaStreamSynchronize(c->st));
            std::memcpy(found, c->h_counters, sizeof(found));
            if (found[3] > c->beam_capacity) {
                // the reference prints the same warning and continues (renderer.cpp:188-195)
                std::fprintf(stderr, "error: device finds more beams than memory allocated\n");
            }
        } else {
            P.iteration = (unsigned)iteration;
        }
        UPBP_CK(cudaEventRecord(ev[13], c->st));
        if (guide_training) {
            // train on every record collected so far, then bake the network
            // into the back table, which the next iteration renders with
            for (int k = 0; k < gs.steps_per_iteration; k++)
                UPBP_CK(guide_train_step(c->st, gs, (unsigned)(iteration * gs.steps_per_iteration + k + 1)));
            const int back = gs.front == 0 ? 1 : 0;
            UPBP_CK(guide_fill_table(c->st, gs, gs.table[back]));
            UPBP_CK(cudaMemcpyAsync(gs.h_scal, gs.batch.scal, 3 * sizeof(float), cudaMemcpyDeviceToHost, c->st));
            UPBP_CK(cudaStreamSynchronize(c->st));
            if (reinterpret_cast<const unsigned&>(gs.h_scal[2]) != 0u) {
                upbp_host::set_error("learned proposal: a tensor-core chain of the training kernels did not complete");
                return UPBP_ERR_CUDA;
            }
            gs.last_loss = gs.h_scal[0] / (float)gs.batch.rows;
            gs.front_next = back;
            launches += gs.steps_per_iteration * 3 + 1;
        }
        UPBP_CK(cudaEventRecord(ev[1], c->st));

        // photon maps (renderer.cpp:206-307 builds OptiX structures here)
        const unsigned ns = std::min(found[1], c->vertex_capacity);
        const unsigned nm = std::min(found[2], c->vertex_capacity);
        const unsigned nb = std::min(found[3], c->beam_capacity);
        P.surf_map = PointMap{BvhView{c->d_surf_nodes, 0}, c->d_surf_pos};
        P.med_map = PointMap{BvhView{c->d_med_nodes, 0, c->d_med_qnodes}, c->d_med_pos};
        // beam-map boxes: the beam radius (BB1D and BP2D), the box tests' rounding
        // and the BB1D predicate's t1 error on nearly parallel lines
        const float beam_dilate = P.rad_beam * 1.0001f + P.beam_cull_eps;
        P.beam_map = BeamMap{BvhView{c->d_beam_nodes, 0, c->d_beam_qnodes}, c->d_beam_seg, beam_dilate};
        if (P.build_surf && ns > 0) {
            BoxSource src{};
            src.kind = 1;
            src.slots = c->d_idx_s;
            src.vertices = c->d_vertices;
            src.dilate = P.radius_surf * 1.0001f + P.cull_eps;
            const unsigned* order = nullptr;
            UPBP_CK(build_lbvh(src, ns, c->d_surf_nodes, c->sc, c->st, &order));
            k_gather_points<<<(ns + 255) / 256, 256, 0, c->st>>>(c->d_idx_s, c->d_vertices, order, ns, c->d_surf_pos);
            launches += (ns > 1 ? 4 : 2) + 1;
            P.surf_map.bvh.count = ns;
        }
        if ((P.build_pb2d || P.build_pp3d) && nm > 0) {
            BoxSource src{};
            src.kind = 1;
            src.slots = c->d_idx_m;
            src.vertices = c->d_vertices;
            src.dilate = P.rad_point_med * 1.0001f + P.cull_eps;  // PP3D and PB2D
            const unsigned* order = nullptr;
            UPBP_CK(build_lbvh(src, nm, c->d_med_nodes, c->sc, c->st, &order));
            k_gather_points<<<(nm + 255) / 256, 256, 0, c->st>>>(c->d_idx_m, c->d_vertices, order, nm, c->d_med_pos);
            if (nm > 1) k_quantize<<<(nm - 1 + 255) / 256, 256, 0, c->st>>>(c->d_med_nodes, (int)nm - 1, c->d_med_qnodes);
            launches += (nm > 1 ? 5 : 2) + 1;
            P.med_map.bvh.count = nm;
        }
        if ((P.build_bb1d || P.build_bp2d) && nb > 0) {
            // split beams into chunks of about 6 beam radii, at most 64 per beam
            const float chunk_len = 6.f * P.rad_beam;
            k_chunk_counts<<<(nb + 255) / 256, 256, 0, c->st>>>(c->d_beams, nb, chunk_len, 64u, c->d_chunk_counts);
            size_t tb = c->scan_temp_bytes;
            UPBP_CK(cub::DeviceScan::ExclusiveSum(c->d_scan_temp, tb, c->d_chunk_counts, c->d_chunk_offsets, (int)nb, c->st));
            unsigned tail[2] = {0, 0};
            d2h += 2 * sizeof(unsigned);
            UPBP_CK(cudaMemcpyAsync(&tail[0], c->d_chunk_offsets + nb - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
            UPBP_CK(cudaMemcpyAsync(&tail[1], c->d_chunk_counts + nb - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
            UPBP_CK(cudaStreamSynchronize(c->st));
            const unsigned nchunks = tail[0] + tail[1];
            if (ensure_chunks(c, nchunks) != UPBP_OK) return UPBP_ERR_CUDA;
            P.beam_map = BeamMap{BvhView{c->d_beam_nodes, 0, c->d_beam_qnodes}, c->d_beam_seg, beam_dilate};
            k_chunk_expand<<<(nb + 255) / 256, 256, 0, c->st>>>(c->d_chunk_counts, c->d_chunk_offsets, nb, c->d_chunks);
            BoxSource src{};
            src.kind = 3;
            src.beams = c->d_beams;
            src.chunks = c->d_chunks;
            src.dilate = beam_dilate;
            const unsigned* order = nullptr;
            bool clustered = false;
            if (!c->ploc_off && nchunks > c->ploc.capacity) {
                UPBP_CK(cudaStreamSynchronize(c->st));
                alloc_ploc(c->ploc, nchunks + nchunks / 4);
            }
            if (!c->ploc_off && nchunks >= 2 && nchunks <= c->ploc.capacity) {
                // the passes the last build needed and a margin: a build that
                // runs out falls back to the LBVH and the next gets them all
                const int budget = c->ploc_budget;
                UPBP_CK(build_ploc(src, nchunks, c->d_beam_nodes, c->sc, c->ploc, c->st, &order, &launches,
                                   c->h_ploc, budget));
                clustered = true;
                c->ploc_pending = true;  // checked after the camera pass's synchronisation
                c->ploc_src = src;
                c->ploc_n = nchunks;
            }
            if (!clustered) {
                c->beam_map_passes = 0;
                UPBP_CK(build_lbvh(src, nchunks, c->d_beam_nodes, c->sc, c->st, &order));
            }
            k_gather_chunks<<<(nchunks + 255) / 256, 256, 0, c->st>>>(c->d_chunks, c->d_beams, order, nchunks,
                                                                      P.bb1d_used_light_subpath_count, c->d_beam_seg);
            if (nchunks > 1)
                k_quantize<<<(nchunks - 1 + 255) / 256, 256, 0, c->st>>>(c->d_beam_nodes, (int)nchunks - 1,
                                                                         c->d_beam_qnodes);
            P.beam_map.bvh.count = nchunks;
            c->last_chunks = nchunks;
            launches += 3 + (nchunks > 1 ? 1 : 0) + (clustered ? 0 : (nchunks > 1 ? 4 : 2));
        }
        UPBP_CK(cudaGetLastError());
        P.n_surface = found[1];
        P.n_medium = found[2];
        P.n_beams = found[3];

        UPBP_CK(cudaMemsetAsync(c->d_cam_fb, 0, npx * sizeof(float), c->st));
        UPBP_CK(cudaEventRecord(ev[2], c->st));
        if (P.trace_camera_paths) {
            // extend: tracing, emitter hits, NEE and BPT sampling; queues the
            // range queries and the connections
            for (int attempt = 0; attempt < 2; attempt++) {
                // [0] segment queries [1] point queries [2] next pixel to hand out
                // [3] connection vertices [4] NEE samples [5] BPT pairs
                UPBP_CK(cudaMemsetAsync(c->d_qcount, 0, 6 * sizeof(unsigned), c->st));
                h2d += sizeof(P);
                UPBP_CK(upload_params(c));
                    UPBP_CK(cudaMemsetAsync(c->d_work + (size_t)kKernCameraExtend * kCtrCount, 0,
                                        kCtrCount * sizeof(unsigned long long), c->st));
                PK(c).camera_pass<<<cap_grid(c, std::min<unsigned>(c->camera_grid, (P.screen_pixel_count + 127) / 128)),
                                     128, 0, c->st>>>(c->slot);
                launches++;
                UPBP_CK(cudaGetLastError());
                d2h += 6 * sizeof(unsigned);
                UPBP_CK(cudaMemcpyAsync(c->h_qcount, c->d_qcount, 6 * sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
                UPBP_CK(cudaStreamSynchronize(c->st));
                const unsigned* q = c->h_qcount;
                if (q[0] <= c->seg_capacity && q[1] <= c->pt_capacity && q[3] <= c->conn_capacity &&
                    q[4] <= c->nee_capacity && q[5] <= c->bpt_capacity)
                    break;
                // a queue overflowed: grow it and render the camera pass again (the
                // pass is a pure function of the iteration, so the rerun is exact)
                unsigned nee_cap = c->nee_capacity, bpt_cap = c->bpt_capacity;
                if (grow(&c->d_seg_queue, c->seg_capacity, q[0]) != cudaSuccess ||
                    grow(&c->d_pt_queue, c->pt_capacity, q[1]) != cudaSuccess ||
                    grow(&c->d_conn, c->conn_capacity, q[3]) != cudaSuccess ||
                    grow(&c->d_nee, c->nee_capacity, q[4]) != cudaSuccess ||
                    grow(&c->d_bpt, c->bpt_capacity, q[5]) != cudaSuccess ||
                    grow(&c->d_nee_color, nee_cap, q[4]) != cudaSuccess ||
                    grow(&c->d_bpt_color, bpt_cap, q[5]) != cudaSuccess) {
                    upbp_host::set_error("camera-pass queue allocation failed");
                    return UPBP_ERR_CUDA;
                }
                P.seg_queue = c->d_seg_queue;
                P.seg_capacity = c->seg_capacity;
                P.pt_queue = c->d_pt_queue;
                P.pt_capacity = c->pt_capacity;
                P.conn_vertices = c->d_conn;
                P.conn_capacity = c->conn_capacity;
                P.nee_queue = c->d_nee;
                P.nee_capacity = c->nee_capacity;
                P.bpt_pairs = c->d_bpt;
                P.bpt_capacity = c->bpt_capacity;
                P.nee_color = c->d_nee_color;
                P.bpt_color = c->d_bpt_color;
                UPBP_CK(cudaMemsetAsync(c->d_cam_fb, 0, npx * sizeof(float), c->st));
            }
        }
        if (c->ploc_pending) {
            // the clustered beam map's outcome (copied before the camera pass,
            // which the host has waited for); an incomplete tree is replaced
            // by the LBVH before any search walks it
            c->ploc_pending = false;
            UPBP_CK(cudaStreamSynchronize(c->st));
            const unsigned n = c->ploc_n;
            if (ploc_complete(c->h_ploc, n)) {
                c->beam_map_passes = c->h_ploc[kPcPasses] + c->h_ploc[kPcTailIters];
                c->ploc_budget = std::min((int)c->h_ploc[kPcPasses] + 4, c->ploc_cap);
            } else {
                // replaced by the LBVH; a context whose builds run out of
                // passes even with all of them (boxes too alike to merge
                // fast) builds the LBVH from then on
                c->beam_map_passes = 0;
                if (c->ploc_budget >= c->ploc_cap && ++c->ploc_failures >= 2) c->ploc_off = true;
                c->ploc_budget = c->ploc_cap;
                const unsigned* order = nullptr;
                UPBP_CK(build_lbvh(c->ploc_src, n, c->d_beam_nodes, c->sc, c->st, &order));
                k_gather_chunks<<<(n + 255) / 256, 256, 0, c->st>>>(c->d_chunks, c->d_beams, order, n,
                                                                    P.bb1d_used_light_subpath_count, c->d_beam_seg);
                k_quantize<<<(n - 1 + 255) / 256, 256, 0, c->st>>>(c->d_beam_nodes, (int)n - 1, c->d_beam_qnodes);
                launches += 7;
            }
        }
        UPBP_CK(cudaEventRecord(ev[3], c->st));
        auto grid_for = [c](unsigned n) { return cap_grid(c, std::max(1u, std::min((n + 127) / 128, 148u * 64u))); };
        // deferred NEE and BPT connections, then the colours of every camera path
        // whose steps all succeeded (the query kernels below check the same)
        const unsigned nnee = P.trace_camera_paths ? std::min(c->h_qcount[4], c->nee_capacity) : 0;
        const unsigned nbpt = P.trace_camera_paths ? std::min(c->h_qcount[5], c->bpt_capacity) : 0;
        if (P.trace_camera_paths)
            UPBP_CK(cudaMemsetAsync(c->d_path_err, 0xff, P.screen_pixel_count * sizeof(unsigned), c->st));
        if (nnee > 0) {
            PK(c).nee_connect<<<grid_for(nnee), 128, 0, c->st>>>(c->slot);
            launches++;
        }
        UPBP_CK(cudaEventRecord(ev[4], c->st));
        if (nbpt > 0) {
            PK(c).bpt_connect<<<grid_for(nbpt), 128, 0, c->st>>>(c->slot);
            launches++;
        }
        if (P.trace_camera_paths) {
            PK(c).resolve_camera<<<std::max(1u, std::min((nnee + nbpt + P.screen_pixel_count + 255) / 256, 148u * 32u)), 256, 0,
                               c->st>>>(c->slot);
            launches++;
        }
        UPBP_CK(cudaGetLastError());
        UPBP_CK(cudaEventRecord(ev[5], c->st));
        const unsigned nseg = std::min(c->h_qcount[0], c->seg_capacity);
        const unsigned npt = std::min(c->h_qcount[1], c->pt_capacity);
        const bool run_pb2d = P.trace_camera_paths && P.build_pb2d && P.n_medium > 0 && nseg > 0;
        const bool run_bb1d = P.trace_camera_paths && P.build_bb1d && P.n_beams > 0 && nseg > 0;
        const bool run_surf = P.trace_camera_paths && P.build_surf && P.n_surface > 0 && npt > 0;
        const bool run_pp3d = P.trace_camera_paths && P.build_pp3d && P.n_medium > 0 && npt > 0;
        const bool run_bp2d = P.trace_camera_paths && P.build_bp2d && P.n_beams > 0 && npt > 0;
        // Morton order of the query records for coherent traversal
        {
            const unsigned* so = nullptr;
            const unsigned* po = nullptr;
            if ((run_pb2d || run_bb1d) && sort_queries(c, 0, nseg, &so) != UPBP_OK) return UPBP_ERR_CUDA;
            if ((run_surf || run_pp3d || run_bp2d) && sort_queries(c, 1, npt, &po) != UPBP_OK) return UPBP_ERR_CUDA;
            P.seg_order = so;
            P.pt_order = po;
            launches += (so ? 1 : 0) + (po ? 1 : 0);
            h2d += sizeof(P);
            UPBP_CK(upload_params(c));
        }
        // The estimators: search (query, neighbour) pairs into the hit list, then
        // evaluate them, in rounds over the query order.  A round stops handing
        // out queries when the list is 3/4 full; if the queries in flight then
        // overflow it, the round is repeated (the search is a pure function of
        // the queries and the map) with a larger list or a shorter range.  A list
        // that needed more than one round is grown for the next estimator and
        // iteration (up to max_hits).
        auto estimator = [&](int mode, unsigned nq) -> int {
            static constexpr int kKern[kRangeModes] = {kKernPb2d, kKernBb1d, kKernBp2d};
            unsigned long long* work = c->d_work + (size_t)kKern[mode] * kCtrCount;
            const size_t work_bytes = kCtrCount * sizeof(unsigned long long);
            if (c->hit_capacity == 0 && ensure_hits(c, (size_t)std::max(nseg, npt) * 32) != UPBP_OK) return UPBP_ERR_CUDA;
            UPBP_CK(cudaMemsetAsync(work, 0, work_bytes, c->st));
            unsigned long long found = 0;
            unsigned begin = 0, span = nq;  // span: longest range of a round, halved after an overflow
            int repeats = 0;
            while (begin < nq) {
                const unsigned end = begin + std::min(span, nq - begin);
                UPBP_CK(cudaMemsetAsync(c->d_hit_state, 0, sizeof(HitState), c->st));
                UPBP_CK(cudaMemcpyAsync(c->d_work_saved, work, work_bytes, cudaMemcpyDeviceToDevice, c->st));
                P.hit_qb = c->d_hit_qb;
                P.hit_capacity = c->hit_capacity;
                P.hit_soft_limit = c->hit_capacity - c->hit_capacity / 4;
                P.query_begin = begin;
                P.query_end = end;
                h2d += sizeof(P);
                UPBP_CK(upload_params(c));
                const int g = (int)cap_grid(c, (unsigned)c->search_grid[mode]);
                switch (mode) {
                case kModePb2d: PK(c).range_search[kModePb2d]<<<g, 128, 0, c->st>>>(c->slot); break;
                case kModeBb1d: PK(c).range_search[kModeBb1d]<<<g, 128, 0, c->st>>>(c->slot); break;
                default: PK(c).range_search[kModeBp2d]<<<g, 128, 0, c->st>>>(c->slot); break;
                }
                launches++;
                UPBP_CK(cudaGetLastError());
                d2h += sizeof(HitState);
                UPBP_CK(cudaMemcpyAsync(&c->h_hit_state, c->d_hit_state, sizeof(HitState), cudaMemcpyDeviceToHost, c->st));
                UPBP_CK(cudaStreamSynchronize(c->st));
                const unsigned long long total = c->h_hit_state.total;
                const unsigned done = (unsigned)std::min<unsigned long long>(c->h_hit_state.fetched, end - begin);
                if (total > c->hit_capacity || done == 0) {
                    if (++repeats > 64) {  // repeats of one round
                        upbp_host::set_error("range search made no progress");
                        return UPBP_ERR_CUDA;
                    }
                    UPBP_CK(cudaMemcpyAsync(work, c->d_work_saved, work_bytes, cudaMemcpyDeviceToDevice, c->st));
                    if (c->hit_capacity < c->max_hits) {
                        if (ensure_hits(c, (size_t)std::min<unsigned long long>(total, c->max_hits)) != UPBP_OK)
                            return UPBP_ERR_CUDA;
                    } else {
                        span = std::max(1u, std::min(done, end - begin) / 2);
                    }
                    continue;
                }
                if (total > 0) {
                    // no more blocks than are resident: the blocks then sweep
                    // the list once, side by side, and the records of the
                    // pairs in flight (neighbours in the list share queries
                    // and nearby beams) stay in L2; with more blocks every
                    // wave of resident blocks swept the whole list and read
                    // the records again
                    const unsigned g2 = cap_grid(
                        c, std::max(1u, std::min<unsigned>((unsigned)((total + 127) / 128), (unsigned)c->eval_grid[mode])));
                    const bool gd = P.guide.entries != nullptr;
                    switch (mode) {
                    case kModePb2d:
                        if (gd) PK(c).range_eval[kModePb2d][1]<<<g2, 128, 0, c->st>>>(c->slot);
                        else PK(c).range_eval[kModePb2d][0]<<<g2, 128, 0, c->st>>>(c->slot);
                        break;
                    case kModeBb1d:
                        if (gd) PK(c).range_eval[kModeBb1d][1]<<<g2, 128, 0, c->st>>>(c->slot);
                        else PK(c).range_eval[kModeBb1d][0]<<<g2, 128, 0, c->st>>>(c->slot);
                        break;
                    default:
                        if (gd) PK(c).range_eval[kModeBp2d][1]<<<g2, 128, 0, c->st>>>(c->slot);
                        else PK(c).range_eval[kModeBp2d][0]<<<g2, 128, 0, c->st>>>(c->slot);
                        break;
                    }
                    launches++;
                    UPBP_CK(cudaGetLastError());
                }
                found += total;
                begin += done;
                repeats = 0;
                span = span > nq / 2 ? nq : 2 * span;
            }
            if (found > c->hit_capacity - c->hit_capacity / 4 &&
                ensure_hits(c, (size_t)std::min<unsigned long long>(found + found / 8, c->max_hits)) != UPBP_OK)
                return UPBP_ERR_CUDA;
            return UPBP_OK;
        };
        UPBP_CK(cudaEventRecord(ev[6], c->st));
        if (run_surf) {
            if (P.guide.entries) PK(c).point_merge[0][1]<<<grid_for(npt), 128, 0, c->st>>>(c->slot);
            else PK(c).point_merge[0][0]<<<grid_for(npt), 128, 0, c->st>>>(c->slot);
            launches++;
        }
        UPBP_CK(cudaEventRecord(ev[7], c->st));
        if (run_pp3d) {
            if (P.guide.entries) PK(c).point_merge[1][1]<<<grid_for(npt), 128, 0, c->st>>>(c->slot);
            else PK(c).point_merge[1][0]<<<grid_for(npt), 128, 0, c->st>>>(c->slot);
            launches++;
        }
        UPBP_CK(cudaEventRecord(ev[8], c->st));
        if (run_bp2d && estimator(kModeBp2d, npt) != UPBP_OK) return UPBP_ERR_CUDA;
        UPBP_CK(cudaEventRecord(ev[9], c->st));
        if (run_pb2d && estimator(kModePb2d, nseg) != UPBP_OK) return UPBP_ERR_CUDA;
        UPBP_CK(cudaEventRecord(ev[10], c->st));
        if (run_bb1d && estimator(kModeBb1d, nseg) != UPBP_OK) return UPBP_ERR_CUDA;
        UPBP_CK(cudaEventRecord(ev[11], c->st));
        k_finish_iteration<<<(unsigned)((npx + 255) / 256), 256, 0, c->st>>>(c->d_fb, c->d_cam_fb, c->d_acc,
                                                                             (unsigned)npx);
        launches++;
        UPBP_CK(cudaEventRecord(ev[12], c->st));
        // the iteration's device status bits, returned as the reference's
        // run_iteration reports its failed paths (renderer.cpp:171-195)
        d2h += sizeof(unsigned);
        UPBP_CK(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
        c->launches = launches;
        c->h2d_iter = h2d;
        c->d2h_iter = d2h;
        UPBP_CK(cudaGetLastError());
        UPBP_CK(cudaStreamSynchronize(c->st));
        c->iterations++;
        c->ev_pending = std::min(c->ev_pending + 1, (unsigned)kEventRing);
        c->status_seen |= *c->h_status;
        if (c->d_assert) {
            // -assert: the reference's exception program prints a line per
            // event (kernel/exception.cu:27-52); here one per kind, counted
            static const char* const what[kAssertCounts] = {
                "assertion failed", "boundary_stack too small", "intersection_array too small",
                "vol_segment_array or vol_lite_segment_array too small", "intersection_stack too small",
                "beam buffer too small", "traversal stack too small"};
            unsigned counts[kAssertCounts];
            UPBP_CK(cudaMemcpy(counts, c->d_assert, sizeof(counts), cudaMemcpyDeviceToHost));
            for (int k = 0; k < kAssertCounts; k++)
                if (counts[k])
                    std::fprintf(stderr, "[ 5][            USER]: %s (%u times in iteration %d)\n", what[k], counts[k],
                                 iteration);
        }
        if (guide_training) gs.front = gs.front_next;
        return (int)*c->h_status;
    });
}

extern "C" int upbp_accumulate_to_host(upbp_ctx* c, float* rgb, double scale)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !rgb) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        const size_t n = (size_t)c->P.screen_pixel_count * 3;
        std::vector<double> tmp(n);
        UPBP_CK(cudaMemcpyAsync(tmp.data(), c->d_acc, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        UPBP_CK(cudaStreamSynchronize(c->st));
        for (size_t i = 0; i < n; i++) rgb[i] += (float)(scale * tmp[i]);
        return UPBP_OK;
    });
}

extern "C" int upbp_read_iteration(upbp_ctx* c, float* rgb)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !rgb) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        const size_t n = (size_t)c->P.screen_pixel_count * 3;
        UPBP_CK(cudaMemcpyAsync(rgb, c->d_fb, n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
        UPBP_CK(cudaStreamSynchronize(c->st));
        return UPBP_OK;
    });
}

extern "C" int upbp_get_stats(upbp_ctx* c, upbp_stats* o)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !o) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        std::memset(o, 0, sizeof(*o));
        UPBP_CK(cudaStreamSynchronize(c->st));
        const unsigned status = c->status_seen;
        o->light_vertices = c->h_counters[0];
        o->surface_vertices = c->h_counters[1];
        o->medium_vertices = c->h_counters[2];
        o->light_beams = c->h_counters[3];
        o->light_paths = c->P.light_subpath_count;
        o->camera_paths = c->P.screen_pixel_count;
        o->status = status;
        o->iterations_done = c->iterations;
        o->triangle_count = c->triangles;
        o->scene_radius = c->P.scene_radius;
        unsigned long long work[kKernCount * kCtrCount];
        UPBP_CK(cudaMemcpy(work, c->d_work, sizeof(work), cudaMemcpyDeviceToHost));
        for (int k = 0; k < kKernCount && k < UPBP_KERNEL_KINDS; k++)
            for (int i = 0; i < kCtrCount && i < 8; i++) o->work[k][i] = work[k * kCtrCount + i];
        for (int i = 0; i < kCtrCount && i < 8; i++) {
            o->work_light[i] = work[i];
            unsigned long long cam = 0;
            for (int k = 1; k < kKernCount; k++) cam += work[k * kCtrCount + i];
            o->work_camera[i] = cam;
        }
        o->segment_queries = c->h_qcount[0];
        o->point_queries = c->h_qcount[1];
        o->nee_samples = c->h_qcount[4];
        o->bpt_pairs = c->h_qcount[5];
        o->beam_chunks = c->last_chunks;
        o->radius[0] = c->P.radius_bb1d;
        o->radius[1] = c->P.radius_bp2d;
        o->radius[2] = c->P.radius_pb2d;
        o->radius[3] = c->P.radius_pp3d;
        o->radius[4] = c->P.radius_surf;
        o->radius[5] = c->P.rad_beam;
        o->h2d_bytes = (uint32_t)c->h2d_iter;
        o->d2h_bytes = (uint32_t)c->d2h_iter;
        o->kernel_launches = c->launches;
        o->ms_scene_bvh = c->ms_scene_bvh;
        o->beam_map_passes = c->beam_map_passes;
        // per-pass times: the last iteration, and sums over the iterations run
        // since the previous stats call (up to the event ring size)
        for (unsigned k = 0; k < c->ev_pending; k++) {
            cudaEvent_t* ev = c->ev_ring[(c->iterations - 1 - k) % kEventRing];
            float light, guide, build, cam;
            UPBP_CK(cudaEventElapsedTime(&light, ev[0], ev[13]));
            UPBP_CK(cudaEventElapsedTime(&guide, ev[13], ev[1]));
            UPBP_CK(cudaEventElapsedTime(&build, ev[1], ev[2]));
            UPBP_CK(cudaEventElapsedTime(&cam, ev[2], ev[12]));
            if (k == 0) {
                o->ms_light = light;
                o->ms_build = build;
                o->ms_camera = cam;
                o->ms_guide = guide;
            }
            o->ms_guide_sum += guide;
            o->ms_light_sum += light;
            o->ms_build_sum += build;
            o->ms_camera_sum += cam;
            for (const EvInterval& iv : kKindInterval) {
                float t;
                UPBP_CK(cudaEventElapsedTime(&t, ev[iv.from], ev[iv.to]));
                o->ms_kernel_sum[iv.kind] += t;
            }
            o->timed_iterations++;
        }
        c->ev_pending = 0;
        return UPBP_OK;
    });
}

extern "C" int upbp_debug_photons(upbp_ctx* c, int kind, float* out, uint32_t capacity, uint32_t* count)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !count || kind < 0 || kind > 2) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        UPBP_CK(cudaStreamSynchronize(c->st));
        if (kind < 2) {
            const PointMap& m = kind == 0 ? c->P.surf_map : c->P.med_map;
            *count = m.bvh.count;
            const unsigned n = std::min(m.bvh.count, capacity);
            if (out && n) UPBP_CK(cudaMemcpy(out, m.pos, n * sizeof(float4), cudaMemcpyDeviceToHost));
            return UPBP_OK;
        }
        const unsigned nb = std::min(c->h_counters[3], c->beam_capacity);
        *count = (c->P.build_bb1d || c->P.build_bp2d) ? nb : 0;
        const unsigned n = std::min(*count, capacity);
        if (out && n) {
            std::vector<BeamRec> tmp(n);
            UPBP_CK(cudaMemcpy(tmp.data(), c->d_beams, n * sizeof(BeamRec), cudaMemcpyDeviceToHost));
            for (unsigned i = 0; i < n; i++) {
                const float4 q0 = tmp[i].q[0], q1 = tmp[i].q[1], q3 = tmp[i].q[3];
                float* o = out + 8 * (size_t)i;
                o[0] = q0.x;
                o[1] = q0.y;
                o[2] = q0.z;
                o[3] = q0.w;
                o[4] = q1.x;
                o[5] = q1.y;
                o[6] = q1.z;
                std::memcpy(&o[7], &q3.z, 4);  // path index bits
            }
        }
        return UPBP_OK;
    });
}

// The static scene's BVH of one class of triangles (real 1, imaginary 0)
// as built on the device: nodes (16 words each) and the triangles in leaf
// order (12 floats each, v0.w the original index's bits).
extern "C" int upbp_debug_scene_bvh(upbp_ctx* c, int real, float* nodes, uint64_t node_capacity, float* tris,
                                    uint64_t tri_capacity, uint32_t* count)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !count) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        const Geometry& g = real ? c->real : c->imag;
        *count = g.count;
        UPBP_CK(cudaStreamSynchronize(c->st));
        const uint64_t nn = g.count > 1 ? (uint64_t)(g.count - 1) * 16 : 0, nt = (uint64_t)g.count * 12;
        if (nodes && nn) UPBP_CK(cudaMemcpy(nodes, g.nodes, std::min(nn, node_capacity) * sizeof(float),
                                            cudaMemcpyDeviceToHost));
        if (tris && nt) UPBP_CK(cudaMemcpy(tris, g.tri, std::min(nt, tri_capacity) * sizeof(float),
                                           cudaMemcpyDeviceToHost));
        return UPBP_OK;
    });
}

extern "C" int upbp_debug_query(upbp_ctx* c, int kind, const float* queries, uint32_t n, uint32_t* counts,
                                uint32_t* ids, uint32_t ids_per_query)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !queries || !counts || kind < 0 || kind > 4) return UPBP_ERR_ARGS;
        if (n == 0) return UPBP_OK;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        float* dq = nullptr;
        unsigned *dc = nullptr, *di = nullptr;
        UPBP_CK(dalloc(&dq, 8 * (size_t)n));
        UPBP_CK(dalloc(&dc, n));
        UPBP_CK(dalloc(&di, (size_t)n * std::max(1u, ids_per_query)));
        UPBP_CK(cudaMemcpyAsync(dq, queries, 8 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, c->st));
        c->P.work = c->d_work;  // the query counts into its own row (kKernDebug)
        SlotLease lease(c->dev, c->slot, c->st);
        UPBP_CK(upload_params(c));
        k_debug_query<<<(n + 127) / 128, 128, 0, c->st>>>(c->slot, kind, dq, n, dc, di, ids_per_query);
        UPBP_CK(cudaGetLastError());
        UPBP_CK(cudaMemcpyAsync(counts, dc, n * sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
        if (ids && ids_per_query)
            UPBP_CK(cudaMemcpyAsync(ids, di, (size_t)n * ids_per_query * sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
        UPBP_CK(cudaStreamSynchronize(c->st));
        cudaFree(dq);
        cudaFree(dc);
        cudaFree(di);
        return UPBP_OK;
    });
}

extern "C" int upbp_debug_query_static(upbp_ctx* c, int kind, const float* queries, uint32_t n, uint32_t* counts,
                                       uint32_t* ids, uint32_t ids_per_query)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !queries || !counts || kind < 0 || kind > 4) return UPBP_ERR_ARGS;
        if (n > kStaticQueryMax || ids_per_query > kStaticIdsMax) {
            upbp_host::set_error("upbp_debug_query_static: at most " + std::to_string(kStaticQueryMax) +
                                 " queries and " + std::to_string(kStaticIdsMax) + " ids per query");
            return UPBP_ERR_ARGS;
        }
        if (n == 0) return UPBP_OK;
        // the context's device, whose address of the array upbp_create
        // resolved; the kernel and copies run on the context's stream there
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        unsigned char* base = c->static_scratch;
        float* dq = reinterpret_cast<float*>(base);
        unsigned* dc = reinterpret_cast<unsigned*>(base + kStaticQueryBytes);
        unsigned* di = reinterpret_cast<unsigned*>(base + kStaticQueryBytes + kStaticCountBytes);
        const size_t id_bytes = (size_t)n * ids_per_query * sizeof(unsigned);
        UPBP_CK(cudaMemcpyAsync(dq, queries, 8 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, c->st));
        // the array keeps the previous call's ids; clear this call's id slots
        if (id_bytes) UPBP_CK(cudaMemsetAsync(di, 0, id_bytes, c->st));
        c->P.work = c->d_work;  // the query counts into its own row (kKernDebug)
        SlotLease lease(c->dev, c->slot, c->st);
        UPBP_CK(upload_params(c));
        k_debug_query<<<(n + 127) / 128, 128, 0, c->st>>>(c->slot, kind, dq, n, dc, di, ids_per_query);
        UPBP_CK(cudaGetLastError());
        UPBP_CK(cudaMemcpyAsync(counts, dc, n * sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
        if (ids && id_bytes) UPBP_CK(cudaMemcpyAsync(ids, di, id_bytes, cudaMemcpyDeviceToHost, c->st));
        UPBP_CK(cudaStreamSynchronize(c->st));
        return UPBP_OK;
    });
}

// MIS records of the last iteration (recording build, libupbp_b200_misdbg.so):
// which 0 light-subpath vertices, 1 camera-subpath vertices, 2 contributions,
// 3 a header of kMisHeader floats (layout in include/upbp.h).
constexpr int kMisHeader = 64;
extern "C" int upbp_debug_mis_records(upbp_ctx* c, int which, float* out, uint64_t capacity, uint64_t* count)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !count || which < 0 || which > 3) return UPBP_ERR_ARGS;
#ifndef UPBP_MIS_DEBUG
        (void)out;
        (void)capacity;
        *count = 0;
        upbp_host::set_error("MIS records are kept only by the recording build (libupbp_b200_misdbg.so)");
        return UPBP_ERR_ARGS;
#else
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        UPBP_CK(cudaStreamSynchronize(c->st));
        const MisDebug& m = c->mis;
        unsigned nev = 0;
        UPBP_CK(cudaMemcpy(&nev, m.event_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
        const unsigned kept = std::min(nev, m.event_capacity);
        if (which == 3) {
            const DeviceParams& P = c->P;
            float h[kMisHeader] = {};
            const float vals[] = {(float)m.max_verts, (float)m.light_paths, (float)m.camera_paths, (float)nev,
                                  (float)m.event_capacity, (float)kMisVtxWords, (float)kMisEvWords, (float)kMisSegs,
                                  P.camera.origin.x, P.camera.origin.y, P.camera.origin.z, P.camera.direction.x,
                                  P.camera.direction.y, P.camera.direction.z, P.camera.image_plane_dist,
                                  (float)P.res_x, (float)P.res_y, P.mis_factor_surf, P.mis_factor_pp3d,
                                  P.mis_factor_pb2d, P.mis_factor_bp2d, P.mis_factor_bb1d, P.subpath_count_bpt,
                                  (float)P.light_subpath_count, (float)P.photon_beam_type, (float)P.camera_beam_type,
                                  (float)P.light_count, (float)P.mis_exact, (float)P.connect_to_camera_from_surf,
                                  (float)P.max_path_length, (float)P.min_path_length, P.scene_radius};
            std::memcpy(h, vals, sizeof(vals));
            *count = kMisHeader;
            if (out) std::memcpy(out, h, sizeof(float) * std::min<uint64_t>(capacity, kMisHeader));
            return UPBP_OK;
        }
        const float4* src = which == 0 ? m.light : which == 1 ? m.camera : m.events;
        const uint64_t n4 = which == 0 ? (uint64_t)m.light_paths * m.max_verts * kMisVtxWords
                            : which == 1 ? (uint64_t)m.camera_paths * m.max_verts * kMisVtxWords
                                         : (uint64_t)kept * kMisEvWords;
        *count = 4 * n4;
        if (out && capacity) UPBP_CK(cudaMemcpy(out, src, sizeof(float) * std::min<uint64_t>(capacity, 4 * n4),
                                                cudaMemcpyDeviceToHost));
        return UPBP_OK;
#endif
    });
}

// State of the learned proposal: training iterations, Adam steps, last batch
// loss, records collected, table rows, cells per axis, direction bins per
// axis, media slots, table in use (-1 none).
extern "C" int upbp_guide_info(upbp_ctx* c, float* out, uint32_t n)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !out) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        const GuideState& g = c->guide;
        unsigned recs = 0;
        if (g.rec_count) {
            UPBP_CK(cudaStreamSynchronize(c->st));
            UPBP_CK(cudaMemcpy(&recs, g.rec_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
        }
        const float v[] = {(float)g.train_iterations, (float)g.net.steps, g.last_loss, (float)recs,
                           (float)g.table_rows, (float)g.cells, (float)g.dir_res, (float)g.slots, (float)g.front};
        for (uint32_t i = 0; i < n; i++) out[i] = i < sizeof(v) / sizeof(v[0]) ? v[i] : 0.f;
        return UPBP_OK;
    });
}

// One forward and backward pass of the proposal's network on given inputs,
// for checking the tensor-core training kernels against a float64 restatement.
extern "C" int upbp_guide_gradients(const float* params, uint32_t n_params, const float* x, const float* t,
                                    uint32_t rows, float* grads, float* outputs, float* loss)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!params || !x || !t || !grads || rows == 0) return UPBP_ERR_ARGS;
        if (n_params != (uint32_t)kGuideParams) {
            upbp_host::set_error("upbp_guide_gradients: the network has " + std::to_string(kGuideParams) +
                                 " parameters");
            return UPBP_ERR_ARGS;
        }
        cudaStream_t st = nullptr;
        UPBP_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        GuideNet net;
        GuideBatch b;
        int rc = UPBP_OK;
        auto run = [&]() -> int {
            UPBP_CK(guide_alloc_net(net, st));
            UPBP_CK(guide_set_params(net, params, st));
            UPBP_CK(guide_alloc_batch(b, rows, true));
            std::vector<__half> xh((size_t)rows * kGuideInPad);
            for (size_t i = 0; i < xh.size(); i++) xh[i] = __float2half(x[i]);
            UPBP_CK(cudaMemcpyAsync(b.X, xh.data(), xh.size() * sizeof(__half), cudaMemcpyHostToDevice, st));
            UPBP_CK(cudaMemcpyAsync(b.T, t, (size_t)rows * kGuideTargetWords * sizeof(float), cudaMemcpyHostToDevice,
                                    st));
            UPBP_CK(cudaMemsetAsync(b.scal, 0, 3 * sizeof(float), st));
            UPBP_CK(cudaMemsetAsync(net.grad, 0, kGuideParams * sizeof(float), st));
            k_guide_weight_sum<<<148, 256, 0, st>>>(b.T, rows, b.scal + 1);
            float* dout = nullptr;
            if (outputs) UPBP_CK(dalloc(&dout, (size_t)rows * kGuideOutPad));
            GuideTcArgs a = guide_tc_args(net, rows, b.scal);
            a.X = b.X;
            a.T = b.T;
            a.O = dout;
            const cudaError_t le = guide_tc_launch<kTcTrainRows>(st, a);
            if (le == cudaSuccess && outputs)
                UPBP_CK(cudaMemcpyAsync(outputs, dout, (size_t)rows * kGuideOutPad * sizeof(float),
                                        cudaMemcpyDeviceToHost, st));
            cudaStreamSynchronize(st);
            if (dout) cudaFree(dout);
            UPBP_CK(le);
            UPBP_CK(cudaMemcpyAsync(grads, net.grad, kGuideParams * sizeof(float), cudaMemcpyDeviceToHost, st));
            float scal[3];
            UPBP_CK(cudaMemcpyAsync(scal, b.scal, sizeof(scal), cudaMemcpyDeviceToHost, st));
            UPBP_CK(cudaStreamSynchronize(st));
            if (reinterpret_cast<const unsigned&>(scal[2]) != 0u) {
                upbp_host::set_error("upbp_guide_gradients: a tensor-core chain did not complete");
                return UPBP_ERR_CUDA;
            }
            if (loss) *loss = scal[0];
            return UPBP_OK;
        };
        rc = run();
        cudaStreamSynchronize(st);
        guide_free_net(net);
        guide_free_batch(b);
        cudaStreamDestroy(st);
        return rc;
    });
}

// ---------------------------------------------------------------- checkpoints
//
// File: "UPBPCKP1", u32 version 1, u64 render fingerprint, u32 iterations
// rendered, u32 status bits seen, u32 width, u32 height, then width x height
// x 3 doubles of the accumulation; then i32 1 if the learned proposal's
// state follows: i32 Adam steps, i32 table in use (-1 none), f32 last loss,
// u32 training records, kGuideParams floats each of the parameters and the
// two Adam moments, the records (8 floats each).  Little-endian, as the
// machines that write and read them.
namespace {
constexpr char kCkptMagic[8] = {'U', 'P', 'B', 'P', 'C', 'K', 'P', '1'};

struct FileCloser {
    FILE* f;
    ~FileCloser()
    {
        if (f) std::fclose(f);
    }
};
}  // namespace

extern "C" int upbp_save_checkpoint(upbp_ctx* c, const char* path)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !path) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        UPBP_CK(cudaStreamSynchronize(c->st));
        const size_t n = (size_t)c->P.screen_pixel_count * 3;
        std::vector<double> acc(n);
        UPBP_CK(cudaMemcpy(acc.data(), c->d_acc, n * sizeof(double), cudaMemcpyDeviceToHost));
        const GuideState& g = c->guide;
        const int32_t has_guide = g.net.w32 ? 1 : 0;
        std::vector<float> w, m, v;
        std::vector<GuideRecord> recs;
        unsigned nrec = 0;
        if (has_guide) {
            w.resize(kGuideParams);
            m.resize(kGuideParams);
            v.resize(kGuideParams);
            UPBP_CK(cudaMemcpy(w.data(), g.net.w32, kGuideParams * sizeof(float), cudaMemcpyDeviceToHost));
            UPBP_CK(cudaMemcpy(m.data(), g.net.m, kGuideParams * sizeof(float), cudaMemcpyDeviceToHost));
            UPBP_CK(cudaMemcpy(v.data(), g.net.v, kGuideParams * sizeof(float), cudaMemcpyDeviceToHost));
            UPBP_CK(cudaMemcpy(&nrec, g.rec_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
            nrec = std::min(nrec, g.rec_capacity);
            recs.resize(nrec);
            if (nrec)
                UPBP_CK(cudaMemcpy(recs.data(), g.recs, nrec * sizeof(GuideRecord), cudaMemcpyDeviceToHost));
        }
        FileCloser fc{std::fopen(path, "wb")};
        if (!fc.f) {
            upbp_host::set_error(std::string("cannot write ") + path);
            return UPBP_ERR_IO;
        }
        const uint32_t head[5] = {1u, c->iterations, c->status_seen, c->cfg.res_x, c->cfg.res_y};
        bool ok = std::fwrite(kCkptMagic, 1, 8, fc.f) == 8 && std::fwrite(head, 4, 1, fc.f) == 1 &&
                  std::fwrite(&c->render_hash, 8, 1, fc.f) == 1 && std::fwrite(head + 1, 4, 4, fc.f) == 4 &&
                  std::fwrite(acc.data(), sizeof(double), n, fc.f) == n && std::fwrite(&has_guide, 4, 1, fc.f) == 1;
        if (ok && has_guide) {
            const int32_t gi[2] = {g.net.steps, g.front};
            ok = std::fwrite(gi, 4, 2, fc.f) == 2 && std::fwrite(&g.last_loss, 4, 1, fc.f) == 1 &&
                 std::fwrite(&nrec, 4, 1, fc.f) == 1 &&
                 std::fwrite(w.data(), 4, kGuideParams, fc.f) == (size_t)kGuideParams &&
                 std::fwrite(m.data(), 4, kGuideParams, fc.f) == (size_t)kGuideParams &&
                 std::fwrite(v.data(), 4, kGuideParams, fc.f) == (size_t)kGuideParams &&
                 std::fwrite(recs.data(), sizeof(GuideRecord), nrec, fc.f) == nrec;
        }
        if (!ok) {
            upbp_host::set_error(std::string("short write to ") + path);
            return UPBP_ERR_IO;
        }
        return UPBP_OK;
    });
}

extern "C" int upbp_load_checkpoint(upbp_ctx* c, const char* path)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!c || !path) return UPBP_ERR_ARGS;
        DeviceGuard dg(c->dev);
        UPBP_CK(dg.error());
        FileCloser fc{std::fopen(path, "rb")};
        if (!fc.f) {
            upbp_host::set_error(std::string("cannot read ") + path);
            return UPBP_ERR_IO;
        }
        auto bad = [&](const std::string& why) {
            upbp_host::set_error(std::string(path) + ": " + why);
            return UPBP_ERR_ARGS;
        };
        char magic[8];
        uint32_t version = 0, head[4];
        uint64_t hash = 0;
        if (std::fread(magic, 1, 8, fc.f) != 8 || std::memcmp(magic, kCkptMagic, 8) != 0) return bad("not a checkpoint");
        if (std::fread(&version, 4, 1, fc.f) != 1 || version != 1) return bad("unknown checkpoint version");
        if (std::fread(&hash, 8, 1, fc.f) != 1 || std::fread(head, 4, 4, fc.f) != 4) return bad("truncated header");
        if (hash != c->render_hash)
            return bad("written by a render of another scene or configuration (fingerprint differs)");
        if (head[2] != c->cfg.res_x || head[3] != c->cfg.res_y) return bad("resolution differs");
        const size_t n = (size_t)c->P.screen_pixel_count * 3;
        std::vector<double> acc(n);
        int32_t has_guide = 0;
        if (std::fread(acc.data(), sizeof(double), n, fc.f) != n || std::fread(&has_guide, 4, 1, fc.f) != 1)
            return bad("truncated accumulation");
        GuideState& g = c->guide;
        if ((has_guide != 0) != (g.net.w32 != nullptr)) return bad("learned-proposal state does not match");
        std::vector<float> w, m, v;
        std::vector<GuideRecord> recs;
        int32_t gi[2] = {0, -1};
        float last_loss = 0.f;
        unsigned nrec = 0;
        if (has_guide) {
            w.resize(kGuideParams);
            m.resize(kGuideParams);
            v.resize(kGuideParams);
            if (std::fread(gi, 4, 2, fc.f) != 2 || std::fread(&last_loss, 4, 1, fc.f) != 1 ||
                std::fread(&nrec, 4, 1, fc.f) != 1 || nrec > g.rec_capacity ||
                std::fread(w.data(), 4, kGuideParams, fc.f) != (size_t)kGuideParams ||
                std::fread(m.data(), 4, kGuideParams, fc.f) != (size_t)kGuideParams ||
                std::fread(v.data(), 4, kGuideParams, fc.f) != (size_t)kGuideParams)
                return bad("truncated learned-proposal state");
            recs.resize(nrec);
            if (std::fread(recs.data(), sizeof(GuideRecord), nrec, fc.f) != nrec) return bad("truncated records");
        }
        UPBP_CK(cudaStreamSynchronize(c->st));
        UPBP_CK(cudaMemcpy(c->d_acc, acc.data(), n * sizeof(double), cudaMemcpyHostToDevice));
        if (has_guide) {
            UPBP_CK(guide_set_params(g.net, w.data(), c->st));
            UPBP_CK(cudaMemcpy(g.net.m, m.data(), kGuideParams * sizeof(float), cudaMemcpyHostToDevice));
            UPBP_CK(cudaMemcpy(g.net.v, v.data(), kGuideParams * sizeof(float), cudaMemcpyHostToDevice));
            g.net.steps = gi[0];
            g.last_loss = last_loss;
            UPBP_CK(cudaMemcpy(g.rec_count, &nrec, sizeof(unsigned), cudaMemcpyHostToDevice));
            if (nrec) UPBP_CK(cudaMemcpy(g.recs, recs.data(), nrec * sizeof(GuideRecord), cudaMemcpyHostToDevice));
            g.front = -1;
            g.front_next = -1;
            if (gi[1] >= 0) {
                // the table in use is the bake of the network as saved
                UPBP_CK(guide_fill_table(c->st, g, g.table[0]));
                UPBP_CK(cudaStreamSynchronize(c->st));
                g.front = 0;
                g.front_next = 0;
            }
        }
        c->iterations = head[0];
        c->status_seen = head[1];
        c->ev_pending = 0;
        return UPBP_OK;
    });
}

extern "C" int upbp_set_grid_limit(upbp_ctx* c, uint32_t max_blocks)
{
    if (!c) return UPBP_ERR_ARGS;
    c->grid_limit = max_blocks;
    return UPBP_OK;
}

// Batched rendering: one iteration of many contexts (jobs), each driven on
// its own stream and parameter slot by one of `workers` host threads, so the
// jobs' kernels and host synchronisations overlap instead of queueing.
extern "C" int upbp_run_batch(upbp_ctx* const* ctxs, uint32_t n, int iteration, int workers)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!ctxs || n == 0 || iteration < 0) return UPBP_ERR_ARGS;
        for (uint32_t i = 0; i < n; i++)
            if (!ctxs[i]) return UPBP_ERR_ARGS;
        const unsigned w = (unsigned)std::max(1, std::min<int>(workers > 0 ? workers : 16, (int)n));
        // Range-query hit lists: up to w of them are in use at once (one per
        // worker, from the device's pool), each growing toward its job's
        // need.  Each worker's list is held to an even share of half the
        // device memory that is free or idle in the pool; a job that needs
        // more runs its searches in rounds.  The contexts' own limits are
        // restored afterwards.
        std::vector<size_t> saved_max(n);
        {
            const int dev = ctxs[0]->dev;
            DeviceGuard dg(dev);
            UPBP_CK(dg.error());
            size_t free_b = 0, total_b = 0;
            UPBP_CK(cudaMemGetInfo(&free_b, &total_b));
            size_t idle_b = 0;
            {
                std::lock_guard<std::mutex> lk(g_hit_pool[dev].mu);
                for (auto& h : g_hit_pool[dev].idle) idle_b += (size_t)h.second * sizeof(uint2);
            }
            const size_t share = std::max<size_t>((free_b + idle_b) / 2 / w / sizeof(uint2), 1u << 20);
            for (uint32_t i = 0; i < n; i++) {
                saved_max[i] = ctxs[i]->max_hits;
                if (ctxs[i]->dev == dev) ctxs[i]->max_hits = std::min(ctxs[i]->max_hits, share);
            }
        }
        struct Restore {
            upbp_ctx* const* c;
            std::vector<size_t>& m;
            ~Restore()
            {
                for (size_t i = 0; i < m.size(); i++) c[i]->max_hits = m[i];
            }
        } restore{ctxs, saved_max};
        std::atomic<uint32_t> next{0};
        std::atomic<unsigned> status{0};
        std::mutex mu;
        int err = UPBP_OK;
        std::string msg;
        auto work = [&]() {
            for (;;) {
                const uint32_t j = next.fetch_add(1);
                if (j >= n) return;
                const int rc = upbp_run_iteration(ctxs[j], iteration);
                if (rc < 0) {
                    std::lock_guard<std::mutex> lk(mu);
                    if (err == UPBP_OK) {
                        err = rc;
                        msg = std::string("job ") + std::to_string(j) + ": " + upbp_last_error();
                    }
                } else {
                    status.fetch_or((unsigned)rc);
                }
            }
        };
        std::vector<std::thread> pool;
        for (unsigned k = 1; k < w; k++) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        if (err != UPBP_OK) {
            upbp_host::set_error(msg);
            return err;
        }
        return (int)status.load();
    });
}

extern "C" void* upbp_get_stream(upbp_ctx* c) { return c ? (void*)c->st : nullptr; }

extern "C" int upbp_get_device(const upbp_ctx* c) { return c ? c->dev : UPBP_ERR_ARGS; }

extern "C" void upbp_destroy(upbp_ctx* c)
{
    if (!c) return;
    DeviceGuard dg(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->h_ploc) cudaFreeHost(c->h_ploc);
    void* bufs[] = {c->d_assert, c->mis.light, c->mis.camera, c->mis.events, c->mis.event_count, c->d_mat, c->d_med, c->d_lights, c->real.nodes, c->real.tri, c->real.normals, c->real.record,
                    c->d_env_img, c->d_env_dist, c->d_env_row_int, c->real.spheres, c->real.sph_mat, c->imag.spheres, c->imag.sph_mat,
                    c->imag.nodes, c->imag.tri, c->imag.normals, c->imag.record, c->d_vertices, c->d_path_count,
                    c->d_counters, c->d_idx_s, c->d_idx_m, c->d_beams, c->d_fb, c->d_acc, c->d_status,
                    c->d_surf_nodes, c->d_med_nodes, c->d_beam_nodes, c->d_med_qnodes, c->d_beam_qnodes, c->d_surf_pos, c->d_med_pos, c->d_beam_seg,
                    c->d_chunk_counts, c->d_chunk_offsets, c->d_chunks, c->d_scan_temp, c->d_work,
                    c->d_qcount, c->d_conn, c->d_nee, c->d_bpt, c->d_nee_color, c->d_bpt_color,
                    c->d_path_err, c->d_path_color, c->d_hit_state, c->d_work_saved, c->d_hit_qb, c->d_cam_fb, c->d_seg_queue, c->d_pt_queue, c->d_sort[0][0], c->d_sort[0][1],
                    c->d_sort[0][2], c->d_sort[0][3], c->d_sort[1][0], c->d_sort[1][1], c->d_sort[1][2],
                    c->d_sort[1][3], c->d_sort_temp};
    for (void* b : bufs)
        if (b) cudaFree(b);
    free_scratch(c->sc);
    free_ploc(c->ploc);
    {
        GuideState& g = c->guide;
        guide_free_net(g.net);
        guide_free_batch(g.batch);
        void* p[] = {g.recs, g.rec_count, g.table[0], g.table[1], g.medium_slot, g.med_g};
        for (void* x : p)
            if (x) cudaFree(x);
    }
    for (auto& slot : c->ev_ring)
        for (auto& e : slot)
            if (e) cudaEventDestroy(e);
    if (c->st) cudaStreamDestroy(c->st);
    bool last = false;
    {
        std::lock_guard<std::mutex> lk(g_hit_pool[c->dev].mu);
        last = --g_hit_pool[c->dev].contexts == 0;
    }
    if (last) hit_pool_release_idle(c->dev);
    delete c;
}
