// Host side of the learned proposal (kernels in upbp_guide.cuh and
// upbp_guide_tc.cuh): network state, the training step (batch weight sum,
// the fused tcgen05 forward / loss / backward kernel, Adam) on the context's
// stream, and the table the render kernels read.  Included by upbp_capi.cu after its
// allocation and error-check helpers.
#pragma once

#include <random>

#include "upbp_guide_tc.cuh"

namespace {

struct GuideNet {
    float* w32 = nullptr;    // FP32 master weights then biases (kGuideParams)
    float* m = nullptr;      // Adam moments
    float* v = nullptr;
    float* grad = nullptr;   // gradient sums of one batch
    __half* w16 = nullptr;   // FP16 weights the GEMMs read (kGuideWeights)
    int steps = 0;           // Adam steps taken
};

// Buffers of one training step: the batch's own rows exist only in the
// fused kernel's shared memory; X and T hold given rows (the gradient check
// entry point).
struct GuideBatch {
    unsigned rows = 0;
    __half* X = nullptr;      // rows x kGuideInPad, given rows only
    float* T = nullptr;       // rows x kGuideTargetWords: direction, weight, phase pdf; given rows only
    float* scal = nullptr;    // [0] weighted loss sum [1] weight sum [2] error bits (unsigned)
};

struct GuideState {
    int train_iterations = 0;   // iterations whose light records train the network
    int steps_per_iteration = 4;
    GuideNet net;
    GuideBatch batch;
    GuideRecord* recs = nullptr;
    unsigned* rec_count = nullptr;
    unsigned rec_capacity = 0;
    // two tables: an iteration renders with the one trained before it began,
    // training after its light pass writes the other
    float4* table[2] = {nullptr, nullptr};
    int front = -1;             // table in use (-1: none yet)
    int* medium_slot = nullptr;
    float* med_g = nullptr;
    int slots = 0, cells = 12, dir_res = 8;
    unsigned table_rows = 0;
    float3 lo{}, ext{};
    float last_loss = 0.f;
    float h_scal[3] = {0.f, 0.f, 0.f};
    int front_next = -1;        // table the last training step filled
};

cudaError_t guide_alloc_batch(GuideBatch& b, unsigned rows, bool given_rows)
{
    b.rows = rows;
    cudaError_t e;
    if (given_rows) {
        if ((e = dalloc(&b.X, (size_t)rows * kGuideInPad)) != cudaSuccess) return e;
        if ((e = dalloc(&b.T, (size_t)kGuideTargetWords * rows)) != cudaSuccess) return e;
    }
    return dalloc(&b.scal, 3);
}

void guide_free_batch(GuideBatch& b)
{
    void* p[] = {b.X, b.T, b.scal};
    for (void* x : p)
        if (x) cudaFree(x);
    b = GuideBatch{};
}

// Initial weights: He-normal for the hidden layers, a small output layer
// (the mixture starts nearly uniform), zero biases; a fixed seed.
void guide_init_params(std::vector<float>& w)
{
    w.assign(kGuideParams, 0.f);
    std::mt19937 rng(1234567u);
    for (int l = 0; l < kGuideLayers; l++) {
        const float sd = l == kGuideLayers - 1 ? 0.01f : std::sqrt(2.f / (float)kGuideLayerIn[l]);
        std::normal_distribution<float> nd(0.f, sd);
        for (int i = kGuideWOff[l]; i < kGuideWOff[l + 1]; i++) w[i] = nd(rng);
    }
    // mean directions need a nonzero start: spread the 8 lobes over the sphere
    // through the output biases of the mean components
    const float dirs[kGuideLobes][3] = {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {1, -1, -1},
                                        {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
    float* b4 = w.data() + kGuideWeights + kGuideBOff[3];
    for (int j = 0; j < kGuideLobes; j++) {
        for (int k = 0; k < 3; k++) b4[kGuideLobes + 3 * j + k] = dirs[j][k] * 0.577f;
        b4[4 * kGuideLobes + j] = std::log(2.f);  // kappa 2
    }
    // selection probability 0.5 to begin with
    b4[kGuideAlphaCol] = std::log(0.5f / kGuideAlphaMax / (1.f - 0.5f / kGuideAlphaMax));
}

cudaError_t guide_alloc_net(GuideNet& n, cudaStream_t st)
{
    cudaError_t e;
    if ((e = dalloc(&n.w32, kGuideParams)) != cudaSuccess) return e;
    if ((e = dalloc(&n.m, kGuideParams)) != cudaSuccess) return e;
    if ((e = dalloc(&n.v, kGuideParams)) != cudaSuccess) return e;
    if ((e = dalloc(&n.grad, kGuideParams)) != cudaSuccess) return e;
    if ((e = dalloc(&n.w16, kGuideWeights)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(n.m, 0, kGuideParams * sizeof(float), st)) != cudaSuccess) return e;
    return cudaMemsetAsync(n.v, 0, kGuideParams * sizeof(float), st);
}

void guide_free_net(GuideNet& n)
{
    void* p[] = {n.w32, n.m, n.v, n.grad, n.w16};
    for (void* x : p)
        if (x) cudaFree(x);
    n = GuideNet{};
}

// Uploads FP32 parameters and their FP16 copies.
cudaError_t guide_set_params(GuideNet& n, const float* w, cudaStream_t st)
{
    std::vector<__half> h(kGuideWeights);
    for (int i = 0; i < kGuideWeights; i++) h[i] = __float2half(w[i]);
    cudaError_t e = cudaMemcpyAsync(n.w32, w, kGuideParams * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(n.w16, h.data(), kGuideWeights * sizeof(__half), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);  // h is a host temporary
}

// Launches one of the fused tcgen05 kernels: one CTA per SM (at most one
// per tile), each with the kernel's shared-memory arrays.
template <int MODE>
cudaError_t guide_tc_launch(cudaStream_t st, const GuideTcArgs& a)
{
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_guide_tc<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(GuideTcSmem))) != cudaSuccess)
        return e;
    const unsigned tiles = (a.rows + kTcRows - 1) / kTcRows;
    k_guide_tc<MODE><<<std::max(1u, std::min(tiles, (unsigned)sms)), kTcThreads, sizeof(GuideTcSmem), st>>>(a);
    return cudaGetLastError();
}

GuideTcArgs guide_tc_args(const GuideNet& n, unsigned rows, float* scal)
{
    GuideTcArgs a{};
    a.w16 = n.w16;
    a.w32 = n.w32;
    a.rows = rows;
    a.weight_sum = scal + 1;
    a.grad = n.grad;
    a.loss_sum = scal;
    a.err = reinterpret_cast<unsigned*>(scal + 2);
    return a;
}

void guide_adam(cudaStream_t st, GuideNet& n, unsigned rows, float lr)
{
    n.steps++;
    const float b1 = .9f, b2 = .999f;
    const float bc1 = 1.f - std::pow(b1, (float)n.steps), bc2 = 1.f - std::pow(b2, (float)n.steps);
    k_guide_adam<<<(kGuideParams + 255) / 256, 256, 0, st>>>(n.w32, n.m, n.v, n.grad, kGuideParams, lr, b1, b2, 1e-8f,
                                                            bc1, bc2, 1.f / (float)rows, n.w16, kGuideWeights);
}

// One training step on a batch drawn from the records: its weight sum,
// then the fused forward / loss / backward kernel, then Adam.
cudaError_t guide_train_step(cudaStream_t st, GuideState& g, unsigned seed)
{
    GuideBatch& b = g.batch;
    cudaError_t e;
    if ((e = cudaMemsetAsync(b.scal, 0, 3 * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(g.net.grad, 0, kGuideParams * sizeof(float), st)) != cudaSuccess) return e;
    k_guide_record_weights<<<148, 256, 0, st>>>(g.recs, g.rec_count, g.rec_capacity, b.rows, seed, g.med_g,
                                                g.medium_slot, b.scal + 1);
    GuideTcArgs a = guide_tc_args(g.net, b.rows, b.scal);
    a.recs = g.recs;
    a.rec_count = g.rec_count;
    a.rec_capacity = g.rec_capacity;
    a.seed = seed;
    a.lo = g.lo;
    a.inv_ext = make_float3(1.f / g.ext.x, 1.f / g.ext.y, 1.f / g.ext.z);
    a.med_g = g.med_g;
    a.medium_slot = g.medium_slot;
    if ((e = guide_tc_launch<kTcTrainRecords>(st, a)) != cudaSuccess) return e;
    guide_adam(st, g.net, b.rows, 1e-3f);
    return cudaGetLastError();
}

// Bakes the network into a table (cell centres x direction bins x media
// slots) with the fused forward kernel.
cudaError_t guide_fill_table(cudaStream_t st, GuideState& g, float4* table)
{
    GuideTcArgs a = guide_tc_args(g.net, g.table_rows, g.batch.scal);
    a.cells = g.cells;
    a.dir_res = g.dir_res;
    a.lo = g.lo;
    a.cell = make_float3(g.ext.x / g.cells, g.ext.y / g.cells, g.ext.z / g.cells);
    a.inv_ext = make_float3(1.f / g.ext.x, 1.f / g.ext.y, 1.f / g.ext.z);
    a.entries = table;
    return guide_tc_launch<kTcBake>(st, a);
}

}  // namespace
