// Host side of the learned proposal (kernels in upbp_guide.cuh): network
// state, the training step (forward, loss, backward, Adam) as a sequence of
// tensor-core GEMMs and element-wise kernels on the context's stream, and the
// table the render kernels read.  Included by upbp_capi.cu after its
// allocation and error-check helpers.
#pragma once

#include <random>

#include "upbp_guide.cuh"

namespace {

struct GuideNet {
    float* w32 = nullptr;    // FP32 master weights then biases (kGuideParams)
    float* m = nullptr;      // Adam moments
    float* v = nullptr;
    float* grad = nullptr;   // gradient sums of one batch
    __half* w16 = nullptr;   // FP16 weights the GEMMs read (kGuideWeights)
    int steps = 0;           // Adam steps taken
};

struct GuideBatch {
    unsigned rows = 0;
    __half* X = nullptr;      // rows x kGuideInPad
    __half* H[3] = {};        // rows x kGuideHidden, after ReLU
    float* Hf = nullptr;      // rows x kGuideHidden scratch (FP32 GEMM output)
    float* O = nullptr;       // rows x kGuideOutPad
    __half* dO = nullptr;     // rows x kGuideOutPad
    __half* dH = nullptr;     // rows x kGuideHidden
    float4* T = nullptr;      // rows: target direction, weight
    float* scal = nullptr;    // [0] weighted loss sum [1] weight sum
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
    float h_scal[2] = {0.f, 0.f};
    int front_next = -1;        // table the last training step filled
};

cudaError_t guide_alloc_batch(GuideBatch& b, unsigned rows)
{
    b.rows = rows;
    cudaError_t e;
    if ((e = dalloc(&b.X, (size_t)rows * kGuideInPad)) != cudaSuccess) return e;
    for (auto& h : b.H)
        if ((e = dalloc(&h, (size_t)rows * kGuideHidden)) != cudaSuccess) return e;
    if ((e = dalloc(&b.Hf, (size_t)rows * kGuideHidden)) != cudaSuccess) return e;
    if ((e = dalloc(&b.O, (size_t)rows * kGuideOutPad)) != cudaSuccess) return e;
    if ((e = dalloc(&b.dO, (size_t)rows * kGuideOutPad)) != cudaSuccess) return e;
    if ((e = dalloc(&b.dH, (size_t)rows * kGuideHidden)) != cudaSuccess) return e;
    if ((e = dalloc(&b.T, rows)) != cudaSuccess) return e;
    return dalloc(&b.scal, 2);
}

void guide_free_batch(GuideBatch& b)
{
    void* p[] = {b.X, b.H[0], b.H[1], b.H[2], b.Hf, b.O, b.dO, b.dH, b.T, b.scal};
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

void guide_gemm(cudaStream_t st, const __half* A, long long sam, long long sak, const __half* B, long long sbk,
                long long sbn, float* C, int ldc, int M, int N, int K, const float* bias, int relu, __half* H,
                bool accumulate, int split)
{
    GemmArgs g{A, sam, sak, B, sbk, sbn, C, ldc, M, N, K, 0, bias, relu, H, accumulate ? 1 : 0};
    split = std::max(1, std::min(split, (K + kGemmBK - 1) / kGemmBK));
    const int per = ((K + split - 1) / split + kGemmBK - 1) / kGemmBK * kGemmBK;
    g.k_per_block = per;
    split = (K + per - 1) / per;
    dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + kGemmBN - 1) / kGemmBN, split);
    k_guide_gemm<<<grid, 128, 0, st>>>(g);
}

// Forward pass of `rows` inputs: H[0..2] (FP16, after ReLU) and O (FP32).
void guide_forward(cudaStream_t st, const GuideNet& n, GuideBatch& b, const __half* X, unsigned rows)
{
    const float* bias = n.w32 + kGuideWeights;
    const __half* in = X;
    for (int l = 0; l < 3; l++) {
        const int K = kGuideLayerIn[l], N = kGuideLayerOut[l];
        guide_gemm(st, in, K, 1, n.w16 + kGuideWOff[l], N, 1, b.Hf, N, (int)rows, N, K, bias + kGuideBOff[l], 1, b.H[l],
                   false, 1);
        in = b.H[l];
    }
    guide_gemm(st, in, kGuideHidden, 1, n.w16 + kGuideWOff[3], kGuideOutPad, 1, b.O, kGuideOutPad, (int)rows,
               kGuideOutPad, kGuideHidden, bias + kGuideBOff[3], 0, nullptr, false, 1);
}

// Backward pass of the batch in b (after guide_forward and the loss's dO):
// gradient sums into n.grad.
void guide_backward(cudaStream_t st, GuideNet& n, GuideBatch& b, unsigned rows)
{
    const int R = (int)rows;
    const int split = std::max(1, std::min(148, R / 1024));
    float* gw = n.grad;
    float* gb = n.grad + kGuideWeights;
    const __half* dY = b.dO;
    int ny = kGuideOutPad;
    for (int l = kGuideLayers - 1; l >= 0; l--) {
        const int K = kGuideLayerIn[l];
        const __half* Hin = l == 0 ? b.X : b.H[l - 1];
        // dW_l = H_in^T dY, db_l = column sums of dY
        guide_gemm(st, Hin, 1, K, dY, ny, 1, gw + kGuideWOff[l], ny, K, ny, R, nullptr, 0, nullptr, true, split);
        k_guide_colsum<<<296, 256, 0, st>>>(dY, rows, ny, gb + kGuideBOff[l]);
        if (l == 0) break;
        // dH_in = (dY W_l^T) masked by the ReLU of H_in
        guide_gemm(st, dY, ny, 1, n.w16 + kGuideWOff[l], 1, ny, b.Hf, kGuideHidden, R, kGuideHidden, ny, nullptr, 0,
                   nullptr, false, 1);
        const size_t cnt = (size_t)rows * kGuideHidden;
        k_guide_relu_mask<<<(unsigned)std::min<size_t>((cnt + 255) / 256, 148 * 64), 256, 0, st>>>(b.H[l - 1], b.Hf,
                                                                                                    b.dH, cnt);
        dY = b.dH;
        ny = kGuideHidden;
    }
}

void guide_adam(cudaStream_t st, GuideNet& n, unsigned rows, float lr)
{
    n.steps++;
    const float b1 = .9f, b2 = .999f;
    const float bc1 = 1.f - std::pow(b1, (float)n.steps), bc2 = 1.f - std::pow(b2, (float)n.steps);
    k_guide_adam<<<(kGuideParams + 255) / 256, 256, 0, st>>>(n.w32, n.m, n.v, n.grad, kGuideParams, lr, b1, b2, 1e-8f,
                                                            bc1, bc2, 1.f / (float)rows, n.w16, kGuideWeights);
}

// Loss and output gradients of the batch in b (weights normalised by the
// batch mean).
void guide_loss(cudaStream_t st, GuideBatch& b, unsigned rows)
{
    cudaMemsetAsync(b.scal, 0, 2 * sizeof(float), st);
    k_guide_weight_sum<<<148, 256, 0, st>>>(b.T, rows, b.scal + 1);
    k_guide_loss<<<(rows + 255) / 256, 256, 0, st>>>(b.O, b.T, rows, b.scal + 1, b.dO, b.scal);
}

// One training step on a batch drawn from the records.
void guide_train_step(cudaStream_t st, GuideState& g, unsigned seed)
{
    GuideBatch& b = g.batch;
    const float3 inv_ext = make_float3(1.f / g.ext.x, 1.f / g.ext.y, 1.f / g.ext.z);
    k_guide_batch<<<(b.rows + kGuideRowsPerBlock - 1) / kGuideRowsPerBlock, kGuideRowsPerBlock, 0, st>>>(
        g.recs, g.rec_count, g.rec_capacity, b.rows, seed, g.lo, inv_ext, g.med_g, g.medium_slot, b.X, b.T);
    guide_forward(st, g.net, b, b.X, b.rows);
    guide_loss(st, b, b.rows);
    cudaMemsetAsync(g.net.grad, 0, kGuideParams * sizeof(float), st);
    guide_backward(st, g.net, b, b.rows);
    guide_adam(st, g.net, b.rows, 1e-3f);
}

// Bakes the network into the back table (cell centres x direction bins x
// media slots), in chunks of the batch's rows.
void guide_fill_table(cudaStream_t st, GuideState& g, float4* table)
{
    GuideBatch& b = g.batch;
    const float3 cell = make_float3(g.ext.x / g.cells, g.ext.y / g.cells, g.ext.z / g.cells);
    const float3 inv_ext = make_float3(1.f / g.ext.x, 1.f / g.ext.y, 1.f / g.ext.z);
    k_guide_table_inputs<<<(g.table_rows + kGuideRowsPerBlock - 1) / kGuideRowsPerBlock, kGuideRowsPerBlock, 0, st>>>(
        g.cells, g.dir_res, g.slots, g.lo, cell, inv_ext, b.X);
    guide_forward(st, g.net, b, b.X, g.table_rows);
    k_guide_table_entries<<<(g.table_rows + 255) / 256, 256, 0, st>>>(b.O, g.table_rows, table);
}

}  // namespace
