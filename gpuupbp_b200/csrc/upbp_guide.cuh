// Learned proposal for scattering in media: a small MLP maps a position
// (12-band frequency encoding), the direction of travel and a one-hot medium
// id to an 8-lobe von Mises-Fisher mixture, which is blended 50/50 with the
// Henyey-Greenstein phase function when camera subpaths scatter in a medium.
//
// Training is online: the light pass writes a record (position, direction
// of travel, medium, throughput) at every medium vertex; a training step
// draws a batch of records, pairs each with a random incoming direction w_i,
// and maximises the weighted log-likelihood of the light's arrival direction
// -d under the mixture conditioned on (x, w_i), each record weighted by its
// throughput times the phase function between w_i and -d: the maximiser is
// the normalised product of the phase function and the incident radiance the
// light subpaths carry, the density a camera path at x arriving along w_i
// would want to sample.  Forward and backward passes are FP16 tensor-core
// GEMMs with FP32 accumulation (mma.sync m16n8k16), FP32 master weights,
// Adam.
//
// For sampling and for every MIS pdf, the trained mixture is baked into a
// table over a grid of positions x directions of travel x media (the
// network evaluated at cell centres and direction-bin centres): every
// evaluation of the proposal's pdf, wherever in the recursive MIS it occurs,
// reads the same table entry as the sampling did, so the pdfs that enter the
// MIS quantities are exactly the sampling pdfs and the estimator stays
// unbiased.  Light subpaths keep sampling the phase function; the proposal's
// pdf enters every camera-direction pdf of the recursion (camera sampling,
// the reverse pdfs at light vertices, connections and merges).
#pragma once

#include <cuda_fp16.h>

#include "upbp_device.cuh"

namespace upbp {

constexpr int kGuideBands = 12;
constexpr int kGuideMedia = 20;                        // one-hot width
constexpr int kGuideIn = 3 * 2 * kGuideBands + 3 + kGuideMedia;  // 95
constexpr int kGuideInPad = 96;
constexpr int kGuideHidden = 64;
constexpr int kGuideLobes = 8;
constexpr int kGuideOut = kGuideLobes * 5;             // logits, mean xyz, log kappa
constexpr int kGuideOutPad = 48;
// layer shapes (in x out), row-major weights, FP16 copies of FP32 masters
constexpr int kGuideLayers = 4;
constexpr int kGuideLayerIn[kGuideLayers] = {kGuideInPad, kGuideHidden, kGuideHidden, kGuideHidden};
constexpr int kGuideLayerOut[kGuideLayers] = {kGuideHidden, kGuideHidden, kGuideHidden, kGuideOutPad};
constexpr int kGuideWOff[kGuideLayers + 1] = {0, kGuideInPad * kGuideHidden,
                                              kGuideInPad * kGuideHidden + kGuideHidden * kGuideHidden,
                                              kGuideInPad * kGuideHidden + 2 * kGuideHidden * kGuideHidden,
                                              kGuideInPad * kGuideHidden + 2 * kGuideHidden * kGuideHidden +
                                                  kGuideHidden * kGuideOutPad};
constexpr int kGuideWeights = kGuideWOff[kGuideLayers];
constexpr int kGuideBOff[kGuideLayers + 1] = {0, kGuideHidden, 2 * kGuideHidden, 3 * kGuideHidden,
                                              3 * kGuideHidden + kGuideOutPad};
constexpr int kGuideBiases = kGuideBOff[kGuideLayers];
constexpr int kGuideParams = kGuideWeights + kGuideBiases;
static_assert(kGuideWeights == 96 * 64 + 2 * 64 * 64 + 64 * 48 && kGuideParams == kGuideWeights + 240,
              "parameter layout (the float64 restatement and the C ABI share it)");
constexpr float kGuideKappaMin = 1e-2f, kGuideKappaMax = 2e3f;

// Table entry: per lobe (mean xyz, kappa), the lobe's weight times its
// normalisation, and the cumulative lobe weights for sampling (GuideTable in
// upbp_device.cuh).
constexpr int kGuideEntryWords = kGuideLobes + 4;  // float4s

// ---------------------------------------------------------------- encoding

// Frequency encoding of a position normalised to the scene box: sin and
// cos of 2^b pi x for b = 0..11 per axis, then the direction of travel, then
// the medium's one-hot.
UPBP_HD void guide_encode(float3 xn, float3 d, int medium, float* out)
{
    const float c[3] = {xn.x, xn.y, xn.z};
    int k = 0;
    for (int a = 0; a < 3; a++) {
        float f = 3.14159265358979f;
        for (int b = 0; b < kGuideBands; b++) {
            const float t = f * c[a];
            out[k++] = sinf(t);
            out[k++] = cosf(t);
            f *= 2.f;
        }
    }
    out[k++] = d.x;
    out[k++] = d.y;
    out[k++] = d.z;
    for (int m = 0; m < kGuideMedia; m++) out[k++] = (m == medium) ? 1.f : 0.f;
    while (k < kGuideInPad) out[k++] = 0.f;
}

// Octahedral map of a unit direction to [0,1)^2 and back.
UPBP_HD float2 oct_encode(float3 d)
{
    const float s = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
    float u = d.x / s, v = d.y / s;
    if (d.z < 0.f) {
        const float uu = (1.f - fabsf(v)) * (u >= 0.f ? 1.f : -1.f);
        const float vv = (1.f - fabsf(u)) * (v >= 0.f ? 1.f : -1.f);
        u = uu;
        v = vv;
    }
    return make_float2(.5f * u + .5f, .5f * v + .5f);
}

UPBP_HD float3 oct_decode(float2 e)
{
    float u = 2.f * e.x - 1.f, v = 2.f * e.y - 1.f;
    const float z = 1.f - fabsf(u) - fabsf(v);
    if (z < 0.f) {
        const float uu = (1.f - fabsf(v)) * (u >= 0.f ? 1.f : -1.f);
        const float vv = (1.f - fabsf(u)) * (v >= 0.f ? 1.f : -1.f);
        u = uu;
        v = vv;
    }
    const float3 d = make_float3(u, v, z);
    return d * (1.f / sqrtf(dot(d, d)));
}

// ---------------------------------------------------------------- vMF mixture

// vMF density normalisation kappa / (2 pi (1 - e^{-2 kappa})), written to stay
// accurate for small kappa.
UPBP_HD float vmf_norm(float kappa)
{
    const float den = kappa < 1e-3f ? (2.f * kappa - 2.f * kappa * kappa) : -expm1f(-2.f * kappa);
    return kappa / (2.f * 3.14159265358979f * den);
}

// Table entry of (cell, direction of travel, medium slot), or nullptr.
UPBP_D const float4* guide_entry(const GuideTable& g, int cell, float3 travel)
{
    if (!g.entries || cell < 0) return nullptr;
    const float2 e = oct_encode(travel);
    const int bx = min((int)(e.x * g.dir_res), g.dir_res - 1);
    const int by = min((int)(e.y * g.dir_res), g.dir_res - 1);
    return g.entries + ((size_t)cell * (g.dir_res * g.dir_res) + by * g.dir_res + bx) * kGuideEntryWords;
}

// Spatial cell (with the medium slot) of a point, -1 where not guided.
UPBP_D int guide_cell(const GuideTable& g, float3 x, int medium)
{
    if (!g.entries || medium < 0) return -1;
    const int slot = g.medium_slot[medium];
    if (slot < 0) return -1;
    const float3 f = (x - g.lo) * g.inv_cell;
    const int ix = min(max((int)f.x, 0), g.cells - 1), iy = min(max((int)f.y, 0), g.cells - 1),
              iz = min(max((int)f.z, 0), g.cells - 1);
    return ((slot * g.cells + iz) * g.cells + iy) * g.cells + ix;
}

UPBP_D float vmf_mix_pdf(const float4* e, float3 w)
{
    float p = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float4 l = __ldg(&e[j]);
        const float wj = reinterpret_cast<const float*>(e + kGuideLobes)[j];
        p += wj * __expf(l.w * (l.x * w.x + l.y * w.y + l.z * w.z - 1.f));
    }
    return p;
}

// Samples the mixture: a lobe by its weight (u0), a direction in it (u1, u2).
UPBP_D float3 vmf_mix_sample(const float4* e, float u0, float u1, float u2)
{
    const float* cdf = reinterpret_cast<const float*>(e + kGuideLobes + 2);
    int j = 0;
    while (j < kGuideLobes - 1 && u0 >= cdf[j]) j++;
    const float4 l = __ldg(&e[j]);
    const float k = l.w;
    // w = 1 + log(u + (1 - u) e^{-2k}) / k, the cosine to the lobe's mean
    const float wc = fminf(1.f, fmaxf(-1.f, 1.f + __logf(u1 + (1.f - u1) * __expf(-2.f * k)) / k));
    const float s = sqrtf(fmaxf(0.f, 1.f - wc * wc));
    const float phi = 6.28318530717959f * u2;
    Frame f;
    f.set_from_z(make_float3(l.x, l.y, l.z));
    return f.to_world(make_float3(s * __cosf(phi), s * __sinf(phi), wc));
}

// ---------------------------------------------------------------- tensor-core GEMM

// C[M x N] (+)= A[M x K] B[K x N] with FP16 operands addressed by strides
// (so transposed operands need no copy) and FP32 accumulation, on
// mma.sync.m16n8k16: a 64x64 block tile of four warps (32x32 each), K in
// steps of 32 staged through shared memory.  gridDim.z splits K; with
// gridDim.z > 1 or `accumulate` the tile is added into C atomically.
// Epilogue (split == 1 only): + bias[n], ReLU, FP16 copy into H.
struct GemmArgs {
    const __half* A;
    long long sam, sak;
    const __half* B;
    long long sbk, sbn;
    float* C;
    int ldc;
    int M, N, K, k_per_block;
    const float* bias;  // optional
    int relu;
    __half* H;          // optional FP16 copy of the output (ldh = ldc)
    int accumulate;
};

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 32, kGemmPad = 8;

UPBP_D void mma_16816(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_guide_gemm(GemmArgs g)
{
    __shared__ __align__(16) __half As[kGemmBM][kGemmBK + kGemmPad];
    __shared__ __align__(16) __half Bs[kGemmBN][kGemmBK + kGemmPad];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * kGemmBN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int kb = blockIdx.z * g.k_per_block;
    const int ke = min(g.K, kb + g.k_per_block);
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
    const __half zero = __float2half(0.f);
    for (int k0 = kb; k0 < ke; k0 += kGemmBK) {
        // consecutive threads read consecutive addresses of whichever
        // operand dimension is contiguous in memory
        const bool a_k_inner = g.sak == 1, b_k_inner = g.sbk == 1;
        for (int i = threadIdx.x; i < kGemmBM * kGemmBK; i += blockDim.x) {
            const int r = a_k_inner ? i / kGemmBK : i % kGemmBM, c = a_k_inner ? i % kGemmBK : i / kGemmBM;
            const int m = m0 + r, k = k0 + c;
            As[r][c] = (m < g.M && k < ke) ? g.A[m * g.sam + k * g.sak] : zero;
        }
        for (int i = threadIdx.x; i < kGemmBN * kGemmBK; i += blockDim.x) {
            const int r = b_k_inner ? i / kGemmBK : i % kGemmBN, c = b_k_inner ? i % kGemmBK : i / kGemmBN;
            const int n = n0 + r, k = k0 + c;
            Bs[r][c] = (n < g.N && k < ke) ? g.B[k * g.sbk + n * g.sbn] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk += 16) {
            unsigned a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int r = wm + 16 * i + gid;
                a[i][0] = *reinterpret_cast<const unsigned*>(&As[r][kk + 2 * tig]);
                a[i][1] = *reinterpret_cast<const unsigned*>(&As[r + 8][kk + 2 * tig]);
                a[i][2] = *reinterpret_cast<const unsigned*>(&As[r][kk + 8 + 2 * tig]);
                a[i][3] = *reinterpret_cast<const unsigned*>(&As[r + 8][kk + 8 + 2 * tig]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int n = wn + 8 * j + gid;
                b[j][0] = *reinterpret_cast<const unsigned*>(&Bs[n][kk + 2 * tig]);
                b[j][1] = *reinterpret_cast<const unsigned*>(&Bs[n][kk + 8 + 2 * tig]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_16816(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
    const bool atomic = g.accumulate || gridDim.z > 1;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int m = m0 + wm + 16 * i + gid + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + 8 * j + 2 * tig + (r & 1);
                if (m >= g.M || n >= g.N) continue;
                float v = acc[i][j][r];
                if (atomic) {
                    atomicAdd(&g.C[(size_t)m * g.ldc + n], v);
                    continue;
                }
                if (g.bias) v += g.bias[n];
                if (g.relu) v = fmaxf(v, 0.f);
                g.C[(size_t)m * g.ldc + n] = v;
                if (g.H) g.H[(size_t)m * g.ldc + n] = __float2half(v);
            }
}

// ---------------------------------------------------------------- training

// The mixture of one output row: softmax weights, unit means, kappas.
struct VmfLobes {
    float pi[kGuideLobes], kappa[kGuideLobes], norm[kGuideLobes];
    float3 mu[kGuideLobes], m_raw[kGuideLobes];
    float m_len[kGuideLobes];
};

UPBP_HD void vmf_from_output(const float* o, VmfLobes& v)
{
    float mx = o[0];
    for (int j = 1; j < kGuideLobes; j++) mx = fmaxf(mx, o[j]);
    float s = 0.f;
    for (int j = 0; j < kGuideLobes; j++) {
        v.pi[j] = expf(o[j] - mx);
        s += v.pi[j];
    }
    for (int j = 0; j < kGuideLobes; j++) {
        v.pi[j] /= s;
        const float3 m = make_float3(o[kGuideLobes + 3 * j], o[kGuideLobes + 3 * j + 1], o[kGuideLobes + 3 * j + 2]);
        v.m_raw[j] = m;
        v.m_len[j] = fmaxf(sqrtf(dot(m, m)), 1e-6f);
        v.mu[j] = m * (1.f / v.m_len[j]);
        v.kappa[j] = fminf(fmaxf(expf(o[4 * kGuideLobes + j]), kGuideKappaMin), kGuideKappaMax);
        v.norm[j] = vmf_norm(v.kappa[j]);
    }
}

// Records -> one training batch: inputs (FP16) and per row the target
// direction and its weight (the phase function between the sampled incoming
// direction and the target, times the record's throughput luminance).
UPBP_HD unsigned guide_hash(unsigned x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

UPBP_HD float guide_u01(unsigned h) { return (float)(h >> 8) * (1.f / 16777216.f); }

// Copies a block's rows of FP16 inputs from shared memory to X with 16-byte
// stores (rows are 96 halves = 12 such stores).
UPBP_D void guide_store_rows(const __half (*rows)[kGuideInPad], unsigned first, unsigned count, __half* X)
{
    __syncthreads();
    const uint4* src = reinterpret_cast<const uint4*>(rows);
    uint4* dst = reinterpret_cast<uint4*>(X + (size_t)first * kGuideInPad);
    const unsigned n = count * (kGuideInPad / 8);
    for (unsigned k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
}

constexpr int kGuideRowsPerBlock = 128;

__global__ void __launch_bounds__(kGuideRowsPerBlock) k_guide_batch(const GuideRecord* recs, const unsigned* rec_count,
                                                                    unsigned rec_capacity, unsigned batch, unsigned seed,
                                                                    float3 lo, float3 inv_ext, const float* med_g,
                                                                    const int* medium_slot, __half* X, float4* T)
{
    __shared__ __align__(16) __half rows[kGuideRowsPerBlock][kGuideInPad];
    const unsigned first = blockIdx.x * kGuideRowsPerBlock;
    const unsigned i = first + threadIdx.x;
    const unsigned count = min((unsigned)kGuideRowsPerBlock, batch - min(batch, first));
    if (i < batch) {
    const unsigned nrec = min(*rec_count, rec_capacity);
    const unsigned h0 = guide_hash(seed * 0x9e3779b9u + i);
    const GuideRecord r = recs[guide_hash(h0) % max(nrec, 1u)];
    const int med = (int)__float_as_uint(r.a.w);
    const int slot = nrec ? medium_slot[med] : -1;
    // incoming direction of travel of a camera path, uniform on the sphere
    const float u0 = guide_u01(guide_hash(h0 ^ 0x68bc21ebu)), u1 = guide_u01(guide_hash(h0 ^ 0x02e5be93u));
    const float z = 1.f - 2.f * u0, s = sqrtf(fmaxf(0.f, 1.f - z * z)), phi = 6.28318530717959f * u1;
    const float3 wi = make_float3(s * cosf(phi), s * sinf(phi), z);
    const float3 target = make_float3(-r.b.x, -r.b.y, -r.b.z);  // toward where the light came from
    const float g = slot >= 0 ? med_g[med] : 0.f;
    const float ct = dot(wi, target);
    const float g2 = g * g, d = 1.f + g2 - 2.f * g * ct;
    const float phase = fabsf(g) < 1e-3f ? 0.0795774715f : 0.0795774715f * (1.f - g2) / (d * sqrtf(d));
    float in[kGuideInPad];
    guide_encode((xyz(r.a) - lo) * inv_ext, wi, slot, in);
    for (int k = 0; k < kGuideInPad; k++) rows[threadIdx.x][k] = __float2half(in[k]);
    T[i] = make_float4(target.x, target.y, target.z, slot >= 0 ? r.b.w * phase : 0.f);
    }
    guide_store_rows(rows, first, count, X);
}

// Loss rows: -w log q(target) with q the vMF mixture of the row's output;
// writes dLoss/dOutput (FP16, per row, scaled so that the batch mean of the
// weights is 1) and the row's weighted loss.
UPBP_HD float guide_row_grad(const float* o, float4 t, float wscale, float* grad, float* loss)
{
    VmfLobes v;
    vmf_from_output(o, v);
    const float3 w = make_float3(t.x, t.y, t.z);
    float val[kGuideLobes], q = 0.f;
    for (int j = 0; j < kGuideLobes; j++) {
        val[j] = v.norm[j] * expf(v.kappa[j] * (dot(v.mu[j], w) - 1.f));
        q += v.pi[j] * val[j];
    }
    q = fmaxf(q, 1e-30f);
    const float wt = t.w * wscale;
    *loss = -wt * logf(q);
    for (int k = 0; k < kGuideOutPad; k++) grad[k] = 0.f;
    for (int j = 0; j < kGuideLobes; j++) {
        const float r = v.pi[j] * val[j] / q;  // responsibility of lobe j
        // d(-log q)/d logit_j = pi_j - r_j
        grad[j] = wt * (v.pi[j] - r);
        // d(-log q)/d mu_j = -r_j kappa_j w; through the normalisation mu = m/|m|
        const float3 gmu = w * (-r * v.kappa[j]);
        const float3 gm = (gmu - v.mu[j] * dot(gmu, v.mu[j])) * (1.f / v.m_len[j]);
        grad[kGuideLobes + 3 * j] = wt * gm.x;
        grad[kGuideLobes + 3 * j + 1] = wt * gm.y;
        grad[kGuideLobes + 3 * j + 2] = wt * gm.z;
        // d log val_j / d kappa = 1/kappa - 2 e^{-2k}/(1 - e^{-2k}) + (mu.w - 1); kappa = exp(o), clamped
        const float k = v.kappa[j];
        const float e2 = expf(-2.f * k);
        const float dlog = 1.f / k - 2.f * e2 / fmaxf(1.f - e2, 1e-30f) + (dot(v.mu[j], w) - 1.f);
        const float raw = expf(o[4 * kGuideLobes + j]);
        const float inside = (raw > kGuideKappaMin && raw < kGuideKappaMax) ? 1.f : 0.f;
        grad[4 * kGuideLobes + j] = wt * (-r * dlog * k * inside);
    }
    return q;
}

__global__ void k_guide_loss(const float* O, const float4* T, unsigned batch, const float* weight_sum, __half* dO,
                             float* loss_sum)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    const float wscale = *weight_sum > 0.f ? (float)batch / *weight_sum : 0.f;
    if (i < batch) {
        float o[kGuideOutPad], gr[kGuideOutPad];
        for (int k = 0; k < kGuideOutPad; k++) o[k] = O[(size_t)i * kGuideOutPad + k];
        guide_row_grad(o, T[i], wscale, gr, &l);
        for (int k = 0; k < kGuideOutPad; k++) dO[(size_t)i * kGuideOutPad + k] = __float2half(gr[k]);
    }
    const unsigned m = __ballot_sync(~0u, true);
    for (int off = 16; off; off >>= 1) l += __shfl_down_sync(m, l, off);
    if ((threadIdx.x & 31) == 0 && loss_sum) atomicAdd(loss_sum, l);
}

// Weighted-batch scale: 1 / mean weight.
__global__ void k_guide_weight_sum(const float4* T, unsigned batch, float* sum)
{
    float s = 0.f;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) s += T[i].w;
    for (int off = 16; off; off >>= 1) s += __shfl_down_sync(~0u, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

// dH *= relu'(H): zero where the forward activation was clamped.
__global__ void k_guide_relu_mask(const __half* H, float* dH, __half* dH16, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = __half2float(H[i]) > 0.f ? dH[i] : 0.f;
        dH[i] = v;
        dH16[i] = __float2half(v);
    }
}

// Bias gradient: column sums of dY [rows x cols], cols <= 64: thread t of a
// 256-thread block sums column t % 64 over every fourth row of the block's
// rows (a warp reads 32 consecutive halves of one row), then the four
// partial sums of a column meet in shared memory.
__global__ void __launch_bounds__(256) k_guide_colsum(const __half* dY, unsigned rows, int cols, float* out)
{
    __shared__ float part[4][64];
    const int c = threadIdx.x & 63, q = threadIdx.x >> 6;
    float s = 0.f;
    if (c < cols)
        for (unsigned r = blockIdx.x * 4 + q; r < rows; r += gridDim.x * 4) s += __half2float(dY[(size_t)r * cols + c]);
    part[q][c] = s;
    __syncthreads();
    if (q == 0 && c < cols) atomicAdd(&out[c], part[0][c] + part[1][c] + part[2][c] + part[3][c]);
}

// Adam on the FP32 masters (gradients are batch sums: scaled by 1/batch),
// then the FP16 copies the GEMMs read.
__global__ void k_guide_adam(float* w, float* m, float* v, const float* g, int n, float lr, float b1, float b2,
                             float eps, float bc1, float bc2, float gscale, __half* w16, int nw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (i < nw) w16[i] = __float2half(wi);
}

// Table inputs: one row per (slot, cell, direction bin): the cell centre,
// the bin's centre direction, the slot's medium.
__global__ void k_guide_table_inputs(int cells, int dir_res, int slots, float3 lo, float3 cell, float3 inv_ext,
                                     __half* X)
{
    const unsigned per_slot = (unsigned)cells * cells * cells * dir_res * dir_res;
    const unsigned n = per_slot * slots;
    __shared__ __align__(16) __half rows[kGuideRowsPerBlock][kGuideInPad];
    const unsigned first = blockIdx.x * kGuideRowsPerBlock;
    const unsigned i = first + threadIdx.x;
    const unsigned count = min((unsigned)kGuideRowsPerBlock, n - min(n, first));
    if (i < n) {
    const unsigned slot = i / per_slot, r = i % per_slot;
    const unsigned b = r % (dir_res * dir_res), c = r / (dir_res * dir_res);
    const unsigned ix = c % cells, iy = (c / cells) % cells, iz = c / (cells * cells);
    const float3 x = lo + make_float3((ix + .5f) * cell.x, (iy + .5f) * cell.y, (iz + .5f) * cell.z);
    const float3 d = oct_decode(make_float2(((b % dir_res) + .5f) / dir_res, ((b / dir_res) + .5f) / dir_res));
    float in[kGuideInPad];
    guide_encode((x - lo) * inv_ext, d, (int)slot, in);
    for (int k = 0; k < kGuideInPad; k++) rows[threadIdx.x][k] = __float2half(in[k]);
    }
    guide_store_rows(rows, first, count, X);
}

// Network outputs -> table entries (lobe means and kappas, weights times
// normalisation, cumulative weights).
__global__ void k_guide_table_entries(const float* O, unsigned n, float4* E)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    VmfLobes v;
    vmf_from_output(O + (size_t)i * kGuideOutPad, v);
    float4* e = E + (size_t)i * kGuideEntryWords;
    float* w = reinterpret_cast<float*>(e + kGuideLobes);
    float* cdf = reinterpret_cast<float*>(e + kGuideLobes + 2);
    float c = 0.f;
    for (int j = 0; j < kGuideLobes; j++) {
        e[j] = make_float4(v.mu[j].x, v.mu[j].y, v.mu[j].z, v.kappa[j]);
        w[j] = v.pi[j] * v.norm[j];
        c += v.pi[j];
        cdf[j] = c;
    }
    cdf[kGuideLobes - 1] = 1.f;
}

}  // namespace upbp
