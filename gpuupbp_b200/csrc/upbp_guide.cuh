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
// would want to sample.  Forward and backward passes run fused, one kernel
// per training step, on the tcgen05 tensor cores (FP16 operands, FP32
// accumulators in tensor memory; upbp_guide_tc.cuh), with FP32 master
// weights and Adam.
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
constexpr int kGuideOut = kGuideLobes * 5 + 1;         // logits, mean xyz, log kappa, selection logit
constexpr int kGuideAlphaCol = kGuideLobes * 5;
// Largest probability of sampling the mixture rather than the phase
// function: the phase function keeps at least a tenth (defensive sampling).
constexpr float kGuideAlphaMax = 0.9f;
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
constexpr int kGuideTargetWords = 5;               // a training target: direction xyz, weight, phase pdf

// ---------------------------------------------------------------- encoding

// Frequency encoding of a position normalised to the scene box, the
// direction of travel and the medium's one-hot, in two halves of 48 inputs
// (the fused kernels give each half to its own thread): half 0 holds sin and
// cos of 2^b pi x and 2^b pi y for b = 0..11, half 1 those of z, then the
// direction, the one-hot of the medium slot and a zero pad.  sincospif takes
// the scaled coordinate exactly (a power-of-two multiple).
constexpr int kGuideHalf = kGuideInPad / 2;

UPBP_D void guide_bands(float x, float* out)
{
#pragma unroll
    for (int b = 0; b < kGuideBands; b++) {
        sincospif(x, &out[2 * b], &out[2 * b + 1]);
        x *= 2.f;
    }
}

UPBP_D void guide_encode_half(float3 xn, float3 d, int medium, int half, float* out)
{
    if (half == 0) {
        guide_bands(xn.x, out);
        guide_bands(xn.y, out + 2 * kGuideBands);
    } else {
        guide_bands(xn.z, out);
        out[2 * kGuideBands] = d.x;
        out[2 * kGuideBands + 1] = d.y;
        out[2 * kGuideBands + 2] = d.z;
#pragma unroll
        for (int m = 0; m < kGuideMedia; m++) out[2 * kGuideBands + 3 + m] = (m == medium) ? 1.f : 0.f;
        out[kGuideHalf - 1] = 0.f;
    }
}
static_assert(2 * kGuideBands + 3 + kGuideMedia + 1 == kGuideHalf, "second half of the input");

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

// Selection probability of a table entry's mixture against the phase function.
UPBP_D float guide_entry_alpha(const float4* e) { return __ldg(&e[kGuideLobes + 3]).w; }

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

// Probability of sampling the mixture rather than the phase function, from
// the network's selection logit.
UPBP_HD float guide_alpha(float logit) { return kGuideAlphaMax / (1.f + expf(-logit)); }

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

// Loss rows: -w log P(target), P = (1 - a) h + a q the blend the renderer
// samples -- h the phase function's pdf of the target direction (given),
// q the vMF mixture of the row's output, a the selection probability -- so
// the network learns where the mixture helps (a grows) and where the phase
// function alone fits the light's arrival directions (a shrinks).  Writes
// dLoss/dOutput (scaled so that the batch mean of the weights is 1) and the
// row's weighted loss.
UPBP_HD float guide_row_grad(const float* o, float4 t, float h, float wscale, float* grad, float* loss)
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
    const float sig = 1.f / (1.f + expf(-o[kGuideAlphaCol])), a = kGuideAlphaMax * sig;
    const float P = fmaxf((1.f - a) * h + a * q, 1e-30f);
    const float wt = t.w * wscale;
    *loss = -wt * logf(P);
    // d(-log P)/dq = -a / P: the mixture's gradients of -log q scaled by a q / P
    const float sq = wt * a * q / P;
    for (int k = 0; k < kGuideOutPad; k++) grad[k] = 0.f;
    for (int j = 0; j < kGuideLobes; j++) {
        const float r = v.pi[j] * val[j] / q;  // responsibility of lobe j
        // d(-log q)/d logit_j = pi_j - r_j
        grad[j] = sq * (v.pi[j] - r);
        // d(-log q)/d mu_j = -r_j kappa_j w; through the normalisation mu = m/|m|
        const float3 gmu = w * (-r * v.kappa[j]);
        const float3 gm = (gmu - v.mu[j] * dot(gmu, v.mu[j])) * (1.f / v.m_len[j]);
        grad[kGuideLobes + 3 * j] = sq * gm.x;
        grad[kGuideLobes + 3 * j + 1] = sq * gm.y;
        grad[kGuideLobes + 3 * j + 2] = sq * gm.z;
        // d log val_j / d kappa = 1/kappa - 2 e^{-2k}/(1 - e^{-2k}) + (mu.w - 1); kappa = exp(o), clamped
        const float k = v.kappa[j];
        const float e2 = expf(-2.f * k);
        const float dlog = 1.f / k - 2.f * e2 / fmaxf(1.f - e2, 1e-30f) + (dot(v.mu[j], w) - 1.f);
        const float raw = expf(o[4 * kGuideLobes + j]);
        const float inside = (raw > kGuideKappaMin && raw < kGuideKappaMax) ? 1.f : 0.f;
        grad[4 * kGuideLobes + j] = sq * (-r * dlog * k * inside);
    }
    // d(-log P)/d logit_a = -(q - h) / P * da/dlogit
    grad[kGuideAlphaCol] = -wt * (q - h) / P * kGuideAlphaMax * sig * (1.f - sig);
    return P;
}

// Weighted-batch scale: 1 / mean weight (targets of 5 floats: direction,
// weight, phase-function pdf).
__global__ void k_guide_weight_sum(const float* T, unsigned batch, float* sum)
{
    float s = 0.f;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x)
        s += T[(size_t)kGuideTargetWords * i + 3];
    for (int off = 16; off; off >>= 1) s += __shfl_down_sync(~0u, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
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

// One training row: record i of the batch (a hash of the step's seed and
// the row picks it), a uniformly drawn incoming direction w_i of a camera
// path, and the target: the direction the light came from, weighted by
// the record's throughput times the phase function between w_i and it.
// Returns false (weight 0) where the record's medium is not guided.
UPBP_D bool guide_train_sample(unsigned i, const GuideRecord* recs, const unsigned* rec_count, unsigned rec_capacity,
                               unsigned seed, const float* med_g, const int* medium_slot, GuideRecord& r, float3& wi,
                               int& slot, float4& target, float& phase_pdf)
{
    const unsigned nrec = min(*rec_count, rec_capacity);
    const unsigned h0 = guide_hash(seed * 0x9e3779b9u + i);
    r = recs[guide_hash(h0) % max(nrec, 1u)];
    const int med = (int)__float_as_uint(r.a.w);
    slot = nrec ? medium_slot[med] : -1;
    const float u0 = guide_u01(guide_hash(h0 ^ 0x68bc21ebu)), u1 = guide_u01(guide_hash(h0 ^ 0x02e5be93u));
    const float z = 1.f - 2.f * u0, s = sqrtf(fmaxf(0.f, 1.f - z * z)), phi = 6.28318530717959f * u1;
    wi = make_float3(s * cosf(phi), s * sinf(phi), z);
    const float3 tdir = make_float3(-r.b.x, -r.b.y, -r.b.z);  // toward where the light came from
    const float g = slot >= 0 ? med_g[med] : 0.f;
    const float ct = dot(wi, tdir);
    const float g2 = g * g, d = 1.f + g2 - 2.f * g * ct;
    const float phase = fabsf(g) < 1e-3f ? 0.0795774715f : 0.0795774715f * (1.f - g2) / (d * sqrtf(d));
    target = make_float4(tdir.x, tdir.y, tdir.z, slot >= 0 ? r.b.w * phase : 0.f);
    phase_pdf = phase;
    return slot >= 0;
}

// Training row i: one half of the network input (encoded position, w_i,
// medium slot) and the target.
UPBP_D void guide_train_row(unsigned i, const GuideRecord* recs, const unsigned* rec_count, unsigned rec_capacity,
                            unsigned seed, float3 lo, float3 inv_ext, const float* med_g, const int* medium_slot,
                            int half, float* in, float4& target, float& phase_pdf)
{
    GuideRecord r;
    float3 wi;
    int slot;
    guide_train_sample(i, recs, rec_count, rec_capacity, seed, med_g, medium_slot, r, wi, slot, target, phase_pdf);
    guide_encode_half((xyz(r.a) - lo) * inv_ext, wi, slot, half, in);
}

UPBP_D float guide_train_weight(unsigned i, const GuideRecord* recs, const unsigned* rec_count, unsigned rec_capacity,
                                unsigned seed, const float* med_g, const int* medium_slot)
{
    GuideRecord r;
    float3 wi;
    int slot;
    float4 target;
    float phase_pdf;
    guide_train_sample(i, recs, rec_count, rec_capacity, seed, med_g, medium_slot, r, wi, slot, target, phase_pdf);
    return target.w;
}

// Table row i: (slot, cell, direction bin) -> the cell centre, the bin's
// centre direction, the slot's medium.
UPBP_D void guide_table_row(unsigned i, int cells, int dir_res, float3 lo, float3 cell, float3 inv_ext, int half,
                            float* in)
{
    const unsigned per_slot = (unsigned)cells * cells * cells * dir_res * dir_res;
    const unsigned slot = i / per_slot, r = i % per_slot;
    const unsigned b = r % (dir_res * dir_res), c = r / (dir_res * dir_res);
    const unsigned ix = c % cells, iy = (c / cells) % cells, iz = c / (cells * cells);
    const float3 x = lo + make_float3((ix + .5f) * cell.x, (iy + .5f) * cell.y, (iz + .5f) * cell.z);
    const float3 d = oct_decode(make_float2(((b % dir_res) + .5f) / dir_res, ((b / dir_res) + .5f) / dir_res));
    guide_encode_half((x - lo) * inv_ext, d, (int)slot, half, in);
}

// Network output row -> table entry: lobe means and kappas, weights times
// normalisation, cumulative weights.
UPBP_D void guide_write_entry(const float* o, float4* e)
{
    VmfLobes v;
    vmf_from_output(o, v);
    float4 out[kGuideEntryWords];
    float* w = reinterpret_cast<float*>(out + kGuideLobes);
    float* cdf = reinterpret_cast<float*>(out + kGuideLobes + 2);
    float c = 0.f;
    for (int j = 0; j < kGuideLobes; j++) {
        out[j] = make_float4(v.mu[j].x, v.mu[j].y, v.mu[j].z, v.kappa[j]);
        w[j] = v.pi[j] * v.norm[j];
        c += v.pi[j];
        cdf[j] = c;
    }
    // the last cumulative weight is 1 and never read: it holds the selection probability
    cdf[kGuideLobes - 1] = guide_alpha(o[kGuideAlphaCol]);
    for (int k = 0; k < kGuideEntryWords; k++) e[k] = out[k];
}

}  // namespace upbp
