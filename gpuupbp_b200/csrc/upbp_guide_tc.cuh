// The learned proposal's network on the 5th-generation tensor cores
// (tcgen05): one fused kernel per use.
//
//   k_guide_tc<kTcTrainRecords>  training step: draws a batch from the light
//                                subpaths' medium records, forward pass,
//                                loss and output gradient, backward pass,
//                                gradient sums of every parameter
//   k_guide_tc<kTcTrainRows>     the same on given input rows and targets
//                                (the gradient check entry point)
//   k_guide_tc<kTcBake>          forward pass over the proposal table's
//                                cell centres x direction bins, written as
//                                table entries
//
// A CTA of 256 threads owns one SM (its shared memory is above half of an
// SM's) and walks 128-row tiles, two threads per row (warps w and w + 4 read
// the same TMEM lanes): each takes half of the row's input encoding and of
// every hidden layer's columns; the first computes the row's loss.  The four FP16 weight matrices stay in
// shared memory for the whole kernel; a tile's inputs, hidden activations
// and gradients live in shared memory too, and nothing but the inputs'
// sources and the results touches global memory.  Each GEMM is a chain of
// tcgen05.mma (M = 128 rows, K = 16 per instruction, FP16 operands from
// shared memory, FP32 accumulators in tensor memory) issued by one thread;
// a tcgen05.commit on an mbarrier tells the CTA when the chain is done, and
// each thread then reads its own row back with tcgen05.ld (TMEM lane = tile
// row) for the element-wise epilogue (bias, ReLU, the vMF loss, the ReLU
// mask), whose FP16 result is the next GEMM's operand.  The weight
// gradients accumulate over all of a CTA's tiles in tensor memory and are
// added to the global sums once, at the end.
//
// Shared-memory operand layout: every matrix [R][C] is stored as 8 x 8
// core matrices of 16-byte rows, core matrix (r/8, c/8) at byte
// (r/8) * C * 16 + (c/8) * 128 (tiled_off).  The same bytes are a K-major
// operand when the matrix's rows are the GEMM's M or N and its columns K
// (leading byte offset 128, stride byte offset C * 16), and an MN-major
// operand when its columns are M or N and its rows K (stride 128, leading
// C * 16): the forward pass reads W [in][out] MN-major, the backward pass
// reads the same W K-major as W^T, and the weight gradients H^T dY read the
// activations and gradients MN-major, so no matrix is ever transposed.
#pragma once

#include "upbp_guide.cuh"

namespace upbp {

constexpr int kTcRows = 128;       // rows per tile = MMA M = TMEM lanes
constexpr int kTcThreads = 256;    // two threads per tile row: half 0 and half 1 of its columns
constexpr int kTcTmemCols = 512;   // forward / dH accumulator (64) + four weight-gradient accumulators (4 x 64)
constexpr int kTcTrainRecords = 0, kTcTrainRows = 1, kTcBake = 2;

UPBP_HD constexpr int tc_layer_in(int l) { return l == 0 ? kGuideInPad : kGuideHidden; }
UPBP_HD constexpr int tc_layer_out(int l) { return l == kGuideLayers - 1 ? kGuideOutPad : kGuideHidden; }
UPBP_HD constexpr int tc_w_off(int l)
{
    return l == 0 ? 0 : kGuideInPad * kGuideHidden + (l - 1) * kGuideHidden * kGuideHidden;
}
UPBP_HD constexpr int tc_b_off(int l) { return l * kGuideHidden; }

// Byte offset of element (r, c) of a [R][cols] matrix in core-matrix tiles.
UPBP_HD constexpr unsigned tiled_off(int r, int c, int cols)
{
    return (unsigned)((r >> 3) * cols * 16 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

struct GuideTcSmem {
    __half w[kGuideWeights];                 // W1..W4, each tiled, at their parameter offsets
    __half x[kTcRows * kGuideInPad];         // input rows
    __half h[3][kTcRows * kGuideHidden];     // hidden activations after ReLU
    __half d[2][kTcRows * kGuideHidden];     // output / hidden gradients, ping-pong
    __half tail[4096];                       // keeps every operand span of d[1] inside the struct
    float bias[kGuideBiases];
    unsigned long long mbar;
    unsigned tmem;
    unsigned pad[3];
};
// An MN-major operand of M = 128 over a matrix of 64 or 96 columns reads 16
// column groups of each row group, the upper ones (lanes of the result that
// are discarded) past the matrix's last row group: the arrays after x and
// each h[] absorb that (1 KB at most), and `tail` gives d[1] 8 KB of room,
// so every read stays in this struct.
static_assert(sizeof(__half) * kTcRows * kGuideHidden >= 1024, "overreach of an MN-major activation operand");
static_assert(offsetof(GuideTcSmem, x) % 16 == 0 && offsetof(GuideTcSmem, h) % 16 == 0 &&
                  offsetof(GuideTcSmem, d) % 16 == 0 && offsetof(GuideTcSmem, mbar) % 8 == 0,
              "operands start on 16-byte boundaries");
static_assert(kGuideWOff[1] == tc_w_off(1) && kGuideWOff[2] == tc_w_off(2) && kGuideWOff[3] == tc_w_off(3) &&
                  kGuideBOff[3] == tc_b_off(3),
              "parameter layout");

// ---------------------------------------------------------------- tcgen05 primitives

UPBP_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor without swizzling: start address, leading
// and stride byte offsets (16-byte units), descriptor version 1 (bit 46).
UPBP_D uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), FP16
// A and B (formats 0), A / B MN-major bits 15 / 16, N >> 3 at bit 17, M >> 4
// at bit 24.
UPBP_HD constexpr uint32_t umma_idesc(int m, int n, int a_mn, int b_mn)
{
    return (1u << 4) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

UPBP_D void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// Arrives on the mbarrier when every tcgen05.mma this thread issued is done.
UPBP_D void umma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

UPBP_D void mbar_init(uint32_t mbar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

UPBP_D bool mbar_try_wait(uint32_t mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for a phase (each try_wait suspends for a while in hardware
// before it gives up): false after the limit, so that a chain that never
// completes ends the kernel with an error instead of hanging it.
constexpr unsigned kTcWaitTries = 1u << 22;

UPBP_D bool mbar_wait_bounded(uint32_t mbar, uint32_t parity)
{
    for (unsigned i = 0; i < kTcWaitTries; i++)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

UPBP_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
UPBP_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's shared-memory stores visible to the tensor cores.
UPBP_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

UPBP_D void tmem_alloc(uint32_t dst, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

UPBP_D void tmem_dealloc(uint32_t taddr, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (the warp's
// 32-lane quarter at taddr), waited for before the values are used.
UPBP_D void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])::"memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// One GEMM as a chain of K = 16 instructions into TMEM columns d_tmem.
// Operand descriptors advance by a_step / b_step bytes per instruction.
UPBP_D void umma_chain(uint32_t d_tmem, uint32_t a, uint32_t a_lbo, uint32_t a_sbo, uint32_t a_step, uint32_t b,
                       uint32_t b_lbo, uint32_t b_sbo, uint32_t b_step, uint32_t idesc, int ksteps, bool accumulate)
{
    for (int k = 0; k < ksteps; k++)
        umma_f16(d_tmem, umma_desc(a + k * a_step, a_lbo, a_sbo), umma_desc(b + k * b_step, b_lbo, b_sbo), idesc,
                 (accumulate || k > 0) ? 1u : 0u);
}

// Stores 8 consecutive values of row r (columns 8 cg .. 8 cg + 7) as FP16.
UPBP_D void tile_store8(__half* m, int cols, int r, int cg, const float* v)
{
    const __half2 p0 = __floats2half2_rn(v[0], v[1]), p1 = __floats2half2_rn(v[2], v[3]),
                  p2 = __floats2half2_rn(v[4], v[5]), p3 = __floats2half2_rn(v[6], v[7]);
    uint4 u;
    u.x = *reinterpret_cast<const unsigned*>(&p0);
    u.y = *reinterpret_cast<const unsigned*>(&p1);
    u.z = *reinterpret_cast<const unsigned*>(&p2);
    u.w = *reinterpret_cast<const unsigned*>(&p3);
    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(m) + tiled_off(r, cg * 8, cols)) = u;
}

// ---------------------------------------------------------------- kernel

struct GuideTcArgs {
    const __half* w16;   // FP16 weights, row-major [in][out] per layer
    const float* w32;    // FP32 parameters (the biases are read from here)
    unsigned rows;       // rows of the batch or table
    // kTcTrainRecords: the batch is drawn from the records
    const GuideRecord* recs;
    const unsigned* rec_count;
    unsigned rec_capacity, seed;
    float3 lo, inv_ext;
    const float* med_g;
    const int* medium_slot;
    // kTcTrainRows: given rows and targets (kGuideTargetWords floats each:
    // direction, weight, phase-function pdf); O (optional) receives the outputs
    const __half* X;
    const float* T;
    float* O;
    // training: the batch's weight sum, gradient sums (kGuideParams) and summed loss, all accumulated atomically
    const float* weight_sum;
    float* grad;
    float* loss_sum;
    // kTcBake: the table's grid and its entries
    int cells, dir_res;
    float3 cell;
    float4* entries;
    unsigned* err;       // bit 0: a tensor-core chain did not complete in time
};

template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 1) k_guide_tc(GuideTcArgs a)
{
    extern __shared__ __align__(128) unsigned char tc_smem_raw[];
    GuideTcSmem& s = *reinterpret_cast<GuideTcSmem*>(tc_smem_raw);
    const int t = threadIdx.x, warp = t >> 5;
    const int r = t & (kTcRows - 1), half = t >> 7;  // tile row, half of its columns
    constexpr bool kTrain = MODE != kTcBake;

    // weights into their tiles (16-byte pieces of a row of W [in][out]), biases
#pragma unroll
    for (int l = 0; l < kGuideLayers; l++) {
        const int out = tc_layer_out(l), pieces = tc_layer_in(l) * out / 8;
        const __half* src = a.w16 + tc_w_off(l);
        char* dst = reinterpret_cast<char*>(s.w + tc_w_off(l));
        for (int i = t; i < pieces; i += kTcThreads) {
            const int j = i / (out / 8), o8 = i % (out / 8);
            *reinterpret_cast<uint4*>(dst + tiled_off(j, o8 * 8, out)) =
                __ldg(reinterpret_cast<const uint4*>(src + j * out + o8 * 8));
        }
    }
    for (int i = t; i < kGuideBiases; i += kTcThreads) s.bias[i] = a.w32[kGuideWeights + i];
    const uint32_t mbar = smem_u32(&s.mbar);
    if (t == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(smem_u32(&s.tmem), kTcTmemCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem;
    const uint32_t lane_tmem = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's quarter of the lanes
    const uint32_t acc_f = tmem;                                      // forward / dH accumulator, 64 columns
    auto acc_dw = [&](int l) { return tmem + 64u + 64u * (uint32_t)l; };

    const uint32_t sx = smem_u32(s.x), sw = smem_u32(s.w);
    const uint32_t sh[3] = {smem_u32(s.h[0]), smem_u32(s.h[1]), smem_u32(s.h[2])};
    const uint32_t sd[2] = {smem_u32(s.d[0]), smem_u32(s.d[1])};

    float wscale = 0.f;
    if (kTrain) wscale = *a.weight_sum > 0.f ? (float)a.rows / *a.weight_sum : 0.f;
    float bsum[kGuideLayers] = {0.f, 0.f, 0.f, 0.f};  // bias gradient: column t % 64, rows of half t / 64
    float loss = 0.f;
    uint32_t phase = 0;
    bool ok = true;
    int tiles_done = 0;

    // waits for the chain committed last; uniform over the CTA
    auto wait_chain = [&]() {
        bool done = mbar_wait_bounded(mbar, phase);
        done = __syncthreads_and(done);
        if (done) {
            phase ^= 1u;
            tc_fence_after();
        }
        return done;
    };
    // hands the tile's shared-memory writes and TMEM reads over to the next chain
    auto to_tensor_cores = [&]() {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
    };

    const unsigned ntiles = (a.rows + kTcRows - 1) / kTcRows;
    for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const unsigned row = tile * kTcRows + r;
        const bool valid = row < a.rows;
        float4 target = make_float4(0.f, 0.f, 0.f, 0.f);
        float phase_pdf = 0.f;  // the phase function's pdf of the target direction

        // ---- input row r: this thread's half of its 96 columns
        if (MODE == kTcTrainRows) {
            const uint4* src = reinterpret_cast<const uint4*>(a.X + (size_t)row * kGuideInPad);
            for (int cg = half * 6; cg < half * 6 + 6; cg++)
                *reinterpret_cast<uint4*>(reinterpret_cast<char*>(s.x) + tiled_off(r, cg * 8, kGuideInPad)) =
                    valid ? __ldg(src + cg) : make_uint4(0, 0, 0, 0);
            if (valid) {
                const float* tr = a.T + (size_t)kGuideTargetWords * row;
                target = make_float4(tr[0], tr[1], tr[2], tr[3]);
                phase_pdf = tr[4];
            }
        } else {
            float in[kGuideHalf];
            if (!valid) {
                for (int k = 0; k < kGuideHalf; k++) in[k] = 0.f;
            } else if (MODE == kTcTrainRecords) {
                guide_train_row(row, a.recs, a.rec_count, a.rec_capacity, a.seed, a.lo, a.inv_ext, a.med_g,
                                a.medium_slot, half, in, target, phase_pdf);
            } else {
                guide_table_row(row, a.cells, a.dir_res, a.lo, a.cell, a.inv_ext, half, in);
            }
            for (int cg = 0; cg < 6; cg++) tile_store8(s.x, kGuideInPad, r, half * 6 + cg, in + cg * 8);
        }
        to_tensor_cores();

        // ---- forward: H1..H3 (FP16, ReLU; masks of the positive ones), O
        unsigned mask[3];  // positive units of this thread's 32 columns of H1..H3
        float o[kGuideOutPad];
#pragma unroll
        for (int l = 0; l < kGuideLayers; l++) {
            const int K = tc_layer_in(l), N = tc_layer_out(l);
            if (t == 0) {
                tc_fence_after();
                const uint32_t A = l == 0 ? sx : sh[l - 1];
                const uint32_t B = sw + 2u * tc_w_off(l);
                umma_chain(acc_f, A, 128, K * 16, 256, B, N * 16, 128, 2 * N * 16, umma_idesc(kTcRows, N, 0, 1),
                           K / 16, false);
                umma_commit(mbar);
            }
            if (!(ok = wait_chain())) break;
            const float* b = s.bias + tc_b_off(l);
            if (l < kGuideLayers - 1) {
                mask[l] = 0u;
                for (int c0 = 32 * half; c0 < 32 * half + 32; c0 += 16) {
                    float v[16];
                    tmem_ld16(lane_tmem + acc_f + c0, v);
                    for (int i = 0; i < 16; i++) {
                        const float y = fmaxf(v[i] + b[c0 + i], 0.f);
                        v[i] = __half2float(__float2half(y));
                        if (v[i] > 0.f) mask[l] |= 1u << ((c0 + i) & 31);
                    }
                    tile_store8(s.h[l], kGuideHidden, r, c0 / 8, v);
                    tile_store8(s.h[l], kGuideHidden, r, c0 / 8 + 1, v + 8);
                }
            } else if (half == 0) {
                for (int c0 = 0; c0 < N; c0 += 16) {
                    tmem_ld16(lane_tmem + acc_f + c0, o + c0);
                    for (int i = 0; i < 16; i++) o[c0 + i] += b[c0 + i];
                }
            }
            to_tensor_cores();
        }
        if (!ok) break;

        if (MODE == kTcBake) {
            if (valid && half == 0) guide_write_entry(o, a.entries + (size_t)row * kGuideEntryWords);
            tiles_done++;
            continue;
        }
        if (MODE == kTcTrainRows && a.O && valid && half == 0) {
            float4* dst = reinterpret_cast<float4*>(a.O + (size_t)row * kGuideOutPad);
            for (int k = 0; k < kGuideOutPad / 4; k++) dst[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
        }

        // ---- loss and output gradient (row weight over the batch mean), FP16 into d[0]
        if (half == 0) {
            float g[kGuideOutPad], l = 0.f;
            if (valid) {
                guide_row_grad(o, target, phase_pdf, wscale, g, &l);
            } else {
                for (int k = 0; k < kGuideOutPad; k++) g[k] = 0.f;
            }
            loss += l;
            for (int cg = 0; cg < kGuideOutPad / 8; cg++) tile_store8(s.d[0], kGuideOutPad, r, cg, g + cg * 8);
        }
        to_tensor_cores();

        // ---- backward, layer 4 down to 1: dW_l += H_in^T dY, db_l += column sums of dY,
        //      dY_{l-1} = (dY W_l^T) masked by ReLU'(H_in)
        for (int l = kGuideLayers - 1; l >= 0 && ok; l--) {
            const int K = tc_layer_in(l), N = tc_layer_out(l);
            const int cur = (kGuideLayers - 1 - l) & 1;
            const __half* dy = s.d[cur];
            {  // bias gradient from the FP16 gradient rows of this tile
                const int c = t & 63, r0 = (t >> 6) * 32;
                if (c < N) {
                    float sum = 0.f;
                    for (int q = r0; q < r0 + 32; q++)
                        sum += __half2float(*reinterpret_cast<const __half*>(
                            reinterpret_cast<const char*>(dy) + tiled_off(q, c, N)));
                    bsum[l] += sum;
                }
            }
            if (t == 0) {
                tc_fence_after();
                const uint32_t A = l == 0 ? sx : sh[l - 1];
                umma_chain(acc_dw(l), A, K * 16, 128, 2 * K * 16, sd[cur], N * 16, 128, 2 * N * 16,
                           umma_idesc(kTcRows, N, 1, 1), kTcRows / 16, tiles_done > 0);
                if (l > 0)
                    umma_chain(acc_f, sd[cur], 128, N * 16, 256, sw + 2u * tc_w_off(l), 128, N * 16, 256,
                               umma_idesc(kTcRows, K, 0, 0), N / 16, false);
                umma_commit(mbar);
            }
            if (!(ok = wait_chain())) break;
            if (l > 0) {
                __half* nxt = s.d[cur ^ 1];
                for (int c0 = 32 * half; c0 < 32 * half + 32; c0 += 16) {
                    float v[16];
                    tmem_ld16(lane_tmem + acc_f + c0, v);
                    for (int i = 0; i < 16; i++)
                        if (!((mask[l - 1] >> ((c0 + i) & 31)) & 1u)) v[i] = 0.f;
                    tile_store8(nxt, kGuideHidden, r, c0 / 8, v);
                    tile_store8(nxt, kGuideHidden, r, c0 / 8 + 1, v + 8);
                }
                to_tensor_cores();
            }
        }
        if (!ok) break;
        tiles_done++;
    }

    if (!ok) {
        // a chain did not complete: flag it, give the chain in flight a last
        // bounded wait, then free the tensor memory
        if (t == 0) atomicOr(a.err, 1u);
        mbar_wait_bounded(mbar, phase);
    } else if (kTrain && tiles_done > 0) {
        // weight gradients: lane j of accumulator l holds row j of dW_l; the
        // two threads of a lane take the lower and upper columns
        for (int l = 0; l < kGuideLayers; l++) {
            const int K = tc_layer_in(l), N = tc_layer_out(l);
            float* gw = a.grad + tc_w_off(l) + (size_t)r * N;
            for (int c0 = 32 * half; c0 < min(N, 32 * half + 32); c0 += 16) {
                float v[16];
                tmem_ld16(lane_tmem + acc_dw(l) + c0, v);
                if (r < K)
                    for (int i = 0; i < 16; i++) atomicAdd(gw + c0 + i, v[i]);
            }
            const int c = t & 63;
            if (c < N) atomicAdd(a.grad + kGuideWeights + tc_b_off(l) + c, bsum[l]);
        }
        for (int off = 16; off; off >>= 1) loss += __shfl_down_sync(~0u, loss, off);
        if ((t & 31) == 0) atomicAdd(a.loss_sum, loss);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTcTmemCols);
    }
}

// Batch weight sum of a training step drawn from the records (the loss
// normalises the row weights by the batch mean before the FP16 gradients).
__global__ void k_guide_record_weights(const GuideRecord* recs, const unsigned* rec_count, unsigned rec_capacity,
                                       unsigned batch, unsigned seed, const float* med_g, const int* medium_slot,
                                       float* sum)
{
    float w = 0.f;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x)
        w += guide_train_weight(i, recs, rec_count, rec_capacity, seed, med_g, medium_slot);
    for (int off = 16; off; off >>= 1) w += __shfl_down_sync(~0u, w, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, w);
}

}  // namespace upbp
