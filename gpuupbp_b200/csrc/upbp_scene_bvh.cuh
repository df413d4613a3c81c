// Binned-SAH build of the static scene's BVH on the device (once per context
// and class of triangles, real and imaginary).  The reference hands its
// triangles to OptiX's builder (renderer/renderer_init.cpp:134-289); this
// build is its own, a top-down binned SAH:
//
//   * a range of m >= 2 primitives (positions a..e of the order array) is
//     split by the surface-area heuristic over 16 centroid bins per axis:
//     the cost of a split after bin k is area(left box) x left count +
//     area(right box) x right count, evaluated in double precision; the
//     first minimum over axes 0, 1, 2 and bins 0..14 wins.  Ranges at depth
//     48 or more, and ranges whose centroids coincide, are split at their
//     middle.  One primitive per leaf.
//   * the primitives are partitioned stably (left side first, each side in
//     its previous order), so the whole tree -- node slots, boxes, leaf
//     order -- is a function of the input alone: oracle/sah_ref.cpp states
//     the same build sequentially and the tests compare the two bit for bit.
//   * node slots: the root is node 0, a subtree of m primitives occupies m - 1
//     consecutive slots, its root first (left child at slot + 1, right child
//     at slot + left count), so slots need no allocation counter.
//
// Ranges of more than kSahSmall primitives are split a level at a time by
// kernels over chunks of their positions (centroid bounds, bins, split
// choice, stable partition); the host orchestrates the levels and reads the
// split counts back.  Smaller ranges are finished by one thread each,
// running the same steps sequentially.  Every float operation that decides
// a split is written with explicit rounding (no contraction), as in the
// sequential statement.
#pragma once

#include "upbp_device.cuh"

namespace upbp {

constexpr int kSahBins = 16;
constexpr int kSahMaxDepth = 48;
constexpr unsigned kSahSmall = 32;
constexpr unsigned kSahChunk = 2048;        // positions per work item of the level kernels
constexpr int kSahThreads = 256;            // 8 positions per thread per chunk
constexpr float kSahEmptyLo = 1e30f, kSahEmptyHi = -1e30f;

struct SahTask {
    unsigned a, e, slot, depth;
};

struct SahWork {
    unsigned task, a, e;
};

// Bins of one range: counts and primitive boxes per axis and bin, and the
// range's centroid bounds.
struct SahBins {
    float cb[6];                       // centroid lo.xyz, hi.xyz
    unsigned count[3][kSahBins];
    float box[3][kSahBins][6];         // lo.xyz, hi.xyz
};

struct SahSplit {
    int axis, bin;    // axis -1: split at the middle
    unsigned ml;      // primitives on the left
    float lo, scale;  // bin of a centroid coordinate c: sah_bin(c, lo, scale)
};

// Bin of a centroid coordinate: 0 .. kSahBins-1, also for values outside the
// bounds.
UPBP_D int sah_bin(float c, float lo, float scale)
{
    const float f = __fmul_rn(__fsub_rn(c, lo), scale);
    return f > 0.f ? min(kSahBins - 1, (int)fminf(f, (float)kSahBins)) : 0;
}

UPBP_D double sah_area(const float* lo, const float* hi)
{
    const double d0 = fmaxf(0.f, __fsub_rn(hi[0], lo[0])), d1 = fmaxf(0.f, __fsub_rn(hi[1], lo[1])),
                 d2 = fmaxf(0.f, __fsub_rn(hi[2], lo[2]));
    return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(d0, d1), __dmul_rn(d1, d2)), __dmul_rn(d2, d0)));
}

UPBP_D void sah_grow(float* lo, float* hi, const float* blo, const float* bhi)
{
    for (int k = 0; k < 3; k++) {
        lo[k] = fminf(lo[k], blo[k]);
        hi[k] = fmaxf(hi[k], bhi[k]);
    }
}

// The split of a range of m primitives from its bins, and the children's
// boxes (unions of the bins on each side; for a middle split left to the
// caller).
UPBP_D void sah_choose(const SahBins& b, unsigned m, unsigned depth, SahSplit& s, float* lbox, float* rbox)
{
    double best = 1e300;
    s.axis = -1;
    s.bin = -1;
    if (depth < (unsigned)kSahMaxDepth) {
        for (int ax = 0; ax < 3; ax++) {
            const float ext = __fsub_rn(b.cb[3 + ax], b.cb[ax]);
            if (!(ext > 0.f)) continue;
            double right_area[kSahBins];
            unsigned right_count[kSahBins];
            float lo[3] = {kSahEmptyLo, kSahEmptyLo, kSahEmptyLo}, hi[3] = {kSahEmptyHi, kSahEmptyHi, kSahEmptyHi};
            unsigned c = 0;
            for (int k = kSahBins - 1; k > 0; k--) {
                sah_grow(lo, hi, b.box[ax][k], b.box[ax][k] + 3);
                c += b.count[ax][k];
                right_area[k] = sah_area(lo, hi);
                right_count[k] = c;
            }
            for (int k = 0; k < 3; k++) {
                lo[k] = kSahEmptyLo;
                hi[k] = kSahEmptyHi;
            }
            c = 0;
            for (int k = 0; k < kSahBins - 1; k++) {
                sah_grow(lo, hi, b.box[ax][k], b.box[ax][k] + 3);
                c += b.count[ax][k];
                if (c == 0 || right_count[k + 1] == 0) continue;
                const double cost = __dadd_rn(__dmul_rn(sah_area(lo, hi), (double)c),
                                              __dmul_rn(right_area[k + 1], (double)right_count[k + 1]));
                if (cost < best) {
                    best = cost;
                    s.axis = ax;
                    s.bin = k;
                }
            }
        }
    }
    if (s.axis < 0) {
        s.ml = m / 2;
        s.lo = 0.f;
        s.scale = 0.f;
        return;
    }
    s.lo = b.cb[s.axis];
    s.scale = __fdiv_rn((float)kSahBins, __fsub_rn(b.cb[3 + s.axis], b.cb[s.axis]));
    s.ml = 0;
    for (int k = 0; k < 6; k++) {
        lbox[k] = k < 3 ? kSahEmptyLo : kSahEmptyHi;
        rbox[k] = k < 3 ? kSahEmptyLo : kSahEmptyHi;
    }
    for (int k = 0; k < kSahBins; k++) {
        if (k <= s.bin) {
            s.ml += b.count[s.axis][k];
            sah_grow(lbox, lbox + 3, b.box[s.axis][k], b.box[s.axis][k] + 3);
        } else {
            sah_grow(rbox, rbox + 3, b.box[s.axis][k], b.box[s.axis][k] + 3);
        }
    }
}

UPBP_D bool sah_goes_left(const SahSplit& s, float4 cen, unsigned pos_in_range)
{
    if (s.axis < 0) return pos_in_range < s.ml;
    const float c = s.axis == 0 ? cen.x : (s.axis == 1 ? cen.y : cen.z);
    return sah_bin(c, s.lo, s.scale) <= s.bin;
}

// Node words: left box, right box, links, counts (BvhNode).
UPBP_D void sah_write_node(BvhNode* nodes, unsigned slot, unsigned a, unsigned m, unsigned ml, const float* lb,
                           const float* rb)
{
    const unsigned mr = m - ml;
    BvhNode n;
    n.a = make_float4(lb[0], lb[1], lb[2], lb[3]);
    n.b = make_float4(lb[4], lb[5], rb[0], rb[1]);
    n.c = make_float4(rb[2], rb[3], rb[4], rb[5]);
    n.link = make_int4(ml == 1 ? ~(int)a : (int)(slot + 1), mr == 1 ? ~(int)(a + ml) : (int)(slot + ml), (int)ml,
                       (int)mr);
    nodes[slot] = n;
}

// ---------------------------------------------------------------- primitives

// Triangle boxes as the device intersects them (v0, v0 + e1, v0 + e2),
// widened by 1e-6 of their extent plus 1e-7 of the first corner's
// magnitude, and their centroids.
__global__ void k_sah_tri_boxes(const float4* tri, unsigned n, float4* blo, float4* bhi, float4* cen)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v0 = tri[3 * (size_t)i], e1 = tri[3 * (size_t)i + 1], e2 = tri[3 * (size_t)i + 2];
    const float px[3] = {v0.x, __fadd_rn(v0.x, e1.x), __fadd_rn(v0.x, e2.x)};
    const float py[3] = {v0.y, __fadd_rn(v0.y, e1.y), __fadd_rn(v0.y, e2.y)};
    const float pz[3] = {v0.z, __fadd_rn(v0.z, e1.z), __fadd_rn(v0.z, e2.z)};
    float lo[3] = {fminf(fminf(px[0], px[1]), px[2]), fminf(fminf(py[0], py[1]), py[2]), fminf(fminf(pz[0], pz[1]), pz[2])};
    float hi[3] = {fmaxf(fmaxf(px[0], px[1]), px[2]), fmaxf(fmaxf(py[0], py[1]), py[2]), fmaxf(fmaxf(pz[0], pz[1]), pz[2])};
    const float mag = __fmul_rn(1e-7f, __fadd_rn(__fadd_rn(__fadd_rn(fabsf(lo[0]), fabsf(lo[1])), fabsf(lo[2])), 1e-3f));
    float l[3], h[3], c[3];
    for (int k = 0; k < 3; k++) {
        const float ext = __fadd_rn(__fmul_rn(__fsub_rn(hi[k], lo[k]), 1e-6f), mag);
        l[k] = __fsub_rn(lo[k], ext);
        h[k] = __fadd_rn(hi[k], ext);
        c[k] = __fmul_rn(0.5f, __fadd_rn(l[k], h[k]));
    }
    blo[i] = make_float4(l[0], l[1], l[2], 0.f);
    bhi[i] = make_float4(h[0], h[1], h[2], 0.f);
    cen[i] = make_float4(c[0], c[1], c[2], 0.f);
}

// ---------------------------------------------------------------- float atomics (min / max by bit patterns)

UPBP_D void atomic_min_f(float* a, float v)
{
    v = __fadd_rn(v, 0.f);  // -0 -> +0: the integer orderings below treat zero as positive
    if (v >= 0.f)
        atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
    else
        atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}

UPBP_D void atomic_max_f(float* a, float v)
{
    v = __fadd_rn(v, 0.f);
    if (v >= 0.f)
        atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
    else
        atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}

// ---------------------------------------------------------------- level kernels (ranges above kSahSmall)

__global__ void k_sah_init_bins(SahBins* bins, unsigned tasks)
{
    const unsigned t = blockIdx.x;
    if (t >= tasks) return;
    SahBins& b = bins[t];
    for (int i = threadIdx.x; i < 6; i += blockDim.x) b.cb[i] = i < 3 ? kSahEmptyLo : kSahEmptyHi;
    unsigned* cnt = &b.count[0][0];
    for (int i = threadIdx.x; i < 3 * kSahBins; i += blockDim.x) cnt[i] = 0;
    float* bx = &b.box[0][0][0];
    for (int i = threadIdx.x; i < 3 * kSahBins * 6; i += blockDim.x) bx[i] = (i % 6) < 3 ? kSahEmptyLo : kSahEmptyHi;
}

// Centroid bounds of every range, one block per chunk.
__global__ void __launch_bounds__(kSahThreads) k_sah_centroid_bounds(const SahWork* work, const unsigned* perm,
                                                                     const float4* cen, SahBins* bins)
{
    __shared__ float red[6];
    const SahWork w = work[blockIdx.x];
    if (threadIdx.x < 6) red[threadIdx.x] = threadIdx.x < 3 ? kSahEmptyLo : kSahEmptyHi;
    __syncthreads();
    float lo[3] = {kSahEmptyLo, kSahEmptyLo, kSahEmptyLo}, hi[3] = {kSahEmptyHi, kSahEmptyHi, kSahEmptyHi};
    for (unsigned k = w.a + threadIdx.x; k < w.e; k += blockDim.x) {
        const float4 c = cen[perm[k]];
        const float v[3] = {c.x, c.y, c.z};
        sah_grow(lo, hi, v, v);
    }
    for (int k = 0; k < 3; k++) {
        for (int off = 16; off; off >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(~0u, lo[k], off));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(~0u, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++) {
            atomic_min_f(&red[k], lo[k]);
            atomic_max_f(&red[3 + k], hi[k]);
        }
    __syncthreads();
    if (threadIdx.x < 3) atomic_min_f(&bins[w.task].cb[threadIdx.x], red[threadIdx.x]);
    else if (threadIdx.x < 6) atomic_max_f(&bins[w.task].cb[threadIdx.x], red[threadIdx.x]);
}

// Bins of every range along the axes where its centroids spread, one block
// per chunk (shared-memory bins, then one global update per used bin).
__global__ void __launch_bounds__(kSahThreads) k_sah_bins(const SahWork* work, const unsigned* perm,
                                                          const float4* cen, const float4* blo, const float4* bhi,
                                                          SahBins* bins)
{
    __shared__ unsigned cnt[3][kSahBins];
    __shared__ float bx[3][kSahBins][6];
    const SahWork w = work[blockIdx.x];
    SahBins& g = bins[w.task];
    for (int i = threadIdx.x; i < 3 * kSahBins; i += blockDim.x) (&cnt[0][0])[i] = 0;
    for (int i = threadIdx.x; i < 3 * kSahBins * 6; i += blockDim.x)
        (&bx[0][0][0])[i] = (i % 6) < 3 ? kSahEmptyLo : kSahEmptyHi;
    float lo[3], scale[3];
    bool used[3];
    for (int ax = 0; ax < 3; ax++) {
        const float ext = __fsub_rn(g.cb[3 + ax], g.cb[ax]);
        used[ax] = ext > 0.f;
        lo[ax] = g.cb[ax];
        scale[ax] = used[ax] ? __fdiv_rn((float)kSahBins, ext) : 0.f;
    }
    __syncthreads();
    for (unsigned k = w.a + threadIdx.x; k < w.e; k += blockDim.x) {
        const unsigned p = perm[k];
        const float4 c = cen[p], l = blo[p], h = bhi[p];
        const float cv[3] = {c.x, c.y, c.z};
        for (int ax = 0; ax < 3; ax++) {
            if (!used[ax]) continue;
            const int b = sah_bin(cv[ax], lo[ax], scale[ax]);
            atomicAdd(&cnt[ax][b], 1u);
            atomic_min_f(&bx[ax][b][0], l.x);
            atomic_min_f(&bx[ax][b][1], l.y);
            atomic_min_f(&bx[ax][b][2], l.z);
            atomic_max_f(&bx[ax][b][3], h.x);
            atomic_max_f(&bx[ax][b][4], h.y);
            atomic_max_f(&bx[ax][b][5], h.z);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * kSahBins; i += blockDim.x) {
        const int ax = i / kSahBins, b = i % kSahBins;
        if (cnt[ax][b] == 0) continue;
        atomicAdd(&g.count[ax][b], cnt[ax][b]);
        for (int k = 0; k < 3; k++) {
            atomic_min_f(&g.box[ax][b][k], bx[ax][b][k]);
            atomic_max_f(&g.box[ax][b][3 + k], bx[ax][b][3 + k]);
        }
    }
}

// One thread per range: the split, and the node for SAH splits (a middle
// split's boxes are known after the partition, k_sah_middle_nodes).
__global__ void k_sah_choose(const SahTask* tasks, unsigned n_tasks, const SahBins* bins, SahSplit* splits,
                             BvhNode* nodes)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    const SahTask tk = tasks[t];
    SahSplit s;
    float lb[6], rb[6];
    sah_choose(bins[t], tk.e - tk.a, tk.depth, s, lb, rb);
    splits[t] = s;
    if (s.axis >= 0) sah_write_node(nodes, tk.slot, tk.a, tk.e - tk.a, s.ml, lb, rb);
}

// Left-going primitives of each chunk (8 consecutive positions per thread).
__global__ void __launch_bounds__(kSahThreads) k_sah_count_left(const SahWork* work, const SahTask* tasks,
                                                                const SahSplit* splits, const unsigned* perm,
                                                                const float4* cen, unsigned* chunk_left)
{
    __shared__ unsigned total;
    const SahWork w = work[blockIdx.x];
    const SahTask tk = tasks[w.task];
    const SahSplit s = splits[w.task];
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    unsigned c = 0;
    for (unsigned k = w.a + threadIdx.x; k < w.e; k += blockDim.x) c += sah_goes_left(s, cen[perm[k]], k - tk.a);
    for (int off = 16; off; off >>= 1) c += __shfl_xor_sync(~0u, c, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&total, c);
    __syncthreads();
    if (threadIdx.x == 0) chunk_left[blockIdx.x] = total;
}

// Stable partition of each chunk into its range's left and right parts:
// left_off / right_off are the chunk's offsets within them (the earlier
// chunks' counts).
__global__ void __launch_bounds__(kSahThreads) k_sah_scatter(const SahWork* work, const SahTask* tasks,
                                                             const SahSplit* splits, const unsigned* perm,
                                                             const float4* cen, const unsigned* left_off,
                                                             const unsigned* right_off, unsigned* perm_out)
{
    constexpr int kPer = kSahChunk / kSahThreads;
    __shared__ unsigned warp_sum[kSahThreads / 32];
    const SahWork w = work[blockIdx.x];
    const SahTask tk = tasks[w.task];
    const SahSplit s = splits[w.task];
    const unsigned first = w.a + threadIdx.x * kPer;
    bool go[kPer];
    unsigned p[kPer], mine = 0;
    for (int i = 0; i < kPer; i++) {
        const unsigned k = first + i;
        go[i] = false;
        p[i] = 0;
        if (k < w.e) {
            p[i] = perm[k];
            go[i] = sah_goes_left(s, cen[p[i]], k - tk.a);
            mine += go[i];
        }
    }
    // exclusive scan of the threads' left counts in position order
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned incl = mine;
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned v = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += v;
    }
    if (lane == 31) warp_sum[wid] = incl;
    __syncthreads();
    unsigned before = incl - mine;
    for (int i = 0; i < wid; i++) before += warp_sum[i];
    unsigned l = before, r = threadIdx.x * kPer - before;  // lefts / rights before this thread's first position
    const unsigned right_base = tk.a + s.ml + right_off[blockIdx.x];
    const unsigned left_base = tk.a + left_off[blockIdx.x];
    for (int i = 0; i < kPer; i++) {
        const unsigned k = first + i;
        if (k >= w.e) break;
        if (go[i])
            perm_out[left_base + l++] = p[i];
        else
            perm_out[right_base + r++] = p[i];
    }
}

// Nodes of the ranges split at their middle: children's boxes over the
// partitioned positions, one block per range.
__global__ void __launch_bounds__(kSahThreads) k_sah_middle_nodes(const SahTask* tasks, const unsigned* which,
                                                                  const SahSplit* splits, const unsigned* perm,
                                                                  const float4* blo, const float4* bhi,
                                                                  BvhNode* nodes)
{
    __shared__ float red[12];
    const unsigned t = which[blockIdx.x];
    const SahTask tk = tasks[t];
    const unsigned mid = tk.a + splits[t].ml;
    if (threadIdx.x < 12) red[threadIdx.x] = (threadIdx.x % 6) < 3 ? kSahEmptyLo : kSahEmptyHi;
    __syncthreads();
    float b[12];
    for (int k = 0; k < 12; k++) b[k] = (k % 6) < 3 ? kSahEmptyLo : kSahEmptyHi;
    for (unsigned k = tk.a + threadIdx.x; k < tk.e; k += blockDim.x) {
        const unsigned p = perm[k];
        const float4 l = blo[p], h = bhi[p];
        const float lv[3] = {l.x, l.y, l.z}, hv[3] = {h.x, h.y, h.z};
        float* side = k < mid ? b : b + 6;
        sah_grow(side, side + 3, lv, hv);
    }
    for (int k = 0; k < 12; k++) {
        if ((k % 6) < 3) atomic_min_f(&red[k], b[k]);
        else atomic_max_f(&red[k], b[k]);
    }
    __syncthreads();
    if (threadIdx.x == 0) sah_write_node(nodes, tk.slot, tk.a, tk.e - tk.a, splits[t].ml, red, red + 6);
}

// ---------------------------------------------------------------- small ranges, one thread each

// The same build, sequentially, of a range of at most kSahSmall primitives
// (scratch: the same positions of a second order array).
__global__ void k_sah_small(const SahTask* tasks, unsigned n_tasks, unsigned* perm, unsigned* scratch,
                            const float4* cen, const float4* blo, const float4* bhi, BvhNode* nodes)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    SahTask stack[kSahSmall];
    int sp = 0;
    stack[sp++] = tasks[t];
    while (sp > 0) {
        const SahTask tk = stack[--sp];
        const unsigned m = tk.e - tk.a;
        SahBins b;
        for (int k = 0; k < 3; k++) {
            b.cb[k] = kSahEmptyLo;
            b.cb[3 + k] = kSahEmptyHi;
        }
        for (unsigned k = tk.a; k < tk.e; k++) {
            const float4 c = cen[perm[k]];
            const float v[3] = {c.x, c.y, c.z};
            sah_grow(b.cb, b.cb + 3, v, v);
        }
        for (int ax = 0; ax < 3; ax++)
            for (int k = 0; k < kSahBins; k++) {
                b.count[ax][k] = 0;
                for (int q = 0; q < 6; q++) b.box[ax][k][q] = q < 3 ? kSahEmptyLo : kSahEmptyHi;
            }
        for (int ax = 0; ax < 3; ax++) {
            const float ext = __fsub_rn(b.cb[3 + ax], b.cb[ax]);
            if (!(ext > 0.f)) continue;
            const float scale = __fdiv_rn((float)kSahBins, ext);
            for (unsigned k = tk.a; k < tk.e; k++) {
                const unsigned p = perm[k];
                const float4 c = cen[p], l = blo[p], h = bhi[p];
                const float cv = ax == 0 ? c.x : (ax == 1 ? c.y : c.z);
                const int bi = sah_bin(cv, b.cb[ax], scale);
                const float lv[3] = {l.x, l.y, l.z}, hv[3] = {h.x, h.y, h.z};
                b.count[ax][bi]++;
                sah_grow(b.box[ax][bi], b.box[ax][bi] + 3, lv, hv);
            }
        }
        SahSplit s;
        float lb[6], rb[6];
        sah_choose(b, m, tk.depth, s, lb, rb);
        // stable partition through the scratch positions
        unsigned nl = 0;
        for (unsigned k = tk.a; k < tk.e; k++)
            if (sah_goes_left(s, cen[perm[k]], k - tk.a)) nl++;
        {
            unsigned l = 0, r = 0;
            for (unsigned k = tk.a; k < tk.e; k++) {
                const unsigned p = perm[k];
                if (sah_goes_left(s, cen[p], k - tk.a))
                    scratch[tk.a + l++] = p;
                else
                    scratch[tk.a + nl + r++] = p;
            }
            for (unsigned k = tk.a; k < tk.e; k++) perm[k] = scratch[k];
        }
        if (s.axis < 0) {
            for (int k = 0; k < 6; k++) {
                lb[k] = k < 3 ? kSahEmptyLo : kSahEmptyHi;
                rb[k] = k < 3 ? kSahEmptyLo : kSahEmptyHi;
            }
            for (unsigned k = tk.a; k < tk.e; k++) {
                const unsigned p = perm[k];
                const float4 l = blo[p], h = bhi[p];
                const float lv[3] = {l.x, l.y, l.z}, hv[3] = {h.x, h.y, h.z};
                float* side = k < tk.a + s.ml ? lb : rb;
                sah_grow(side, side + 3, lv, hv);
            }
        }
        sah_write_node(nodes, tk.slot, tk.a, m, s.ml, lb, rb);
        const unsigned ml = s.ml, mr = m - ml;
        // right pushed first: the left subtree's slots come first, either order builds the same tree
        if (mr >= 2) stack[sp++] = SahTask{tk.a + ml, tk.e, tk.slot + ml, tk.depth + 1};
        if (ml >= 2) stack[sp++] = SahTask{tk.a, tk.a + ml, tk.slot + 1, tk.depth + 1};
    }
}

// Leaf-order triangles: v0 (w = the triangle's original index), e1, e2.
__global__ void k_sah_leaf_tris(const float4* tri, const unsigned* perm, unsigned n, float4* out)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const unsigned p = perm[k];
    float4 a = tri[3 * (size_t)p];
    a.w = __int_as_float((int)p);
    out[3 * (size_t)k] = a;
    out[3 * (size_t)k + 1] = tri[3 * (size_t)p + 1];
    out[3 * (size_t)k + 2] = tri[3 * (size_t)p + 2];
}

}  // namespace upbp
