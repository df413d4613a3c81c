// Beam-map hierarchy by locally-ordered clustering (PLOC: Meister and
// Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
// Hierarchy Construction", IEEE TVCG 2018).  The chunks are sorted by the
// Morton code of their centres; every cluster then picks, among the
// kPlocRadius clusters on either side in that order, the one whose union
// with it has the smallest surface area, and mutual choices merge into a
// node.  Iterated to one cluster, this yields a tree of surface-area quality
// (the range searches visit fewer nodes than in the Morton-split LBVH) at
// the cost of a few linear passes per iteration.
//
// The tree is then laid out in the LBVH's node form (Karras 2012): the
// leaves in the tree's left-to-right order, and an internal node covering
// leaf range [a, b] with split g stored at b if it is a left child, at a if
// a right child (the root at 0), so that its children are g and g + 1.  Every
// internal node gets a distinct index that way, and the compressed nodes and
// all walks read the result exactly as an LBVH.  The layout is checked on
// the device (each index written once); the caller replaces the tree by the
// LBVH when the check fails or the passes run out.
#pragma once

#include "upbp_build.cuh"

namespace upbp {

constexpr int kPlocRadius = 16;    // clusters searched on each side in Morton order
constexpr int kPlocTail = 2048;    // clusters the one-block tail kernel finishes
constexpr int kPlocTailThreads = 1024;
constexpr int kPlocBlock = 256;
constexpr int kPlocTile = 1024;    // flags per tile of the compaction's prefix sum
constexpr int kPlocGrid = 148 * 8; // blocks of the many-cluster passes (grid-stride)
constexpr int kPlocTailIters = 4 * kPlocTail;  // at least one merge per iteration
constexpr int kPlocPasses = 96;    // most passes of the many-cluster phase

// Device-side state of a build (unsigned words): the many-cluster passes
// read their cluster count and buffer from the slots of their parity and
// write the next pass's, so the host launches a fixed sequence without
// reading anything back until the end.
enum : int {
    kPcNodes = 0,    // nodes created
    kPcLeft,         // clusters left after the tail (1: complete)
    kPcFail,         // layout check failures
    kPcTailIters,    // iterations of the tail
    kPcM0,           // clusters at the start of an even / odd pass
    kPcM1,
    kPcCur0,         // cluster buffer of an even / odd pass
    kPcCur1,
    kPcPasses,       // passes that merged
    kPcN,            // leaves
    kPcBounds = 16,  // nodes created before pass t (kPlocPasses + 1 words)
    kPcWords = kPcBounds + kPlocPasses + 1
};

// A cluster is two float4: (lo, id) and (hi, leaf count), id >= 0 a created
// node, id < 0 the complement of a leaf's Morton position.
struct PlocScratch {
    unsigned capacity = 0;
    float4* cl[2] = {nullptr, nullptr};
    float4* leaf = nullptr;        // leaf boxes in Morton order: (lo, 0), (hi, 0)
    int* nn = nullptr;
    unsigned* flag = nullptr;
    unsigned* tile_sum = nullptr;  // per tile of kPlocTile flags, then its exclusive prefix
    float4* node_box = nullptr;    // per created node: (lo, leaf count), (hi, 0)
    int2* node_child = nullptr;
    int2* node_place = nullptr;    // (first leaf position, index in the laid-out tree)
    unsigned* written = nullptr;   // writes per laid-out node index (the check)
    unsigned* order = nullptr;     // laid-out leaf order: chunk per leaf position
    unsigned* count = nullptr;     // kPcWords words
    // the launches after the leaves are set up, captured once as a graph
    // (they read everything that varies from device memory); re-captured
    // when the pass budget or a buffer changes
    cudaStream_t capture = nullptr;
    cudaGraphExec_t exec = nullptr;
    int exec_budget = -1;
    const void* exec_nodes = nullptr;
    const void* exec_vals = nullptr;
};

UPBP_D float ploc_area(float3 lo, float3 hi)
{
    const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    return dx * dy + dy * dz + dz * dx;
}

UPBP_D float3 min3f(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
UPBP_D float3 max3f(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

// Leaves in Morton order (vals: chunk per Morton position).
__global__ void k_ploc_init(BoxSource src, const unsigned* vals, unsigned n, float4* cl, float4* leaf)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 lo, hi;
    source_box(src, vals[i], lo, hi);
    cl[2 * i] = make_float4(lo.x, lo.y, lo.z, __int_as_float(~(int)i));
    cl[2 * i + 1] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(1u));
    leaf[2 * i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    leaf[2 * i + 1] = make_float4(hi.x, hi.y, hi.z, 0.f);
}

// Cluster count and buffer of pass t; 0 clusters once the tail's size is
// reached (the pass does nothing).
UPBP_D unsigned ploc_pass_m(const unsigned* count, int t, const float4* cl0, const float4* cl1, const float4*& cl)
{
    const unsigned m = count[kPcM0 + (t & 1)];
    cl = count[kPcCur0 + (t & 1)] ? cl1 : cl0;
    return m > (unsigned)kPlocTail ? m : 0u;
}

// Nearest neighbour (smallest union area, ties to the lower index) of each of
// the m clusters within kPlocRadius positions; tiles of kPlocBlock clusters,
// each with its window in shared memory.
__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const float4* cl0, const float4* cl1, const unsigned* count,
                                                        int t, int* nn)
{
    __shared__ float4 s_lo[kPlocBlock + 2 * kPlocRadius], s_hi[kPlocBlock + 2 * kPlocRadius];
    const float4* cl;
    const unsigned m = ploc_pass_m(count, t, cl0, cl1, cl);
    for (unsigned tile = blockIdx.x; tile * kPlocBlock < m; tile += gridDim.x) {
        const int base = (int)(tile * kPlocBlock);
        __syncthreads();
        for (int q = threadIdx.x; q < kPlocBlock + 2 * kPlocRadius; q += blockDim.x) {
            const int j = base - kPlocRadius + q;
            if (j >= 0 && j < (int)m) {
                s_lo[q] = cl[2 * j];
                s_hi[q] = cl[2 * j + 1];
            }
        }
        __syncthreads();
        const int i = base + (int)threadIdx.x;
        if (i < (int)m) {
            const int ti = (int)threadIdx.x + kPlocRadius;
            const float3 lo = xyz(s_lo[ti]), hi = xyz(s_hi[ti]);
            float best = INFINITY;
            int bj = -1;
            const int j0 = max(0, i - kPlocRadius), j1 = min((int)m - 1, i + kPlocRadius);
            for (int j = j0; j <= j1; j++) {
                if (j == i) continue;
                const int tj = j - base + kPlocRadius;
                const float ar = ploc_area(min3f(lo, xyz(s_lo[tj])), max3f(hi, xyz(s_hi[tj])));
                if (ar < best || bj < 0) {  // strict: among equal areas the lowest index, met first
                    best = ar;
                    bj = j;
                }
            }
            nn[i] = bj;
        }
    }
}

// Block-wide exclusive prefix of one value per thread (blockDim.x a
// multiple of 32, at most 1024); returns the prefix, *total the sum.
UPBP_D unsigned ploc_block_scan(unsigned v, unsigned* s_warp, unsigned* total)
{
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned u = __shfl_up_sync(~0u, incl, o);
        if (lane >= (unsigned)o) incl += u;
    }
    __syncthreads();
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        unsigned w = lane < nw ? s_warp[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(~0u, w, o);
            if (lane >= (unsigned)o) w += u;
        }
        if (lane < nw) s_warp[lane] = w;
    }
    __syncthreads();
    *total = s_warp[nw - 1];
    return incl - v + (wid > 0 ? s_warp[wid - 1] : 0u);
}

// Mutual nearest neighbours merge: the lower index creates the node and
// takes its place, the higher one leaves (flag 0).  Tiles of kPlocTile
// clusters, four consecutive ones per thread; each tile's count of clusters
// that stay goes to tile_sum.
__global__ void __launch_bounds__(kPlocBlock) k_ploc_merge(float4* cl0, float4* cl1, unsigned* count, int t,
                                                           const int* nn, float4* node_box, int2* node_child,
                                                           unsigned* flag, unsigned* tile_sum)
{
    __shared__ unsigned s_warp[32];
    const float4* clr;
    const unsigned m = ploc_pass_m(count, t, cl0, cl1, clr);
    float4* cl = const_cast<float4*>(clr);
    constexpr int per = kPlocTile / kPlocBlock;
    for (unsigned tile = blockIdx.x; tile * kPlocTile < m; tile += gridDim.x) {
        unsigned v = 0;
        for (int q = 0; q < per; q++) {
            const unsigned i = tile * kPlocTile + threadIdx.x * per + q;
            if (i >= m) break;
            const int j = nn[i];
            unsigned f = 1u;
            if (j >= 0 && nn[j] == (int)i) {
                if ((int)i > j) {
                    f = 0u;
                } else {
                    const float4 a0 = cl[2 * i], a1 = cl[2 * i + 1], b0 = cl[2 * j], b1 = cl[2 * j + 1];
                    const float3 lo = min3f(xyz(a0), xyz(b0)), hi = max3f(xyz(a1), xyz(b1));
                    const unsigned cnt = __float_as_uint(a1.w) + __float_as_uint(b1.w);
                    const unsigned k = atomicAdd(&count[kPcNodes], 1u);
                    node_box[2 * k] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(cnt));
                    node_box[2 * k + 1] = make_float4(hi.x, hi.y, hi.z, 0.f);
                    node_child[k] = make_int2(__float_as_int(a0.w), __float_as_int(b0.w));
                    cl[2 * i] = make_float4(lo.x, lo.y, lo.z, __int_as_float((int)k));
                    cl[2 * i + 1] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(cnt));
                }
            }
            flag[i] = f;
            v += f;
        }
        unsigned total;
        ploc_block_scan(v, s_warp, &total);
        if (threadIdx.x == 0) tile_sum[tile] = total;
    }
}

// Exclusive prefix of the tile sums (one block), and the next pass's cluster
// count, buffer and node bound.  A pass that does nothing carries its state
// over.
__global__ void __launch_bounds__(1024) k_ploc_tile_scan(unsigned* count, int t, unsigned* tile_sum)
{
    __shared__ unsigned s_warp[32];
    const unsigned m = count[kPcM0 + (t & 1)], cur = count[kPcCur0 + (t & 1)];
    const int nx = (t + 1) & 1;
    if (m <= (unsigned)kPlocTail) {
        if (threadIdx.x == 0) {
            count[kPcM0 + nx] = m;
            count[kPcCur0 + nx] = cur;
            count[kPcBounds + t + 1] = count[kPcNodes];
        }
        return;
    }
    const unsigned nt = (m + kPlocTile - 1) / kPlocTile;
    const unsigned per = (nt + blockDim.x - 1) / blockDim.x;
    unsigned v = 0;
    for (unsigned q = 0; q < per; q++) {
        const unsigned i = threadIdx.x * per + q;
        if (i < nt) v += tile_sum[i];
    }
    unsigned total;
    unsigned at = ploc_block_scan(v, s_warp, &total);
    for (unsigned q = 0; q < per; q++) {
        const unsigned i = threadIdx.x * per + q;
        if (i < nt) {
            const unsigned x = tile_sum[i];
            tile_sum[i] = at;
            at += x;
        }
    }
    if (threadIdx.x == 0) {
        count[kPcM0 + nx] = total;
        count[kPcCur0 + nx] = cur ^ 1u;
        count[kPcBounds + t + 1] = count[kPcNodes];
        count[kPcPasses] += 1u;
    }
}

// The clusters that stay, in order, into the other buffer.
__global__ void __launch_bounds__(kPlocBlock) k_ploc_compact(float4* cl0, float4* cl1, const unsigned* count, int t,
                                                             const unsigned* flag, const unsigned* tile_off)
{
    __shared__ unsigned s_warp[32];
    const float4* cl;
    const unsigned m = ploc_pass_m(count, t, cl0, cl1, cl);
    float4* out = cl == cl0 ? cl1 : cl0;
    constexpr int per = kPlocTile / kPlocBlock;
    for (unsigned tile = blockIdx.x; tile * kPlocTile < m; tile += gridDim.x) {
        const unsigned first = tile * kPlocTile + threadIdx.x * per;
        unsigned f[per], v = 0;
        for (int q = 0; q < per; q++) {
            f[q] = first + q < m ? flag[first + q] : 0u;
            v += f[q];
        }
        unsigned total;
        unsigned at = tile_off[tile] + ploc_block_scan(v, s_warp, &total);
        for (int q = 0; q < per; q++)
            if (f[q]) {
                out[2 * at] = cl[2 * (first + q)];
                out[2 * at + 1] = cl[2 * (first + q) + 1];
                at++;
            }
    }
}

// Places the children of created node k: writes the laid-out node at its
// index (children's boxes and links), the children's places, and the leaf
// order at the leaves' positions.
UPBP_D void ploc_place(unsigned k, unsigned n, const float4* leaf, const unsigned* vals, const float4* node_box,
                       const int2* node_child, int2* node_place, unsigned* written, unsigned* order, BvhNode* nodes,
                       unsigned* count)
{
    const int2 pl = node_place[k];
    if (pl.x < 0 || pl.y < 0 || pl.y >= (int)n - 1) {  // a place never written: the check fails
        atomicAdd(&count[kPcFail], 1u);
        return;
    }
    const int2 ch = node_child[k];
    const int c[2] = {ch.x, ch.y};
    float3 lo[2], hi[2];
    unsigned cnt[2];
    for (int s = 0; s < 2; s++) {
        if (c[s] < 0) {
            lo[s] = xyz(leaf[2 * ~c[s]]);
            hi[s] = xyz(leaf[2 * ~c[s] + 1]);
            cnt[s] = 1u;
        } else {
            const float4 b0 = node_box[2 * c[s]], b1 = node_box[2 * c[s] + 1];
            lo[s] = xyz(b0);
            hi[s] = xyz(b1);
            cnt[s] = __float_as_uint(b0.w);
        }
    }
    const int g = pl.x + (int)cnt[0] - 1;
    if (g < pl.x || g + 1 >= (int)n) {
        atomicAdd(&count[kPcFail], 1u);
        return;
    }
    BvhNode& nd = nodes[pl.y];
    nd.a = make_float4(lo[0].x, lo[0].y, lo[0].z, hi[0].x);
    nd.b = make_float4(hi[0].y, hi[0].z, lo[1].x, lo[1].y);
    nd.c = make_float4(lo[1].z, hi[1].x, hi[1].y, hi[1].z);
    nd.link = make_int4(c[0] < 0 ? ~g : g, c[1] < 0 ? ~(g + 1) : g + 1, (int)cnt[0], (int)cnt[1]);
    atomicAdd(&written[pl.y], 1u);
    if (c[0] < 0)
        order[g] = vals[~c[0]];
    else
        node_place[c[0]] = make_int2(pl.x, g);
    if (c[1] < 0)
        order[g + 1] = vals[~c[1]];
    else
        node_place[c[1]] = make_int2(g + 1, g + 1);
}

// The last m <= kPlocTail clusters (the state after `passes` passes),
// merged to one by a single block in shared memory, then the places of the
// nodes it created (last first; the root at leaf position 0 and index 0).
// count[kPcTailIters] receives its iterations, count[kPcLeft] the clusters
// left (1 when it completed; the passes' count when they ran out).
__global__ void __launch_bounds__(kPlocTailThreads) k_ploc_tail(const float4* cl0, const float4* cl1, int passes,
                                                                 const float4* leaf, const unsigned* vals,
                                                                 unsigned* count,
                                                                 float4* node_box, int2* node_child,
                                                                 int2* node_place, unsigned* written,
                                                                 unsigned* order, BvhNode* nodes)
{
    extern __shared__ float4 smem[];
    float4* s_lo = smem;
    float4* s_hi = s_lo + kPlocTail;
    int* s_nn = reinterpret_cast<int*>(s_hi + kPlocTail);
    unsigned* s_flag = reinterpret_cast<unsigned*>(s_nn + kPlocTail);
    unsigned* s_bounds = s_flag + kPlocTail;  // kPlocTailIters + 1 node counts
    __shared__ unsigned s_nodes, s_m, s_warp[kPlocTailThreads / 32];
    const unsigned tid = threadIdx.x;
    const unsigned node_base = count[kPcNodes];
    const unsigned n = count[kPcN];
    // the state after the last pass of the many-cluster phase
    const unsigned m = count[kPcM0 + (passes & 1)];
    const float4* cl = count[kPcCur0 + (passes & 1)] ? cl1 : cl0;
    if (m > (unsigned)kPlocTail) {  // the passes ran out: the caller falls back
        if (tid == 0) count[kPcLeft] = m;
        return;
    }
    for (unsigned i = tid; i < m; i += blockDim.x) {
        s_lo[i] = cl[2 * i];
        s_hi[i] = cl[2 * i + 1];
    }
    if (tid == 0) {
        s_nodes = 0;
        s_m = m;
        s_bounds[0] = 0;
    }
    __syncthreads();
    int it = 0;
    while (s_m > 1 && it < kPlocTailIters) {
        const int mm = (int)s_m;
        for (int i = (int)tid; i < mm; i += blockDim.x) {
            const float3 lo = xyz(s_lo[i]), hi = xyz(s_hi[i]);
            float best = INFINITY;
            int bj = -1;
            const int j0 = max(0, i - kPlocRadius), j1 = min(mm - 1, i + kPlocRadius);
            for (int j = j0; j <= j1; j++) {
                if (j == i) continue;
                const float a = ploc_area(min3f(lo, xyz(s_lo[j])), max3f(hi, xyz(s_hi[j])));
                if (a < best || bj < 0) {
                    best = a;
                    bj = j;
                }
            }
            s_nn[i] = bj;
        }
        __syncthreads();
        for (int i = (int)tid; i < mm; i += blockDim.x) {
            const int j = s_nn[i];
            unsigned f = 1u;
            if (j >= 0 && s_nn[j] == i) {
                if (i < j) {
                    const float4 a0 = s_lo[i], a1 = s_hi[i], b0 = s_lo[j], b1 = s_hi[j];
                    const float3 lo = min3f(xyz(a0), xyz(b0)), hi = max3f(xyz(a1), xyz(b1));
                    const unsigned cnt = __float_as_uint(a1.w) + __float_as_uint(b1.w);
                    const unsigned k = node_base + atomicAdd(&s_nodes, 1u);
                    node_box[2 * k] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(cnt));
                    node_box[2 * k + 1] = make_float4(hi.x, hi.y, hi.z, 0.f);
                    node_child[k] = make_int2(__float_as_int(a0.w), __float_as_int(b0.w));
                    s_lo[i] = make_float4(lo.x, lo.y, lo.z, __int_as_float((int)k));
                    s_hi[i] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(cnt));
                } else {
                    f = 0u;
                }
            }
            s_flag[i] = f;
        }
        __syncthreads();
        // exclusive prefix of the flags, two entries per thread, then the
        // compaction through registers
        const int per = (kPlocTail + kPlocTailThreads - 1) / kPlocTailThreads;
        unsigned mine = 0;
        for (int q = 0; q < per; q++) {
            const int i = (int)tid * per + q;
            if (i < mm) mine += s_flag[i];
        }
        const unsigned lane = tid & 31u, wid = tid >> 5;
        unsigned incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(~0u, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            unsigned w = lane < kPlocTailThreads / 32 ? s_warp[lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned v = __shfl_up_sync(~0u, w, o);
                if (lane >= (unsigned)o) w += v;
            }
            if (lane < kPlocTailThreads / 32) s_warp[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        unsigned at = incl - mine + (wid > 0 ? s_warp[wid - 1] : 0u);
        float4 keep_lo[per], keep_hi[per];
        unsigned keep_flag[per];
        for (int q = 0; q < per; q++) {
            const int i = (int)tid * per + q;
            keep_flag[q] = i < mm ? s_flag[i] : 0u;
            if (keep_flag[q]) {
                keep_lo[q] = s_lo[i];
                keep_hi[q] = s_hi[i];
            }
        }
        __syncthreads();
        for (int q = 0; q < per; q++) {
            if (keep_flag[q]) {
                s_lo[at] = keep_lo[q];
                s_hi[at] = keep_hi[q];
                at++;
            }
        }
        if (tid == kPlocTailThreads - 1) {
            s_m = s_warp[kPlocTailThreads / 32 - 1];
            s_bounds[it + 1] = s_nodes;
        }
        it++;
        __syncthreads();
    }
    if (tid == 0) {
        count[kPcLeft] = s_m;
        count[kPcTailIters] = (unsigned)it;
        count[kPcNodes] = node_base + s_nodes;
    }
    if (s_m != 1) return;  // the caller sees count[1] != 1 and falls back
    // places, last created first: the root is the last node of all
    const unsigned root = node_base + s_nodes - 1u;
    if (tid == 0) node_place[root] = make_int2(0, 0);
    __syncthreads();
    for (int t = it - 1; t >= 0; t--) {
        for (unsigned k = s_bounds[t] + tid; k < s_bounds[t + 1]; k += blockDim.x)
            ploc_place(node_base + k, n, leaf, vals, node_box, node_child, node_place, written, order, nodes, count);
        __syncthreads();
    }
}

// Places of the nodes created in pass t of the many-cluster phase.
__global__ void k_ploc_place(int t, const float4* leaf, const unsigned* vals, const float4* node_box,
                             const int2* node_child, int2* node_place, unsigned* written, unsigned* order,
                             BvhNode* nodes, unsigned* count)
{
    const unsigned k0 = count[kPcBounds + t], k1 = count[kPcBounds + t + 1], n = count[kPcN];
    for (unsigned k = k0 + blockIdx.x * blockDim.x + threadIdx.x; k < k1; k += gridDim.x * blockDim.x)
        ploc_place(k, n, leaf, vals, node_box, node_child, node_place, written, order, nodes, count);
}

// The check: every internal index of the laid-out tree written exactly once
// (then each node's children cover disjoint, smaller leaf ranges, and every
// walk ends).
__global__ void k_ploc_check(const unsigned* written, unsigned* count)
{
    const unsigned n_internal = count[kPcN] - 1u;
    unsigned bad = 0;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n_internal; i += gridDim.x * blockDim.x)
        bad += written[i] != 1u;
    if (bad) atomicAdd(&count[kPcFail], bad);
}

inline size_t ploc_tail_smem() { return (size_t)kPlocTail * 2 * sizeof(float4) + (size_t)kPlocTail * 8 + (kPlocTailIters + 1) * 4; }

// Builds the n-leaf tree (n >= 2) over the boxes of `src` into `nodes`
// (n - 1 nodes) and its leaf order (*sorted_vals): a fixed sequence of
// launches (`budget` passes, at most kPlocPasses; a pass that finds the
// tail's size reached does nothing), and a copy of the outcome into the
// page-locked words `outcome` (kPcWords).  Nothing waits for it: the caller
// reads the outcome with ploc_complete after its next synchronisation with
// the stream, and until then uses the tree for nothing; a tree that is not
// complete (the passes ran out -- boxes so alike that few merge per pass --
// or the layout check failed) is replaced.
inline cudaError_t build_ploc(const BoxSource& src, unsigned n, BvhNode* nodes, BuildScratch& sc, PlocScratch& ps,
                              cudaStream_t st, const unsigned** sorted_vals, unsigned* launches, unsigned* outcome,
                              int budget)
{
    budget = std::max(1, std::min(budget, kPlocPasses));
    if (n < 2 || n > ps.capacity) return cudaErrorInvalidValue;
    // Morton order of the centres
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    cudaError_t e = cudaMemcpyAsync(sc.ord6, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const unsigned bs = 256;
    const unsigned grid = (n + bs - 1) / bs;
    k_bounds<<<grid < 1184 ? grid : 1184, bs, 0, st>>>(src, n, sc.ord6);
    k_morton<<<grid, bs, 0, st>>>(src, n, sc.ord6, sc.keys, sc.vals);
    cub::DoubleBuffer<unsigned> kb(sc.keys, sc.keys_alt), vb(sc.vals, sc.vals_alt);
    size_t tb = sc.temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(sc.temp, tb, kb, vb, (int)n, 0, 30, st);
    if (e != cudaSuccess) return e;
    const unsigned* vals = vb.Current();
    // state: n clusters in buffer 0, no nodes
    static thread_local unsigned h_init[kPcWords];
    for (int i = 0; i < kPcWords; i++) h_init[i] = 0u;
    h_init[kPcM0] = n;
    h_init[kPcN] = n;
    e = cudaMemcpyAsync(ps.count, h_init, sizeof(h_init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(ps.written, 0, (size_t)(n - 1) * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    k_ploc_init<<<grid, bs, 0, st>>>(src, vals, n, ps.cl[0], ps.leaf);
    const size_t smem = ploc_tail_smem();
    e = cudaFuncSetAttribute(k_ploc_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the passes, the tail, the places and the check: the same launches for
    // every build with this budget and these buffers
    auto sequence = [&](cudaStream_t s) {
        const unsigned g = kPlocGrid;
        for (int t = 0; t < budget; t++) {
            k_ploc_nn<<<g, kPlocBlock, 0, s>>>(ps.cl[0], ps.cl[1], ps.count, t, ps.nn);
            k_ploc_merge<<<g, kPlocBlock, 0, s>>>(ps.cl[0], ps.cl[1], ps.count, t, ps.nn, ps.node_box,
                                                  ps.node_child, ps.flag, ps.tile_sum);
            k_ploc_tile_scan<<<1, 1024, 0, s>>>(ps.count, t, ps.tile_sum);
            k_ploc_compact<<<g, kPlocBlock, 0, s>>>(ps.cl[0], ps.cl[1], ps.count, t, ps.flag, ps.tile_sum);
        }
        k_ploc_tail<<<1, kPlocTailThreads, smem, s>>>(ps.cl[0], ps.cl[1], budget, ps.leaf, vals, ps.count,
                                                      ps.node_box, ps.node_child, ps.node_place, ps.written,
                                                      ps.order, nodes);
        // places of the many-cluster phase's nodes, last pass first (a pass
        // that merged nothing has an empty range)
        for (int t = budget - 1; t >= 0; t--)
            k_ploc_place<<<g, bs, 0, s>>>(t, ps.leaf, vals, ps.node_box, ps.node_child, ps.node_place, ps.written,
                                          ps.order, nodes, ps.count);
        k_ploc_check<<<g, bs, 0, s>>>(ps.written, ps.count);
    };
    if (!ps.exec || ps.exec_budget != budget || ps.exec_nodes != nodes || ps.exec_vals != vals) {
        if (ps.exec) cudaGraphExecDestroy(ps.exec);
        ps.exec = nullptr;
        cudaGraph_t graph = nullptr;
        if (ps.capture && cudaStreamBeginCapture(ps.capture, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            sequence(ps.capture);
            if (cudaStreamEndCapture(ps.capture, &graph) == cudaSuccess && graph) {
                if (cudaGraphInstantiate(&ps.exec, graph, 0) != cudaSuccess) ps.exec = nullptr;
                cudaGraphDestroy(graph);
            }
        }
        cudaGetLastError();
        ps.exec_budget = budget;
        ps.exec_nodes = nodes;
        ps.exec_vals = vals;
    }
    if (ps.exec) {
        e = cudaGraphLaunch(ps.exec, st);
        if (e != cudaSuccess) return e;
    } else {
        sequence(st);  // without a graph (capture unavailable)
    }
    *launches += 7 + 5 * budget;
    e = cudaMemcpyAsync(outcome, ps.count, kPcWords * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    *sorted_vals = ps.order;
    return cudaGetLastError();
}

// Whether the build whose outcome words these are (n leaves) produced a
// complete, checked tree.
inline bool ploc_complete(const unsigned* outcome, unsigned n)
{
    return outcome[kPcLeft] == 1u && outcome[kPcNodes] == n - 1 && outcome[kPcFail] == 0u;
}

}  // namespace upbp
