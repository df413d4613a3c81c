// GPU LBVH construction (Karras 2012, "Maximizing parallelism in the
// construction of BVHs, octrees, and k-d trees"): 30-bit Morton codes of box
// centroids, radix sort, one thread per internal node for the hierarchy,
// bottom-up refit with one atomic flag per node.  Used once for the scene
// triangles and every iteration for the photon-point and photon-beam maps.
#pragma once

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "upbp_device.cuh"

namespace upbp {

UPBP_D unsigned expand_bits10(unsigned v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

UPBP_D unsigned morton3(float3 c)
{
    const float x = fminf(fmaxf(c.x * 1024.f, 0.f), 1023.f);
    const float y = fminf(fmaxf(c.y * 1024.f, 0.f), 1023.f);
    const float z = fminf(fmaxf(c.z * 1024.f, 0.f), 1023.f);
    return (expand_bits10((unsigned)x) << 2) | (expand_bits10((unsigned)y) << 1) | expand_bits10((unsigned)z);
}

// Order-preserving float <-> uint maps for atomic min/max of bounds.
UPBP_HD unsigned f2ord(float f)
{
#ifdef __CUDA_ARCH__
    unsigned u = __float_as_uint(f);
#else
    unsigned u;
    memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
UPBP_HD float ord2f(unsigned u)
{
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

// Primitive source for a build: a box per primitive.
struct BoxSource {
    int kind;                 // 0: triangles (v0,e1,e2 x3 float4), 1: points via slot list, 2: beams, 3: beam chunks
    const float4* tri;        // kind 0: unsorted triangle float4 triples
    const unsigned* slots;    // kind 1: vertex slots
    const LightVertexRec* vertices;
    const BeamRec* beams;     // kind 2
    unsigned bb1d_paths;      // kind 2: beams of paths below this index serve BB1D
    const uint2* chunks;      // kind 3: (beam index, chunk k | chunk count << 16)
    float dilate;             // kinds 1, 3: leaf boxes grown by this much (the maps' query radius)
};

UPBP_D void source_box(const BoxSource& s, unsigned i, float3& lo, float3& hi)
{
    if (s.kind == 0) {
        const float3 v0 = xyz(s.tri[3 * i]), e1 = xyz(s.tri[3 * i + 1]), e2 = xyz(s.tri[3 * i + 2]);
        const float3 v1 = v0 + e1, v2 = v0 + e2;
        lo = make_float3(fminf(v0.x, fminf(v1.x, v2.x)), fminf(v0.y, fminf(v1.y, v2.y)), fminf(v0.z, fminf(v1.z, v2.z)));
        hi = make_float3(fmaxf(v0.x, fmaxf(v1.x, v2.x)), fmaxf(v0.y, fmaxf(v1.y, v2.y)), fmaxf(v0.z, fmaxf(v1.z, v2.z)));
        // the box of v0 + e1 may miss v1 by one rounding step; widen slightly
        const float3 ext = (hi - lo) * 1e-6f + v3(1e-7f * (fabsf(lo.x) + fabsf(lo.y) + fabsf(lo.z) + 1e-3f));
        lo = lo - ext;
        hi = hi + ext;
    } else if (s.kind == 1) {
        const float3 p = xyz(s.vertices[s.slots[i]].q[0]);
        lo = hi = p;
        dilate_box(lo, hi, s.dilate);
    } else if (s.kind == 2) {
        const float4 a = s.beams[i].q[0], b = s.beams[i].q[1];
        const float3 o = xyz(a), e = xyz(a) + xyz(b) * a.w;
        lo = make_float3(fminf(o.x, e.x), fminf(o.y, e.y), fminf(o.z, e.z));
        hi = make_float3(fmaxf(o.x, e.x), fmaxf(o.y, e.y), fmaxf(o.z, e.z));
    } else {
        const uint2 ch = s.chunks[i];
        const float4 a = s.beams[ch.x].q[0], b = s.beams[ch.x].q[1];
        chunk_box(xyz(a), xyz(b), a.w, ch.y & 0xffffu, ch.y >> 16, lo, hi);
        dilate_box(lo, hi, s.dilate);
    }
}

__global__ void k_bounds(BoxSource s, unsigned n, unsigned* ord6)
{
    __shared__ unsigned sh[6][32];
    float3 lo = v3(1e30f), hi = v3(-1e30f);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float3 a, b;
        source_box(s, i, a, b);
        const float3 c = (a + b) * .5f;
        lo = make_float3(fminf(lo.x, c.x), fminf(lo.y, c.y), fminf(lo.z, c.z));
        hi = make_float3(fmaxf(hi.x, c.x), fmaxf(hi.y, c.y), fmaxf(hi.z, c.z));
    }
    unsigned v[6] = {f2ord(lo.x), f2ord(lo.y), f2ord(lo.z), f2ord(hi.x), f2ord(hi.y), f2ord(hi.z)};
    for (int k = 0; k < 6; k++) {
        unsigned x = v[k];
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned y = __shfl_xor_sync(0xffffffffu, x, off);
            x = k < 3 ? min(x, y) : max(x, y);
        }
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        unsigned x = sh[k][0];
        for (unsigned w = 1; w < blockDim.x / 32; w++) x = k < 3 ? min(x, sh[k][w]) : max(x, sh[k][w]);
        if (k < 3)
            atomicMin(&ord6[k], x);
        else
            atomicMax(&ord6[k], x);
    }
}

__global__ void k_morton(BoxSource s, unsigned n, const unsigned* ord6, unsigned* keys, unsigned* vals)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 lo = make_float3(ord2f(ord6[0]), ord2f(ord6[1]), ord2f(ord6[2]));
    const float3 hi = make_float3(ord2f(ord6[3]), ord2f(ord6[4]), ord2f(ord6[5]));
    const float3 ext = hi - lo;
    const float3 inv = make_float3(ext.x > 0.f ? 1.f / ext.x : 0.f, ext.y > 0.f ? 1.f / ext.y : 0.f,
                                   ext.z > 0.f ? 1.f / ext.z : 0.f);
    float3 a, b;
    source_box(s, i, a, b);
    keys[i] = morton3(((a + b) * .5f - lo) * inv);
    vals[i] = i;
}

UPBP_D int lbvh_delta(const unsigned* k, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const unsigned a = k[i], b = k[j];
    if (a == b) return 32 + __clz((unsigned)(i ^ j));
    return __clz(a ^ b);
}

__global__ void k_hierarchy(const unsigned* keys, int n, BvhNode* nodes, int* parent_internal, int* parent_leaf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (lbvh_delta(keys, n, i, i + 1) - lbvh_delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = lbvh_delta(keys, n, i, i - d);
    int lmax = 2;
    while (lbvh_delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (lbvh_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = lbvh_delta(keys, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) / 2;
        if (lbvh_delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int left = (min(i, j) == gamma) ? ~gamma : gamma;
    const int right = (max(i, j) == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    // z, w: primitives under the left and right child
    nodes[i].link = make_int4(left, right, gamma - min(i, j) + 1, max(i, j) - gamma);
    if (left < 0)
        parent_leaf[~left] = i;
    else
        parent_internal[left] = i;
    if (right < 0)
        parent_leaf[~right] = i;
    else
        parent_internal[right] = i;
}

UPBP_D void write_child_box(BvhNode* node, bool left, float3 lo, float3 hi)
{
    float* f = reinterpret_cast<float*>(node);
    if (left) {
        f[0] = lo.x;
        f[1] = lo.y;
        f[2] = lo.z;
        f[3] = hi.x;
        f[4] = hi.y;
        f[5] = hi.z;
    } else {
        f[6] = lo.x;
        f[7] = lo.y;
        f[8] = lo.z;
        f[9] = hi.x;
        f[10] = hi.y;
        f[11] = hi.z;
    }
}

__global__ void k_refit(BoxSource s, int n, const unsigned* vals, BvhNode* nodes, const int* parent_internal,
                        const int* parent_leaf, unsigned* flags)
{
    const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n || n < 2) return;
    float3 lo, hi;
    source_box(s, vals[leaf], lo, hi);
    int node = parent_leaf[leaf];
    int child = ~leaf;
    // bounded by the tree depth (< n); every step moves one level up
    for (int guard = 0; guard < n; guard++) {
        const int4 link = __ldcg(&nodes[node].link);
        write_child_box(&nodes[node], link.x == child, lo, hi);
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0u) return;
        __threadfence();
        const float* f = reinterpret_cast<const float*>(&nodes[node]);
        float v[12];
        for (int k = 0; k < 12; k++) v[k] = __ldcg(f + k);
        lo = make_float3(fminf(v[0], v[6]), fminf(v[1], v[7]), fminf(v[2], v[8]));
        hi = make_float3(fmaxf(v[3], v[9]), fmaxf(v[4], v[10]), fmaxf(v[5], v[11]));
        if (node == 0) return;
        child = node;
        node = parent_internal[node];
    }
}

// Smallest biased exponent e (1..254) with origin + 255 * 2^(e-127) >= hi
// in the decoder's arithmetic.
UPBP_D unsigned qnode_exponent(float origin, float hi)
{
    const float t = (hi - origin) * (1.f / 255.f);
    unsigned e = t > 0.f ? ((__float_as_uint(t) >> 23) & 0xffu) + 1u : 1u;
    e = min(max(e, 1u), 254u);
    while (e < 254u && __fmaf_rn(255.f, qnode_step(e), origin) < hi) e++;
    return e;
}

// Byte q with origin + q * step <= v (lower plane) or >= v (upper plane),
// as tight as the step allows; v lies in [origin, origin + 255 * step].
UPBP_D unsigned qnode_quantize(float v, float origin, float step, bool upper)
{
    const float f = (v - origin) / step;
    int q = upper ? (int)ceilf(f) : (int)floorf(f);
    q = min(max(q, 0), 255);
    // at most 255 steps: q = 0 decodes to origin <= v, q = 255 to >= hi >= v
    if (upper) {
        while (q < 255 && __fmaf_rn((float)q, step, origin) < v) q++;
    } else {
        while (q > 0 && __fmaf_rn((float)q, step, origin) > v) q--;
    }
    return (unsigned)q;
}

// Compressed copy of the n - 1 internal nodes of a tree built with
// one-primitive leaves (every child link is gamma or gamma + 1).
__global__ void k_quantize(const BvhNode* nodes, int n_internal, QNode* q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_internal) return;
    const float4 a = nodes[i].a, b = nodes[i].b, c = nodes[i].c;
    const int4 k = nodes[i].link;
    const float lo[2][3] = {{a.x, a.y, a.z}, {b.z, b.w, c.x}};
    const float hi[2][3] = {{a.w, b.x, b.y}, {c.y, c.z, c.w}};
    float org[3], step[3];
    unsigned ebits = 0;
    for (int ax = 0; ax < 3; ax++) {
        org[ax] = fminf(lo[0][ax], lo[1][ax]);
        const unsigned e = qnode_exponent(org[ax], fmaxf(hi[0][ax], hi[1][ax]));
        step[ax] = qnode_step(e);
        ebits |= e << (8 * ax);
    }
    unsigned bytes[12];
    for (int ch = 0; ch < 2; ch++)
        for (int ax = 0; ax < 3; ax++) {
            bytes[6 * ch + ax] = qnode_quantize(lo[ch][ax], org[ax], step[ax], false);
            bytes[6 * ch + 3 + ax] = qnode_quantize(hi[ch][ax], org[ax], step[ax], true);
        }
    uint4 w;
    w.x = bytes[0] | bytes[1] << 8 | bytes[2] << 16 | bytes[3] << 24;
    w.y = bytes[4] | bytes[5] << 8 | bytes[6] << 16 | bytes[7] << 24;
    w.z = bytes[8] | bytes[9] << 8 | bytes[10] << 16 | bytes[11] << 24;
    const unsigned g = (unsigned)(k.x < 0 ? leaf_first(k.x) : k.x);
    w.w = g | (k.x < 0 ? 1u << 30 : 0u) | (k.y < 0 ? 1u << 31 : 0u);
    q[i].a = make_float4(org[0], org[1], org[2], __uint_as_float(ebits));
    q[i].b = w;
}

// Leaf-order payloads.
__global__ void k_gather_tris(const float4* tri, const unsigned* vals, unsigned n, float4* out)
{
    const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const unsigned i = vals[s];
    float4 a = tri[3 * i];
    a.w = __int_as_float((int)i);
    out[3 * s] = a;
    out[3 * s + 1] = tri[3 * i + 1];
    out[3 * s + 2] = tri[3 * i + 2];
}

__global__ void k_gather_points(const unsigned* slots, const LightVertexRec* vertices, const unsigned* vals, unsigned n,
                                float4* out)
{
    const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const unsigned slot = slots[vals[s]];
    const float4 q = vertices[slot].q[0];
    out[s] = make_float4(q.x, q.y, q.z, __uint_as_float(slot));
}

__global__ void k_gather_beams(const BeamRec* beams, const unsigned* vals, unsigned n, unsigned bb1d_paths, float4* out)
{
    const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const unsigned b = vals[s];
    const float4 q0 = beams[b].q[0], q1 = beams[b].q[1];
    const unsigned path_idx = __float_as_uint(beams[b].q[3].z);
    const unsigned bits = b | (path_idx < bb1d_paths ? 0x80000000u : 0u);
    out[2 * s] = q0;
    out[2 * s + 1] = make_float4(q1.x, q1.y, q1.z, __uint_as_float(bits));
}

// Chunk counts per beam: long beams are split so every BVH leaf box stays
// close to the beam's own extent (an axis-aligned box of a long diagonal beam
// would overlap most queries).
__global__ void k_chunk_counts(const BeamRec* beams, unsigned n, float chunk_len, unsigned max_chunks, unsigned* counts)
{
    const unsigned b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const float len = beams[b].q[0].w;
    unsigned c = chunk_len > 0.f ? (unsigned)ceilf(fminf(len / chunk_len, (float)max_chunks)) : 1u;
    counts[b] = max(1u, min(c, max_chunks));
}

__global__ void k_chunk_expand(const unsigned* counts, const unsigned* offsets, unsigned n, uint2* chunks)
{
    const unsigned b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const unsigned c = counts[b], off = offsets[b];
    for (unsigned k = 0; k < c; k++) chunks[off + k] = make_uint2(b, k | (c << 16));
}

// Leaf payload of the chunked beam map: (origin, length), (direction, bits),
// (t0, t1, medium id bits, chunk k | chunk count << 16) where bits = beam
// index | BB1D-eligible << 31.
__global__ void k_gather_chunks(const uint2* chunks, const BeamRec* beams, const unsigned* vals, unsigned n,
                                unsigned bb1d_paths, float4* out)
{
    const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint2 ch = chunks[vals[s]];
    const unsigned b = ch.x;
    const float4 q0 = beams[b].q[0], q1 = beams[b].q[1];
    const unsigned path_idx = __float_as_uint(beams[b].q[3].z);
    const unsigned bits = b | (path_idx < bb1d_paths ? 0x80000000u : 0u);
    const unsigned k = ch.y & 0xffffu, c = ch.y >> 16;
    out[3 * s] = q0;
    out[3 * s + 1] = make_float4(q1.x, q1.y, q1.z, __uint_as_float(bits));
    out[3 * s + 2] = make_float4(chunk_t(q0.w, k, c), chunk_t(q0.w, k + 1, c), q1.w, __uint_as_float(ch.y));
}

// Scratch owned by a context, sized for the largest build it will run.
struct BuildScratch {
    unsigned capacity = 0;
    unsigned *keys = nullptr, *keys_alt = nullptr, *vals = nullptr, *vals_alt = nullptr;
    int *parent_internal = nullptr, *parent_leaf = nullptr;
    unsigned* flags = nullptr;
    unsigned* ord6 = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
};

// Builds an LBVH over n boxes from `src` into `nodes` (n-1 entries, one
// primitive per leaf; the children of node i are gamma and gamma + 1, as the
// compressed nodes require); on return `sorted_vals` points at the leaf order
// (primitive index per leaf).
inline cudaError_t build_lbvh(const BoxSource& src, unsigned n, BvhNode* nodes, BuildScratch& sc, cudaStream_t st,
                              const unsigned** sorted_vals)
{
    if (n == 0) return cudaSuccess;
    if (n > kMaxBvhPrimitives) return cudaErrorInvalidValue;  // leaf-link encoding limit
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    cudaError_t e = cudaMemcpyAsync(sc.ord6, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const unsigned bs = 256;
    unsigned grid = (n + bs - 1) / bs;
    k_bounds<<<grid < 1184 ? grid : 1184, bs, 0, st>>>(src, n, sc.ord6);
    k_morton<<<grid, bs, 0, st>>>(src, n, sc.ord6, sc.keys, sc.vals);
    cub::DoubleBuffer<unsigned> kb(sc.keys, sc.keys_alt), vb(sc.vals, sc.vals_alt);
    size_t tb = sc.temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(sc.temp, tb, kb, vb, (int)n, 0, 30, st);
    if (e != cudaSuccess) return e;
    *sorted_vals = vb.Current();
    if (n > 1) {
        k_hierarchy<<<(n - 1 + bs - 1) / bs, bs, 0, st>>>(kb.Current(), (int)n, nodes, sc.parent_internal,
                                                          sc.parent_leaf);
        e = cudaMemsetAsync(sc.flags, 0, sizeof(unsigned) * (n - 1), st);
        if (e != cudaSuccess) return e;
        k_refit<<<grid, bs, 0, st>>>(src, (int)n, vb.Current(), nodes, sc.parent_internal, sc.parent_leaf, sc.flags);
    }
    return cudaGetLastError();
}

}  // namespace upbp
