// Sequential statement of the device's binned-SAH scene BVH build
// (gpuupbp_b200/csrc/upbp_scene_bvh.cuh).  Test infrastructure: the checker
// that the device build produces exactly this tree -- node slots, boxes,
// links, leaf order -- for the same triangles.  Built by oracle/Makefile into
// _ref/libsah_ref.so (no reference sources needed); nothing in the product
// links it.  Compiled with -ffp-contract=off, so every float operation
// rounds as written, as the device build's explicitly rounded ones do.
//
// The build: a range of m >= 2 primitives is split by the surface-area
// heuristic over 16 centroid bins per axis (cost area(left) x left count +
// area(right) x right count in double; the first minimum over axes 0..2 and
// bins 0..14), or at its middle from depth 48 on or where the centroids
// coincide; the primitives are partitioned stably; a subtree of m
// primitives occupies m - 1 consecutive node slots, its root first; one
// primitive per leaf.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int kBins = 16;
constexpr int kMaxSahDepth = 48;

struct Box {
    float lo[3], hi[3];
    void reset()
    {
        for (int k = 0; k < 3; k++) {
            lo[k] = 1e30f;
            hi[k] = -1e30f;
        }
    }
    void grow(const float* l, const float* h)
    {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], l[k]);
            hi[k] = std::max(hi[k], h[k]);
        }
    }
    void grow(const Box& b) { grow(b.lo, b.hi); }
    double area() const
    {
        double d[3];
        for (int k = 0; k < 3; k++) d[k] = std::max(0.f, hi[k] - lo[k]);
        return 2.0 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

int bin_of(float c, float lo, float scale)
{
    const float f = (c - lo) * scale;
    return f > 0.f ? std::min(kBins - 1, (int)std::min(f, (float)kBins)) : 0;
}

struct Build {
    std::vector<float> box;  // 6 floats per primitive
    std::vector<float> cen;  // 3 floats per primitive
    uint32_t* idx;
    float* nodes;
};

Box range_box(const Build& b, uint32_t a, uint32_t e)
{
    Box r;
    r.reset();
    for (uint32_t i = a; i < e; i++) r.grow(&b.box[6 * (size_t)b.idx[i]], &b.box[6 * (size_t)b.idx[i] + 3]);
    return r;
}

void write_node(Build& b, uint32_t slot, const Box& l, const Box& r, int32_t ll, int32_t rl, uint32_t nl, uint32_t nr)
{
    float* w = b.nodes + 16 * (size_t)slot;
    const float v[12] = {l.lo[0], l.lo[1], l.lo[2], l.hi[0], l.hi[1], l.hi[2],
                         r.lo[0], r.lo[1], r.lo[2], r.hi[0], r.hi[1], r.hi[2]};
    std::memcpy(w, v, sizeof(v));
    const int32_t k[4] = {ll, rl, (int32_t)nl, (int32_t)nr};
    std::memcpy(w + 12, k, sizeof(k));
}

void build(Build& b, uint32_t a, uint32_t e, uint32_t slot, int depth)
{
    const uint32_t m = e - a;
    Box cb;
    cb.reset();
    for (uint32_t i = a; i < e; i++) {
        const float* c = &b.cen[3 * (size_t)b.idx[i]];
        cb.grow(c, c);
    }
    int best_axis = -1, best_bin = -1;
    if (depth < kMaxSahDepth) {
        double best = 1e300;
        for (int ax = 0; ax < 3; ax++) {
            const float ext = cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.f)) continue;
            const float scale = kBins / ext;
            Box bins[kBins];
            uint32_t counts[kBins] = {};
            for (auto& x : bins) x.reset();
            for (uint32_t i = a; i < e; i++) {
                const uint32_t p = b.idx[i];
                const int k = bin_of(b.cen[3 * (size_t)p + ax], cb.lo[ax], scale);
                bins[k].grow(&b.box[6 * (size_t)p], &b.box[6 * (size_t)p + 3]);
                counts[k]++;
            }
            double right_area[kBins];
            uint32_t right_count[kBins];
            Box acc;
            acc.reset();
            uint32_t c = 0;
            for (int k = kBins - 1; k > 0; k--) {
                acc.grow(bins[k]);
                c += counts[k];
                right_area[k] = acc.area();
                right_count[k] = c;
            }
            acc.reset();
            c = 0;
            for (int k = 0; k < kBins - 1; k++) {
                acc.grow(bins[k]);
                c += counts[k];
                if (c == 0 || right_count[k + 1] == 0) continue;
                const double cost = acc.area() * c + right_area[k + 1] * right_count[k + 1];
                if (cost < best) {
                    best = cost;
                    best_axis = ax;
                    best_bin = k;
                }
            }
        }
    }
    uint32_t mid = a + m / 2;
    if (best_axis >= 0) {
        const float lo = cb.lo[best_axis], scale = kBins / (cb.hi[best_axis] - cb.lo[best_axis]);
        const float* cen = b.cen.data();
        const uint32_t* it = std::stable_partition(b.idx + a, b.idx + e, [&](uint32_t p) {
            return bin_of(cen[3 * (size_t)p + best_axis], lo, scale) <= best_bin;
        });
        mid = (uint32_t)(it - b.idx);
    }
    const uint32_t ml = mid - a, mr = e - mid;
    const Box lb = range_box(b, a, mid), rb = range_box(b, mid, e);
    const int32_t ll = ml == 1 ? ~(int32_t)a : (int32_t)(slot + 1);
    const int32_t rl = mr == 1 ? ~(int32_t)mid : (int32_t)(slot + ml);
    write_node(b, slot, lb, rb, ll, rl, ml, mr);
    if (ml >= 2) build(b, a, mid, slot + 1, depth + 1);
    if (mr >= 2) build(b, mid, e, slot + ml, depth + 1);
}

}  // namespace

// Triangles as 12 floats each (v0.xyzw, e1.xyzw, e2.xyzw; w ignored), the
// device's triangle records.  nodes: 16 words per node, n - 1 nodes;
// order[k]: the triangle at leaf position k; boxes (optional, 6 floats per
// triangle): the widened boxes the build used.
extern "C" int upbp_sah_ref_build(const float* tri, uint32_t n, float* nodes, uint32_t* order, float* boxes)
{
    if (n == 0) return 0;
    Build b;
    b.box.resize(6 * (size_t)n);
    b.cen.resize(3 * (size_t)n);
    for (uint32_t i = 0; i < n; i++) {
        const float* t = tri + 12 * (size_t)i;
        const float px[3] = {t[0], t[0] + t[4], t[0] + t[8]}, py[3] = {t[1], t[1] + t[5], t[1] + t[9]},
                    pz[3] = {t[2], t[2] + t[6], t[2] + t[10]};
        const float lo[3] = {std::min(std::min(px[0], px[1]), px[2]), std::min(std::min(py[0], py[1]), py[2]),
                             std::min(std::min(pz[0], pz[1]), pz[2])};
        const float hi[3] = {std::max(std::max(px[0], px[1]), px[2]), std::max(std::max(py[0], py[1]), py[2]),
                             std::max(std::max(pz[0], pz[1]), pz[2])};
        const float mag = 1e-7f * (std::fabs(lo[0]) + std::fabs(lo[1]) + std::fabs(lo[2]) + 1e-3f);
        for (int k = 0; k < 3; k++) {
            const float ext = (hi[k] - lo[k]) * 1e-6f + mag;
            b.box[6 * (size_t)i + k] = lo[k] - ext;
            b.box[6 * (size_t)i + 3 + k] = hi[k] + ext;
            b.cen[3 * (size_t)i + k] = 0.5f * (b.box[6 * (size_t)i + k] + b.box[6 * (size_t)i + 3 + k]);
        }
    }
    if (boxes) std::memcpy(boxes, b.box.data(), b.box.size() * sizeof(float));
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    b.idx = order;
    b.nodes = nodes;
    if (n >= 2) build(b, 0, n, 0, 0);
    return 0;
}
