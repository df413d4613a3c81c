// Scalar CPU BVH used by the oracle's OptiX emulation (oracle/ref_driver.cpp).
// Binned-SAH build over axis-aligned boxes; traversal reports every primitive
// whose (slightly enlarged) box overlaps a ray segment, which is a superset of
// what OptiX reports.  The reference's programs then apply their own exact
// predicates, so the neighbour sets do not depend on this structure.
// Test infrastructure only.
#ifndef UPBP_ORACLE_REF_BVH_H
#define UPBP_ORACLE_REF_BVH_H

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <vector>

struct OracleBox {
    float lo[3], hi[3];
};

class OracleBvh {
  public:
    void build(const std::vector<OracleBox>& boxes)
    {
        nodes_.clear();
        order_.resize(boxes.size());
        for (size_t i = 0; i < boxes.size(); i++) order_[i] = (uint32_t)i;
        boxes_ = boxes;
        if (boxes.empty()) return;
        centroids_.resize(boxes.size() * 3);
        for (size_t i = 0; i < boxes.size(); i++)
            for (int a = 0; a < 3; a++) centroids_[3 * i + a] = 0.5f * (boxes[i].lo[a] + boxes[i].hi[a]);
        nodes_.reserve(2 * boxes.size());
        nodes_.push_back(Node{});
        struct Task {
            uint32_t node, begin, end;
        };
        std::vector<Task> stack;
        stack.push_back({0, 0, (uint32_t)boxes.size()});
        while (!stack.empty()) {
            Task t = stack.back();
            stack.pop_back();
            Node& n = nodes_[t.node];
            bounds(t.begin, t.end, n.lo, n.hi);
            uint32_t count = t.end - t.begin;
            uint32_t mid = count <= 4 ? t.begin : split(t.begin, t.end);
            if (mid == t.begin || mid == t.end) {
                n.first = t.begin;
                n.count = count;
                continue;
            }
            uint32_t l = (uint32_t)nodes_.size();
            nodes_.push_back(Node{});
            nodes_.push_back(Node{});
            nodes_[t.node].first = l;
            nodes_[t.node].count = 0;
            stack.push_back({l, t.begin, mid});
            stack.push_back({l + 1, mid, t.end});
        }
    }

    bool empty() const { return nodes_.empty(); }

    // Calls f(prim, tmax&) for every primitive whose box overlaps the segment
    // o + t d, t in [tmin, tmax]; f may shrink tmax (closest-hit search) and
    // returns false to stop the traversal.
    template <class F>
    void traverse(const float o[3], const float d[3], float tmin, float& tmax, F&& f) const
    {
        if (nodes_.empty()) return;
        float inv[3];
        for (int a = 0; a < 3; a++) inv[a] = 1.f / d[a];
        uint32_t stack[256];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0 && sp < 254) {
            const Node& n = nodes_[stack[--sp]];
            if (!overlap(n.lo, n.hi, o, inv, tmin, tmax)) continue;
            if (n.count > 0) {
                for (uint32_t i = n.first; i < n.first + n.count; i++) {
                    uint32_t p = order_[i];
                    if (!overlap(boxes_[p].lo, boxes_[p].hi, o, inv, tmin, tmax)) continue;
                    if (!f(p, tmax)) return;
                }
            } else {
                stack[sp++] = n.first;
                stack[sp++] = n.first + 1;
            }
        }
    }

  private:
    struct Node {
        float lo[3], hi[3];
        uint32_t first = 0, count = 0;
    };

    static bool overlap(const float lo[3], const float hi[3], const float o[3], const float inv[3], float tmin,
                        float tmax)
    {
        double t0 = tmin, t1 = tmax;
        for (int a = 0; a < 3; a++) {
            // enlarge by a relative margin so rounding never drops a candidate
            double pad = 1e-5 * (std::fabs((double)lo[a]) + std::fabs((double)hi[a])) + 1e-6;
            double lo_a = (double)lo[a] - pad, hi_a = (double)hi[a] + pad;
            if (std::isinf(inv[a])) {
                if (o[a] < lo_a || o[a] > hi_a) return false;
                continue;
            }
            double ta = (lo_a - o[a]) * inv[a];
            double tb = (hi_a - o[a]) * inv[a];
            if (ta > tb) std::swap(ta, tb);
            t0 = ta > t0 ? ta : t0;
            t1 = tb < t1 ? tb : t1;
            if (t0 > t1) return false;
        }
        return true;
    }

    void bounds(uint32_t b, uint32_t e, float lo[3], float hi[3]) const
    {
        for (int a = 0; a < 3; a++) {
            lo[a] = FLT_MAX;
            hi[a] = -FLT_MAX;
        }
        for (uint32_t i = b; i < e; i++) {
            const OracleBox& bx = boxes_[order_[i]];
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], bx.lo[a]);
                hi[a] = std::max(hi[a], bx.hi[a]);
            }
        }
    }

    // Binned SAH split over centroids; returns the partition point.
    uint32_t split(uint32_t b, uint32_t e)
    {
        const int kBins = 16;
        float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t i = b; i < e; i++)
            for (int a = 0; a < 3; a++) {
                float c = centroids_[3 * order_[i] + a];
                clo[a] = std::min(clo[a], c);
                chi[a] = std::max(chi[a], c);
            }
        double best_cost = DBL_MAX;
        int best_axis = -1, best_bin = 0;
        for (int a = 0; a < 3; a++) {
            float ext = chi[a] - clo[a];
            if (!(ext > 0.f)) continue;
            int cnt[kBins] = {0};
            float blo[kBins][3], bhi[kBins][3];
            for (int k = 0; k < kBins; k++)
                for (int c = 0; c < 3; c++) {
                    blo[k][c] = FLT_MAX;
                    bhi[k][c] = -FLT_MAX;
                }
            for (uint32_t i = b; i < e; i++) {
                uint32_t p = order_[i];
                int k = std::min(kBins - 1, (int)((centroids_[3 * p + a] - clo[a]) / ext * kBins));
                cnt[k]++;
                for (int c = 0; c < 3; c++) {
                    blo[k][c] = std::min(blo[k][c], boxes_[p].lo[c]);
                    bhi[k][c] = std::max(bhi[k][c], boxes_[p].hi[c]);
                }
            }
            double right_area[kBins];
            int right_cnt[kBins];
            float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int rc = 0;
            for (int k = kBins - 1; k > 0; k--) {
                rc += cnt[k];
                for (int c = 0; c < 3; c++) {
                    rlo[c] = std::min(rlo[c], blo[k][c]);
                    rhi[c] = std::max(rhi[c], bhi[k][c]);
                }
                right_area[k] = rc ? area(rlo, rhi) : 0.0;
                right_cnt[k] = rc;
            }
            float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int lc = 0;
            for (int k = 0; k < kBins - 1; k++) {
                lc += cnt[k];
                for (int c = 0; c < 3; c++) {
                    llo[c] = std::min(llo[c], blo[k][c]);
                    lhi[c] = std::max(lhi[c], bhi[k][c]);
                }
                if (lc == 0 || right_cnt[k + 1] == 0) continue;
                double cost = lc * area(llo, lhi) + right_cnt[k + 1] * right_area[k + 1];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_bin = k;
                }
            }
        }
        if (best_axis < 0) return (b + e) / 2;  // all centroids equal: split by count
        float ext = chi[best_axis] - clo[best_axis];
        auto mid_it = std::partition(order_.begin() + b, order_.begin() + e, [&](uint32_t p) {
            int k = std::min(kBins - 1, (int)((centroids_[3 * p + best_axis] - clo[best_axis]) / ext * kBins));
            return k <= best_bin;
        });
        return (uint32_t)(mid_it - order_.begin());
    }

    static double area(const float lo[3], const float hi[3])
    {
        double x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
        return x * y + y * z + z * x;
    }

    std::vector<Node> nodes_;
    std::vector<uint32_t> order_;
    std::vector<OracleBox> boxes_;
    std::vector<float> centroids_;
};

#endif
