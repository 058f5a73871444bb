// Binned-SAH BVH builder (see bvh_build.hpp for the node format).
#include "bvh_build.hpp"

#include <thread>

#include "parallel.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>

namespace cupbr_b200 {

namespace {

constexpr int NBINS = 16;
constexpr int MAX_SAH_DEPTH = 44;  // beyond this depth splits fall back to the object median

struct BNode {
    float lo[3], hi[3];
    int32_t left = -1, right = -1;
    uint32_t start = 0, count = 0;
    bool leaf = false;
};

inline float half_area(const float lo[3], const float hi[3]) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

struct Aabb {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const float l[3], const float h[3]) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], l[k]); hi[k] = std::max(hi[k], h[k]); }
    }
    void grow_pt(const float p[3]) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
};

class TypeBuilder {
  public:
    TypeBuilder(const std::vector<PrimBox>& boxes, const BvhBuildParams& p) : boxes_(boxes), p_(p) {
        size_t n = boxes.size();
        idx_.resize(n);
        cent_.resize(n * 3);
        for (size_t i = 0; i < n; ++i) {
            idx_[i] = (uint32_t)i;
            for (int k = 0; k < 3; ++k) cent_[3 * i + k] = 0.5f * (boxes[i].lo[k] + boxes[i].hi[k]);
        }
        nodes_.resize(std::max<size_t>(1, 2 * n));
        count_ = 1;
    }

    void run() {
        if (boxes_.empty()) return;
        build(0, 0, (uint32_t)boxes_.size(), 0);
        nodes_.resize(count_.load());
    }

    std::vector<BNode> nodes_;
    std::vector<uint32_t> idx_;
    double sah_ = 0.0;

  private:
    const std::vector<PrimBox>& boxes_;
    BvhBuildParams p_;
    std::vector<float> cent_;
    std::atomic<uint32_t> count_{0};
    std::atomic<int> active_{1};

    // A leaf holds its primitives in ascending id order, so the built tree
    // and the slot order depend only on which primitives each node holds
    // (the device builder, bvh_gpu.cu, produces the same arrays).
    void make_leaf(BNode& nd, uint32_t b, uint32_t e) {
        nd.leaf = true;
        nd.start = b;
        nd.count = e - b;
        std::sort(idx_.begin() + b, idx_.begin() + e);
    }

    void build(uint32_t ni, uint32_t b, uint32_t e, int depth) {
        BNode& nd = nodes_[ni];
        Aabb box, cb;
        for (uint32_t i = b; i < e; ++i) {
            box.grow(boxes_[idx_[i]].lo, boxes_[idx_[i]].hi);
            cb.grow_pt(&cent_[3 * (size_t)idx_[i]]);
        }
        std::memcpy(nd.lo, box.lo, 12);
        std::memcpy(nd.hi, box.hi, 12);
        uint32_t n = e - b;
        int max_leaf = std::min(p_.max_leaf, BVH_MAX_LEAF);
        if (n <= 1) { make_leaf(nd, b, e); return; }

        // binned SAH over the three centroid axes
        float best_cost = INFINITY;
        int best_axis = -1, best_split = -1;
        if (depth < MAX_SAH_DEPTH) {
            for (int ax = 0; ax < 3; ++ax) {
                float ext = cb.hi[ax] - cb.lo[ax];
                if (!(ext > 0.0f)) continue;
                float scale = NBINS / ext;
                Aabb bins[NBINS];
                uint32_t cnt[NBINS] = {0};
                for (uint32_t i = b; i < e; ++i) {
                    uint32_t pi = idx_[i];
                    int bi = std::min(NBINS - 1, (int)((cent_[3 * (size_t)pi + ax] - cb.lo[ax]) * scale));
                    bins[bi].grow(boxes_[pi].lo, boxes_[pi].hi);
                    cnt[bi]++;
                }
                float right_area[NBINS];
                uint32_t right_cnt[NBINS];
                Aabb acc;
                uint32_t c = 0;
                for (int s = NBINS - 1; s > 0; --s) {
                    acc.grow(bins[s].lo, bins[s].hi);
                    c += cnt[s];
                    right_area[s] = half_area(acc.lo, acc.hi);
                    right_cnt[s] = c;
                }
                Aabb lacc;
                uint32_t lc = 0;
                for (int s = 1; s < NBINS; ++s) {
                    lacc.grow(bins[s - 1].lo, bins[s - 1].hi);
                    lc += cnt[s - 1];
                    if (lc == 0 || right_cnt[s] == 0) continue;
                    float cost = half_area(lacc.lo, lacc.hi) * lc + right_area[s] * right_cnt[s];
                    if (cost < best_cost) { best_cost = cost; best_axis = ax; best_split = s; }
                }
            }
        }
        float parent_area = half_area(box.lo, box.hi);
        float leaf_cost = (float)n;
        float split_cost = best_axis >= 0 ? p_.trav_cost + (parent_area > 0 ? best_cost / parent_area : (float)n) : INFINITY;
        if (n <= (uint32_t)max_leaf && !(split_cost < leaf_cost)) { make_leaf(nd, b, e); return; }

        uint32_t mid;
        if (best_axis >= 0) {
            float ext = cb.hi[best_axis] - cb.lo[best_axis];
            float scale = NBINS / ext;
            uint32_t* first = idx_.data() + b;
            uint32_t* last = idx_.data() + e;
            uint32_t* m = std::partition(first, last, [&](uint32_t pi) {
                int bi = std::min(NBINS - 1, (int)((cent_[3 * (size_t)pi + best_axis] - cb.lo[best_axis]) * scale));
                return bi < best_split;
            });
            mid = (uint32_t)(m - idx_.data());
        } else {
            mid = b;
        }
        if (mid == b || mid == e) {
            // no usable split: object median along the widest centroid axis
            int ax = 0;
            float w0 = cb.hi[0] - cb.lo[0], w1 = cb.hi[1] - cb.lo[1], w2 = cb.hi[2] - cb.lo[2];
            if (w1 > w0 && w1 >= w2) ax = 1;
            else if (w2 > w0 && w2 > w1) ax = 2;
            mid = b + n / 2;
            // (centroid, id) is a strict order: the n / 2 primitives that go
            // left do not depend on the order of the range
            std::nth_element(idx_.begin() + b, idx_.begin() + mid, idx_.begin() + e, [&](uint32_t x, uint32_t y) {
                const float cx = cent_[3 * (size_t)x + ax], cy = cent_[3 * (size_t)y + ax];
                return cx < cy || (cx == cy && x < y);
            });
        }
        uint32_t l = count_.fetch_add(2);
        nd.left = (int32_t)l;
        nd.right = (int32_t)(l + 1);
        if (n > 65536 && active_.fetch_add(1) < (int)hw_threads()) {
            std::thread left([this, l, b, mid, depth]() { build(l, b, mid, depth + 1); });
            build(l + 1, mid, e, depth + 1);
            left.join();
            active_.fetch_sub(1);
        } else {
            if (n > 65536) active_.fetch_sub(1);
            build(l, b, mid, depth + 1);
            build(l + 1, mid, e, depth + 1);
        }
    }
};

struct GNode {
    float lo[3], hi[3];
    int32_t left = -1, right = -1;
    bool leaf = false;
    uint32_t start = 0, count = 0;
};

inline int32_t leaf_ref(uint32_t start, uint32_t count) { return ~(int32_t)((start << 3) | (count - 1)); }

}  // namespace

void build_bvh(const std::vector<PrimBox>* boxes, int ntypes, const uint32_t* slot_offset, const BvhBuildParams& p,
               std::vector<uint32_t>* perm, FlatBvh& out) {
    std::vector<GNode> g;
    std::vector<int32_t> roots;
    out.stats = BvhStats();
    for (int t = 0; t < ntypes; ++t) {
        perm[t].clear();
        if (boxes[t].empty()) continue;
        TypeBuilder tb(boxes[t], p);
        tb.run();
        perm[t] = tb.idx_;
        int32_t base = (int32_t)g.size();
        for (const BNode& b : tb.nodes_) {
            GNode n;
            std::memcpy(n.lo, b.lo, 12);
            std::memcpy(n.hi, b.hi, 12);
            n.leaf = b.leaf;
            n.start = b.start + slot_offset[t];
            n.count = b.count;
            n.left = b.left >= 0 ? b.left + base : -1;
            n.right = b.right >= 0 ? b.right + base : -1;
            g.push_back(n);
        }
        roots.push_back(base);
    }
    out.nodes.clear();
    if (roots.empty()) {
        // empty scene: one node with four empty children
        out.nodes.assign(4 * BVH_NODE_F4, 0.0f);
        for (int k = 0; k < 4; ++k) {
            for (int a = 0; a < 3; ++a) {
                out.nodes[8 * a + k] = INFINITY;
                out.nodes[8 * a + 4 + k] = -INFINITY;
            }
            std::memcpy(&out.nodes[24 + k], &BVH_EMPTY, 4);
        }
        return;
    }
    // join the type roots pairwise under new inner nodes
    while (roots.size() > 1) {
        GNode n;
        const GNode& a = g[roots[roots.size() - 2]];
        const GNode& b = g[roots[roots.size() - 1]];
        for (int k = 0; k < 3; ++k) { n.lo[k] = std::min(a.lo[k], b.lo[k]); n.hi[k] = std::max(a.hi[k], b.hi[k]); }
        n.left = roots[roots.size() - 2];
        n.right = roots[roots.size() - 1];
        g.push_back(n);
        roots.pop_back();
        roots.back() = (int32_t)g.size() - 1;
    }
    int32_t root = roots[0];

    // Collapse the binary tree into 4-wide nodes: a node takes its two
    // children and keeps replacing the inner child of largest surface area
    // by that child's two children until it has four.
    if (g[root].leaf) {
        // single leaf: wrap it in an inner node
        GNode n;
        std::memcpy(n.lo, g[root].lo, 12);
        std::memcpy(n.hi, g[root].hi, 12);
        n.left = root;
        n.right = -1;
        g.push_back(n);
        root = (int32_t)g.size() - 1;
    }
    auto children4 = [&](int32_t v, int32_t* out) {
        int n = 0;
        for (int32_t c : {g[v].left, g[v].right})
            if (c >= 0) out[n++] = c;
        while (n < 4) {
            int best = -1;
            float best_area = -1.0f;
            for (int k = 0; k < n; ++k) {
                const GNode& c = g[out[k]];
                if (c.leaf) continue;
                const float a = half_area(c.lo, c.hi);
                if (a > best_area) { best_area = a; best = k; }
            }
            if (best < 0) break;
            const int32_t e = out[best];
            int32_t kids[2];
            int nk = 0;
            for (int32_t c : {g[e].left, g[e].right})
                if (c >= 0) kids[nk++] = c;
            if (nk == 0) break;
            out[best] = kids[0];
            if (nk == 2) out[n++] = kids[1];
        }
        return n;
    };
    // 4-wide nodes: breadth-first for the top levels (shared-memory staging),
    // depth-first below
    struct W4 { int32_t src; int32_t child[4]; int n; uint32_t depth; };
    std::vector<W4> order;
    std::vector<int32_t> gpu_index(g.size(), -1);
    {
        auto make = [&](int32_t v, uint32_t depth) {
            W4 w{v, {-1, -1, -1, -1}, 0, depth};
            w.n = children4(v, w.child);
            return w;
        };
        std::vector<W4> frontier;
        std::vector<W4> q{make(root, 0)};
        size_t qi = 0;
        while (qi < q.size()) {
            W4 w = q[qi++];
            if ((int)w.depth < p.top_bfs_levels) {
                gpu_index[w.src] = (int32_t)order.size();
                order.push_back(w);
                for (int k = 0; k < w.n; ++k)
                    if (!g[w.child[k]].leaf) q.push_back(make(w.child[k], w.depth + 1));
            } else {
                frontier.push_back(w);
            }
        }
        std::vector<W4> st;
        for (const W4& f : frontier) {
            st.push_back(f);
            while (!st.empty()) {
                W4 w = st.back();
                st.pop_back();
                gpu_index[w.src] = (int32_t)order.size();
                order.push_back(w);
                for (int k = w.n - 1; k >= 0; --k)
                    if (!g[w.child[k]].leaf) st.push_back(make(w.child[k], w.depth + 1));
            }
        }
    }
    constexpr size_t FLOATS = 4 * BVH_NODE_F4;
    out.nodes.assign(order.size() * FLOATS, 0.0f);
    uint32_t maxd = 0, leaves = 0;
    double sah = 0.0;
    const float root_area = half_area(g[root].lo, g[root].hi);
    for (size_t i = 0; i < order.size(); ++i) {
        const W4& w = order[i];
        float* o = &out.nodes[i * FLOATS];
        for (int k = 0; k < 4; ++k) {
            int32_t ref = BVH_EMPTY;
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            if (k < w.n) {
                const GNode& c = g[w.child[k]];
                std::memcpy(lo, c.lo, 12);
                std::memcpy(hi, c.hi, 12);
                if (c.leaf) {
                    ref = leaf_ref(c.start, c.count);
                    ++leaves;
                    if (root_area > 0) sah += half_area(c.lo, c.hi) / root_area * c.count;
                } else {
                    ref = gpu_index[w.child[k]];
                }
            }
            o[0 + k] = lo[0];
            o[4 + k] = hi[0];
            o[8 + k] = lo[1];
            o[12 + k] = hi[1];
            o[16 + k] = lo[2];
            o[20 + k] = hi[2];
            std::memcpy(&o[24 + k], &ref, 4);
        }
        if (root_area > 0) sah += p.trav_cost * half_area(g[w.src].lo, g[w.src].hi) / root_area;
        maxd = std::max<uint32_t>(maxd, w.depth + 1);
    }
    out.stats.inner_nodes = (uint32_t)order.size();
    out.stats.leaves = leaves;
    out.stats.max_depth = maxd;
    out.stats.sah_cost = sah;
}

}  // namespace cupbr_b200
