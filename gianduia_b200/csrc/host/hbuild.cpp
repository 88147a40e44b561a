// Host BVH build: the reference's binary SAH builder (bvhBuilder.cpp:59-182) and its
// greedy 4-wide collapse (bvhBuilder.cpp:184-262), emitting the 128-byte device nodes.
//
// The builder works on an index permutation partitioned in place, so every subtree owns
// a contiguous range and the leaf order is the depth-first order of the serial reference
// build; subtrees above 4096 primitives are built on separate threads (the reference uses
// tbb::parallel_invoke at the same threshold) without changing the result.
#include <algorithm>
#include <cstring>
#include <future>
#include <limits>

#include "hscene.h"

namespace gndh {

void Bounds::grow(V3 p) {
    lo = gnd::v3(std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z));
    hi = gnd::v3(std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z));
}
void Bounds::grow(const Bounds& b) {
    lo = gnd::v3(std::min(lo.x, b.lo.x), std::min(lo.y, b.lo.y), std::min(lo.z, b.lo.z));
    hi = gnd::v3(std::max(hi.x, b.hi.x), std::max(hi.y, b.hi.y), std::max(hi.z, b.hi.z));
}
float Bounds::area() const {
    V3 d = hi - lo;
    return 2.f * (d.x * d.y + d.x * d.z + d.y * d.z);
}
int Bounds::maxExtent() const {
    V3 d = hi - lo;
    if (d.x > d.y && d.x > d.z) return 0;
    if (d.y > d.z) return 1;
    return 2;
}
Bounds Bounds::transformed(const Transform& t) const {
    Bounds r;
    for (int i = 0; i < 8; ++i) {
        V3 c = gnd::v3((i & 1) ? hi.x : lo.x, (i & 2) ? hi.y : lo.y, (i & 4) ? hi.z : lo.z);
        V3 p = t.point(c);
        if (i == 0) { r.lo = p; r.hi = p; } else r.grow(p);
    }
    return r;
}

namespace {

struct Builder {
    const std::vector<Bounds>& pb;
    const std::vector<V3>& pc;
    std::vector<uint32_t>& idx;
    int parallelDepth;

    // Builds [start, end) and returns its nodes in depth-first order with offsets relative
    // to the returned vector's first element.
    std::vector<BinNode> build(int start, int end, int depth) {
        std::vector<BinNode> out;
        Bounds bounds;
        for (int i = start; i < end; ++i) bounds.grow(pb[idx[i]]);
        int n = end - start;
        auto leaf = [&]() {
            out.push_back(BinNode{bounds, (uint32_t)start, (uint32_t)n});
            return out;
        };
        if (n == 1 || depth == 63) return leaf();
        Bounds cb;
        for (int i = start; i < end; ++i) cb.grow(pc[idx[i]]);
        int dim = cb.maxExtent();
        float cmin = gnd::comp(cb.lo, dim), cmax = gnd::comp(cb.hi, dim);
        if (cmax == cmin) return leaf();
        constexpr int nB = 12;
        int count[nB] = {0};
        Bounds bb[nB];
        float denom = cmax - cmin;
        if (denom == 0) denom = 1.0f;
        auto bucketOf = [&](uint32_t p) {
            int b = (int)(nB * (gnd::comp(pc[p], dim) - cmin) / denom);
            return b == nB ? nB - 1 : b;
        };
        for (int i = start; i < end; ++i) {
            int b = bucketOf(idx[i]);
            count[b]++;
            bb[b].grow(pb[idx[i]]);
        }
        float cost[nB - 1];
        float sa = bounds.area();
        for (int i = 0; i < nB - 1; ++i) {
            Bounds b0, b1;
            int c0 = 0, c1 = 0;
            for (int j = 0; j <= i; ++j) { b0.grow(bb[j]); c0 += count[j]; }
            for (int j = i + 1; j < nB; ++j) { b1.grow(bb[j]); c1 += count[j]; }
            cost[i] = 1 + (c0 * b0.area() + c1 * b1.area()) / sa;
        }
        float minCost = cost[0];
        int split = 0;
        for (int i = 1; i < nB - 1; ++i)
            if (cost[i] < minCost) { minCost = cost[i]; split = i; }
        if (!(n > 4 || minCost < (float)n)) return leaf();
        uint32_t* mid = std::partition(idx.data() + start, idx.data() + end, [&](uint32_t p) { return bucketOf(p) <= split; });
        int m = (int)(mid - idx.data());
        std::vector<BinNode> L, R;
        if (n > 4096 && depth < parallelDepth) {
            auto fut = std::async(std::launch::async, [&]() { return build(start, m, depth + 1); });
            R = build(m, end, depth + 1);
            L = fut.get();
        } else {
            L = build(start, m, depth + 1);
            R = build(m, end, depth + 1);
        }
        Bounds ub = L[0].b;
        ub.grow(R[0].b);
        out.reserve(1 + L.size() + R.size());
        out.push_back(BinNode{ub, (uint32_t)(1 + L.size()), 0});
        for (BinNode nd : L) { if (nd.count == 0) nd.offset += 1; out.push_back(nd); }
        uint32_t rb = (uint32_t)(1 + L.size());
        for (BinNode nd : R) { if (nd.count == 0) nd.offset += rb; out.push_back(nd); }
        return out;
    }
};

}  // namespace

BinTree buildSAH(const std::vector<Bounds>& pb, const std::vector<V3>& pc, int parallelDepth) {
    BinTree t;
    if (pb.empty()) return t;
    t.order.resize(pb.size());
    for (size_t i = 0; i < pb.size(); ++i) t.order[i] = (uint32_t)i;
    Builder b{pb, pc, t.order, parallelDepth};
    t.nodes = b.build(0, (int)pb.size(), 0);
    return t;
}

namespace {
struct ChildRef {
    uint32_t ref;
    Bounds b;
};

void writeNode(gnd::Node4& nd, const ChildRef* ch, int n) {
    const float inf = std::numeric_limits<float>::infinity();
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            nd.lox[i] = ch[i].b.lo.x; nd.loy[i] = ch[i].b.lo.y; nd.loz[i] = ch[i].b.lo.z;
            nd.hix[i] = ch[i].b.hi.x; nd.hiy[i] = ch[i].b.hi.y; nd.hiz[i] = ch[i].b.hi.z;
            nd.child[i] = ch[i].ref;
        } else {
            nd.lox[i] = nd.loy[i] = nd.loz[i] = inf;
            nd.hix[i] = nd.hiy[i] = nd.hiz[i] = -inf;
            nd.child[i] = gnd::kEmpty;
        }
        nd.pad[i] = 0;
    }
}

// A leaf of more than kLeafMax primitives (only produced for coincident centroids or at
// depth 63) becomes a small subtree of <=16-primitive leaves.
ChildRef emitLeaf(uint32_t first, uint32_t count, uint32_t leafBase, const BinTree& t,
                  const std::vector<Bounds>& pb, std::vector<gnd::Node4>& out) {
    Bounds b;
    for (uint32_t i = 0; i < count; ++i) b.grow(pb[t.order[first + i]]);
    if (count <= (uint32_t)gnd::kLeafMax) return ChildRef{gnd::makeLeaf(leafBase + first, count), b};
    uint32_t me = (uint32_t)out.size();
    out.emplace_back();
    ChildRef ch[4];
    uint32_t per = (count + 3) / 4;
    int n = 0;
    for (uint32_t s = 0; s < count; s += per) ch[n++] = emitLeaf(first + s, std::min(per, count - s), leafBase, t, pb, out);
    writeNode(out[me], ch, n);
    return ChildRef{me, b};
}

uint32_t collapse(const BinTree& t, int bi, uint32_t leafBase, const std::vector<Bounds>& pb, std::vector<gnd::Node4>& out) {
    uint32_t me = (uint32_t)out.size();
    out.emplace_back();
    std::vector<int> cand = {bi};
    while (cand.size() < 4) {
        int best = -1;
        float bestArea = -1.0f;
        for (size_t i = 0; i < cand.size(); ++i) {
            const BinNode& c = t.nodes[cand[i]];
            if (c.count == 0) {
                float a = c.b.area();
                if (a > bestArea) { bestArea = a; best = (int)i; }
            }
        }
        if (best == -1) break;
        int e = cand[best];
        cand.erase(cand.begin() + best);
        cand.push_back(e + 1);
        cand.push_back((int)t.nodes[e].offset);
    }
    ChildRef ch[4];
    int n = 0;
    for (int ci : cand) {
        const BinNode& c = t.nodes[ci];
        if (c.count > 0) ch[n++] = emitLeaf(c.offset, c.count, leafBase, t, pb, out);
        else { uint32_t k = collapse(t, ci, leafBase, pb, out); ch[n++] = ChildRef{k, c.b}; }
    }
    writeNode(out[me], ch, n);
    return me;
}
}  // namespace

uint32_t collapseToNode4(const BinTree& t, uint32_t leafBase, const std::vector<Bounds>& pb, std::vector<gnd::Node4>& out) {
    if (t.nodes.empty()) return gnd::kEmpty;
    return collapse(t, 0, leafBase, pb, out);
}

}  // namespace gndh
