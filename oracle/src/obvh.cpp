// Oracle (test infrastructure only): SAH BVH build, BVH4 collapse, 4-wide traversal,
// triangle packs and the analytic shapes of the reference, restated on the CPU.
#include "oscene.h"
#include <algorithm>
#include <cstring>

namespace orc {

namespace {
struct BuildNode {
    Bounds3 bounds;
    BuildNode* children[2] = {nullptr, nullptr};
    int splitAxis = 0, firstPrimOffset = 0, nPrimitives = 0;
};
struct Bucket { int count = 0; Bounds3 bounds; };

// bvhBuilder.cpp:36-51
int flatten(BuildNode* node, int* offset, std::vector<BVHNode>& out) {
    BVHNode* ln = &out[*offset];
    ln->bounds = node->bounds;
    int cur = (*offset)++;
    if (node->nPrimitives > 0) {
        ln->offset = node->firstPrimOffset;
        ln->nPrimitives = (uint16_t)node->nPrimitives;
    } else {
        ln->axis = (uint8_t)node->splitAxis;
        ln->nPrimitives = 0;
        flatten(node->children[0], offset, out);
        out[cur].offset = flatten(node->children[1], offset, out);
    }
    return cur;
}
void freeTree(BuildNode* n) {
    if (n->children[0]) freeTree(n->children[0]);
    if (n->children[1]) freeTree(n->children[1]);
    delete n;
}
}  // namespace

// bvhBuilder.cpp:59-182. Serial: leaf offsets follow depth-first order (the reference
// assigns them with an atomic counter, in task order above 4096 primitives).
BVHBuildResult buildBVH(std::vector<BVHBuildInfo>& data) {
    BVHBuildResult result;
    if (data.empty()) return result;
    int totalNodes = 0;
    std::vector<BVHBuildInfo> ordered(data.size());
    int orderedOffset = 0;
    std::function<BuildNode*(int, int, int)> rec = [&](int start, int end, int depth) -> BuildNode* {
        BuildNode* node = new BuildNode();
        ++totalNodes;
        Bounds3 bounds;
        for (int i = start; i < end; ++i) bounds = Union(bounds, data[i].bounds);
        int n = end - start;
        auto leaf = [&]() {
            int my = orderedOffset;
            orderedOffset += n;
            for (int i = 0; i < n; ++i) ordered[my + i] = data[start + i];
            node->firstPrimOffset = my;
            node->nPrimitives = n;
            node->bounds = bounds;
            return node;
        };
        if (n == 1 || depth == 63) return leaf();
        Bounds3 cb;
        for (int i = start; i < end; ++i) cb = Union(cb, data[i].centroid);
        int dim = cb.maximumExtent();
        if (cb.pMax[dim] == cb.pMin[dim]) return leaf();
        constexpr int nB = 12;
        Bucket buckets[nB];
        float denom = cb.pMax[dim] - cb.pMin[dim];
        if (denom == 0) denom = 1.0f;
        for (int i = start; i < end; ++i) {
            int b = (int)(nB * (data[i].centroid - cb.pMin)[dim] / denom);
            if (b == nB) b = nB - 1;
            buckets[b].count++;
            buckets[b].bounds = Union(buckets[b].bounds, data[i].bounds);
        }
        float cost[nB - 1];
        for (int i = 0; i < nB - 1; ++i) {
            Bounds3 b0, b1;
            int c0 = 0, c1 = 0;
            for (int j = 0; j <= i; ++j) { b0 = Union(b0, buckets[j].bounds); c0 += buckets[j].count; }
            for (int j = i + 1; j < nB; ++j) { b1 = Union(b1, buckets[j].bounds); c1 += buckets[j].count; }
            cost[i] = 1 + (c0 * b0.surfaceArea() + c1 * b1.surfaceArea()) / bounds.surfaceArea();
        }
        float minCost = cost[0];
        int split = 0;
        for (int i = 1; i < nB - 1; ++i) if (cost[i] < minCost) { minCost = cost[i]; split = i; }
        float leafCost = (float)n;
        if (n > 4 || minCost < leafCost) {
            auto pmid = std::partition(&data[start], &data[end - 1] + 1, [=](const BVHBuildInfo& pi) {
                int b = (int)(nB * (pi.centroid - cb.pMin)[dim] / denom);
                if (b == nB) b = nB - 1;
                return b <= split;
            });
            int mid = (int)(pmid - &data[0]);
            BuildNode* c0 = rec(start, mid, depth + 1);
            BuildNode* c1 = rec(mid, end, depth + 1);
            node->children[0] = c0;
            node->children[1] = c1;
            node->bounds = Union(c0->bounds, c1->bounds);
            node->splitAxis = dim;
            node->nPrimitives = 0;
        } else {
            return leaf();
        }
        return node;
    };
    BuildNode* root = rec(0, (int)data.size(), 0);
    result.nodes.resize(totalNodes);
    int off = 0;
    flatten(root, &off, result.nodes);
    result.orderedIndices.reserve(ordered.size());
    for (auto& o : ordered) result.orderedIndices.push_back(o.originalIndex);
    freeTree(root);
    return result;
}

// bvhBuilder.cpp:184-262 (greedy collapse; expand the largest-area interior candidate)
std::vector<BVHNode4> buildWide(const std::vector<BVHNode>& bin) {
    std::vector<BVHNode4> nodes4;
    if (bin.empty()) return nodes4;
    nodes4.reserve(bin.size() / 2);
    std::function<int(int)> collapse = [&](int idx) -> int {
        int me = (int)nodes4.size();
        nodes4.push_back(BVHNode4());
        std::vector<int> cand = {idx};
        while (cand.size() < 4) {
            int best = -1;
            float bestArea = -1.0f;
            for (size_t i = 0; i < cand.size(); ++i) {
                const BVHNode& c = bin[cand[i]];
                if (c.nPrimitives == 0) {
                    float a = c.bounds.surfaceArea();
                    if (a > bestArea) { bestArea = a; best = (int)i; }
                }
            }
            if (best == -1) break;
            int e = cand[best];
            cand.erase(cand.begin() + best);
            cand.push_back(e + 1);
            cand.push_back((int)bin[e].offset);
        }
        struct CD { uint8_t type; uint32_t off, cnt; Bounds3 b; };
        std::vector<CD> cd;
        for (int ci : cand) {
            const BVHNode& c = bin[ci];
            if (c.nPrimitives > 0) cd.push_back({2, c.offset, c.nPrimitives, c.bounds});
            else { int k = collapse(ci); cd.push_back({1, (uint32_t)k, 0, c.bounds}); }
        }
        BVHNode4& n4 = nodes4[me];
        for (int i = 0; i < 4; ++i) {
            if (i < (int)cd.size()) {
                n4.childType[i] = cd[i].type; n4.offset[i] = cd[i].off; n4.packCount[i] = cd[i].cnt;
                n4.minX[i] = cd[i].b.pMin.x; n4.minY[i] = cd[i].b.pMin.y; n4.minZ[i] = cd[i].b.pMin.z;
                n4.maxX[i] = cd[i].b.pMax.x; n4.maxY[i] = cd[i].b.pMax.y; n4.maxZ[i] = cd[i].b.pMax.z;
            } else {
                n4.childType[i] = 0; n4.offset[i] = 0; n4.packCount[i] = 0;
                n4.minX[i] = n4.minY[i] = n4.minZ[i] = Infinity;
                n4.maxX[i] = n4.maxY[i] = n4.maxZ[i] = -Infinity;
            }
        }
        return me;
    };
    collapse(0);
    return nodes4;
}

// Lane-wise min/max with the x86 SSE semantics Highway uses (second operand on NaN).
static inline float vmin(float a, float b) { return a < b ? a : b; }
static inline float vmax(float a, float b) { return a > b ? a : b; }

// bvhTraversal.h:19-98
bool traverseBVH4(const std::vector<BVHNode4>& nodes, const Ray& ray, bool shadow,
                  const std::function<bool(int, int)>& leaf, TraversalStats* st) {
    if (nodes.empty()) return false;
    bool hitAny = false;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    float ox = ray.o.x, oy = ray.o.y, oz = ray.o.z;
    float ix = 1.0f / ray.d.x, iy = 1.0f / ray.d.y, iz = 1.0f / ray.d.z;
    float tMinR = ray.tMin;
    float tMaxR = ray.tMax;
    while (sp > 0) {
        int ni = stack[--sp];
        const BVHNode4& n = nodes[ni];
        if (st) st->nodes++;
        // the four lanes as one straight-line loop over fixed-size arrays, so that the
        // compiler turns it into 4-wide vector code as the Highway lanes are
        float tminL[4], tmaxL[4];
        for (int i = 0; i < 4; ++i) {
            float t1x = (n.minX[i] - ox) * ix, t2x = (n.maxX[i] - ox) * ix;
            float tminx = vmin(t1x, t2x), tmaxx = vmax(t1x, t2x);
            float t1y = (n.minY[i] - oy) * iy, t2y = (n.maxY[i] - oy) * iy;
            float tminy = vmin(t1y, t2y), tmaxy = vmax(t1y, t2y);
            float t1z = (n.minZ[i] - oz) * iz, t2z = (n.maxZ[i] - oz) * iz;
            float tminz = vmin(t1z, t2z), tmaxz = vmax(t1z, t2z);
            tminL[i] = vmax(vmax(tminx, tminy), vmax(tminz, tMinR));
            tmaxL[i] = vmin(vmin(tmaxx, tmaxy), vmin(tmaxz, tMaxR));
        }
        int mask = 0;
        for (int i = 0; i < 4; ++i) mask |= (tminL[i] <= tmaxL[i] ? 1 : 0) << i;
        if (!mask) continue;
        for (int i = 0; i < 4; ++i) {
            if (!(mask & (1 << i))) continue;
            if (n.childType[i] == 1) {
                stack[sp++] = (int)n.offset[i];
            } else if (n.childType[i] == 2) {
                if (st) st->leaves++;
                bool h = leaf((int)n.offset[i], (int)n.packCount[i]);
                if (h) {
                    hitAny = true;
                    if (shadow) return true;
                    tMaxR = ray.tMax;
                }
            }
        }
    }
    return hitAny;
}

// ---------------------------------------------------------------- mesh

// mesh.cpp:17-146 (from "BVH construction" on)
void Mesh::buildAccel() {
    size_t triCount = indices.size() / 3;
    std::vector<BVHBuildInfo> bd;
    bd.reserve(triCount);
    for (size_t i = 0; i < triCount; ++i) {
        const Vec3& p0 = positions[indices[i * 3 + 0]];
        const Vec3& p1 = positions[indices[i * 3 + 1]];
        const Vec3& p2 = positions[indices[i * 3 + 2]];
        Bounds3 b;
        b = Union(b, p0); b = Union(b, p1); b = Union(b, p2);
        bd.push_back({b, b.centroid(), (int)i});
    }
    BVHBuildResult r = buildBVH(bd);
    std::vector<BVHNode> nodes = std::move(r.nodes);
    if (!nodes.empty()) bounds = nodes[0].bounds;
    packs.clear();
    for (auto& node : nodes) {
        if (node.nPrimitives > 0) {
            int oo = (int)node.offset, oc = node.nPrimitives;
            int po = (int)packs.size();
            int np = (oc + 3) / 4;
            for (int p = 0; p < np; ++p) {
                TrianglePack4 pk;
                for (int l = 0; l < 4; ++l) {
                    pk.v0x[l] = pk.v0y[l] = pk.v0z[l] = 0.f;
                    pk.v1x[l] = pk.v1y[l] = pk.v1z[l] = 0.f;
                    pk.v2x[l] = pk.v2y[l] = pk.v2z[l] = 0.f;
                    pk.primIndex[l] = (uint32_t)-1;
                }
                for (int l = 0; l < 4; ++l) {
                    int ti = p * 4 + l;
                    if (ti < oc) {
                        int orig = r.orderedIndices[oo + ti];
                        pk.primIndex[l] = (uint32_t)orig;
                        const Vec3& p0 = positions[indices[orig * 3 + 0]];
                        const Vec3& p1 = positions[indices[orig * 3 + 1]];
                        const Vec3& p2 = positions[indices[orig * 3 + 2]];
                        pk.v0x[l] = p0.x; pk.v0y[l] = p0.y; pk.v0z[l] = p0.z;
                        pk.v1x[l] = p1.x; pk.v1y[l] = p1.y; pk.v1z[l] = p1.z;
                        pk.v2x[l] = p2.x; pk.v2y[l] = p2.y; pk.v2z[l] = p2.z;
                    }
                }
                packs.push_back(pk);
            }
            node.offset = (uint32_t)po;
            node.nPrimitives = (uint16_t)np;
        }
    }
    if (!nodes.empty()) nodes4 = buildWide(nodes);
    // area CDF, mesh.cpp:120-145
    cdf.assign(triCount + 1, 0.0f);
    totalArea = 0.0f;
    for (size_t i = 0; i < triCount; ++i) {
        const Vec3& p0 = positions[indices[i * 3 + 0]];
        const Vec3& p1 = positions[indices[i * 3 + 1]];
        const Vec3& p2 = positions[indices[i * 3 + 2]];
        float area = 0.5f * Cross(p1 - p0, p2 - p0).length();
        totalArea += area;
        cdf[i + 1] = totalArea;
    }
    if (totalArea > 0.0f) for (size_t i = 1; i <= triCount; ++i) cdf[i] /= totalArea;
}

// mesh.cpp:259-291: Moller-Trumbore on the four lanes of a pack, in the Highway code's
// operation order. Straight-line lanes (no short-circuit branches) over restrict
// pointers, so that the compiler emits 4-wide vector code as the Highway lanes do.
static inline void packTest(const TrianglePack4& pk, float ox, float oy, float oz, float dx, float dy, float dz,
                            float tMin, float tMax, float* __restrict__ tA, float* __restrict__ uA,
                            float* __restrict__ vA, int* __restrict__ valid) {
    const float* __restrict__ v0x = pk.v0x; const float* __restrict__ v0y = pk.v0y; const float* __restrict__ v0z = pk.v0z;
    const float* __restrict__ v1x = pk.v1x; const float* __restrict__ v1y = pk.v1y; const float* __restrict__ v1z = pk.v1z;
    const float* __restrict__ v2x = pk.v2x; const float* __restrict__ v2y = pk.v2y; const float* __restrict__ v2z = pk.v2z;
    for (int l = 0; l < 4; ++l) {
        float e1x = v1x[l] - v0x[l], e1y = v1y[l] - v0y[l], e1z = v1z[l] - v0z[l];
        float e2x = v2x[l] - v0x[l], e2y = v2y[l] - v0y[l], e2z = v2z[l] - v0z[l];
        float px = dy * e2z - dz * e2y;
        float py = dz * e2x - dx * e2z;
        float pz = dx * e2y - dy * e2x;
        float det = (e1x * px + e1y * py) + e1z * pz;
        int ok = std::abs(det) > 1e-8f;
        float invDet = 1.0f / det;
        float tx = ox - v0x[l], ty = oy - v0y[l], tz = oz - v0z[l];
        float u = ((tx * px + ty * py) + tz * pz) * invDet;
        ok = ok & (u >= 0.0f) & (u <= 1.0f);
        float qx = ty * e1z - tz * e1y;
        float qy = tz * e1x - tx * e1z;
        float qz = tx * e1y - ty * e1x;
        float v = ((dx * qx + dy * qy) + dz * qz) * invDet;
        ok = ok & (v >= 0.0f) & (u + v <= 1.0f);
        float t = ((e2x * qx + e2y * qy) + e2z * qz) * invDet;
        ok = ok & (t > tMin) & (t < tMax);
        tA[l] = t; uA[l] = u; vA[l] = v; valid[l] = ok;
    }
}

// mesh.cpp:231-326 (four lanes per pack, same operation order as the Highway code)
bool Mesh::rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats* st) const {
    const float ox = ray.o.x, oy = ray.o.y, oz = ray.o.z;
    const float dx = ray.d.x, dy = ray.d.y, dz = ray.d.z;
    auto leafFn = [&](int offset, int count) -> bool {
        bool hitLocal = false;
        float tMaxPack = ray.tMax;
        for (int p = 0; p < count; ++p) {
            const TrianglePack4& pk = packs[offset + p];
            float tA[4], uA[4], vA[4];
            int valid[4];
            if (st) st->tris += 4;
            packTest(pk, ox, oy, oz, dx, dy, dz, ray.tMin, tMaxPack, tA, uA, vA, valid);
            for (int l = 0; l < 4; ++l) {
                if (valid[l] && tA[l] < ray.tMax) {
                    if (predicate) return true;
                    ray.tMax = tA[l];
                    tMaxPack = ray.tMax;
                    si.t = tA[l];
                    si.uv = Vec2(uA[l], vA[l]);
                    si.primIndex = pk.primIndex[l];
                    hitLocal = true;
                }
            }
        }
        return hitLocal;
    };
    return traverseBVH4(nodes4, ray, predicate, leafFn, st);
}

// mesh.cpp:328-390
void Mesh::fillInteraction(const Ray&, SurfaceInteraction& si) const {
    uint32_t i0 = indices[si.primIndex * 3 + 0], i1 = indices[si.primIndex * 3 + 1], i2 = indices[si.primIndex * 3 + 2];
    const Vec3& p0 = positions[i0];
    const Vec3& p1 = positions[i1];
    const Vec3& p2 = positions[i2];
    float u = si.uv.x, v = si.uv.y;
    float w = 1.0f - u - v;
    si.p = (p0 * w + p1 * u) + p2 * v;
    if (!normals.empty()) {
        si.n = Normalize((normals[i0] * w + normals[i1] * u) + normals[i2] * v);
    } else {
        si.n = Normalize(Cross(positions[i1] - positions[i0], positions[i2] - positions[i0]));
    }
    auto fallbackDpdu = [&]() {
        if (std::abs(si.n.x) > std::abs(si.n.y))
            return Vec3(-si.n.z, 0.0f, si.n.x) / std::sqrt(si.n.x * si.n.x + si.n.z * si.n.z);
        return Vec3(0.0f, si.n.z, -si.n.y) / std::sqrt(si.n.y * si.n.y + si.n.z * si.n.z);
    };
    if (!uvs.empty()) {
        Vec2 uv0 = uvs[i0], uv1 = uvs[i1], uv2 = uvs[i2];
        si.uv = Vec2((uv0.x * w + uv1.x * u) + uv2.x * v, (uv0.y * w + uv1.y * u) + uv2.y * v);
        Vec3 dp1 = p1 - p0, dp2 = p2 - p0;
        Vec2 duv1 = uv1 - uv0, duv2 = uv2 - uv0;
        float det = duv1.x * duv2.y - duv1.y * duv2.x;
        Vec3 dpdu;
        if (std::abs(det) < 1e-8f) dpdu = fallbackDpdu();
        else {
            float invDet = 1.0f / det;
            dpdu = (dp1 * duv2.y - dp2 * duv1.y) * invDet;
        }
        si.dpdu = Normalize(dpdu - si.n * Dot(si.n, dpdu));
    } else {
        si.dpdu = Normalize(fallbackDpdu());
    }
}

// mesh.cpp:396-434
float Mesh::sampleSurface(const Vec3&, const Vec2& s, SurfaceInteraction& info) const {
    if (totalArea == 0.0f) return 0.0f;
    auto it = std::lower_bound(cdf.begin(), cdf.end(), s.x);
    size_t tri = (size_t)std::distance(cdf.begin(), it);
    tri = std::clamp(tri, (size_t)1, cdf.size() - 1) - 1;
    float pdfTri = cdf[tri + 1] - cdf[tri];
    float rx = (s.x - cdf[tri]) / pdfTri;
    rx = std::clamp(rx, 0.0f, 1.0f);
    float sq = std::sqrt(rx);
    float u = 1.0f - sq;
    float v = s.y * sq;
    float w = 1.0f - u - v;
    uint32_t i0 = indices[tri * 3 + 0], i1 = indices[tri * 3 + 1], i2 = indices[tri * 3 + 2];
    info.p = (positions[i0] * w + positions[i1] * u) + positions[i2] * v;
    if (!normals.empty()) info.n = Normalize((normals[i0] * w + normals[i1] * u) + normals[i2] * v);
    else info.n = Normalize(Cross(positions[i1] - positions[i0], positions[i2] - positions[i0]));
    if (!uvs.empty())
        info.uv = Vec2((uvs[i0].x * w + uvs[i1].x * u) + uvs[i2].x * v, (uvs[i0].y * w + uvs[i1].y * u) + uvs[i2].y * v);
    return 1.0f / totalArea;
}

// ---------------------------------------------------------------- sphere, cube

// sphere.cpp:15-39
bool Sphere::rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats*) const {
    Vec3 ov = ray.o;
    float A = ray.d.lengthSquared();
    float B = 2.0f * Dot(ov, ray.d);
    float C = ov.lengthSquared() - (radius * radius);
    float t0, t1;
    if (!SolveQuadratic(A, B, C, t0, t1)) return false;
    float tHit;
    if (t0 > ray.tMin && t0 < ray.tMax) tHit = t0;
    else if (t1 > ray.tMin && t1 < ray.tMax) tHit = t1;
    else return false;
    if (predicate) return true;
    si.t = tHit;
    return true;
}
static void sphereUV(SurfaceInteraction& si) {
    float phi = std::atan2(si.n.x, si.n.z);
    if (phi < 0.0f) phi = (float)(phi + 2.0f * M_PI);
    float u = phi * Inv2Pi;
    float theta = std::acos(std::clamp(si.n.y, -1.0f, 1.0f));
    float v = theta * InvPi;
    si.uv = Vec2(u, v);
    si.dpdu = Vec3((float)(si.p.z * 2.0f * M_PI), 0.0f, (float)(-si.p.x * 2.0f * M_PI));
}
// sphere.cpp:41-55
void Sphere::fillInteraction(const Ray& ray, SurfaceInteraction& si) const {
    si.p = ray.o + ray.d * si.t;
    si.n = Normalize(si.p);
    sphereUV(si);
}
// sphere.cpp:64-81
float Sphere::sampleSurface(const Vec3&, const Vec2& s, SurfaceInteraction& info) const {
    Vec3 res = warp::squareToUniformSphere(s);
    info.p = res * radius;
    info.n = Normalize(info.p);
    sphereUV(info);
    return Inv4Pi / (radius * radius);
}

// cube.cpp:16-46
bool Cube::rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats*) const {
    float t0 = 0.0f, t1 = ray.tMax;
    for (int i = 0; i < 3; ++i) {
        float inv = 1.0f / ray.d[i];
        float tn = (mn[i] - ray.o[i]) * inv;
        float tf = (mx[i] - ray.o[i]) * inv;
        if (tn > tf) std::swap(tn, tf);
        t0 = tn > t0 ? tn : t0;
        t1 = tf < t1 ? tf : t1;
        if (t0 > t1) return false;
    }
    float tHit = t0;
    if (tHit < ray.tMin) {
        tHit = t1;
        if (tHit < ray.tMin) return false;
    }
    if (predicate) return true;
    si.t = tHit;
    return true;
}
// cube.cpp:48-81
void Cube::fillInteraction(const Ray& ray, SurfaceInteraction& si) const {
    si.p = ray.o + ray.d * si.t;
    Vec3 dmin = si.p - mn, dmax = mx - si.p;
    float minDist = std::numeric_limits<float>::max();
    int axis = 0;
    float sign = 1.0f;
    for (int i = 0; i < 3; ++i) {
        if (dmin[i] < minDist) { minDist = dmin[i]; axis = i; sign = -1.0f; }
        if (dmax[i] < minDist) { minDist = dmax[i]; axis = i; sign = 1.0f; }
    }
    si.n = Vec3(0.0f);
    si.n[axis] = sign;
    if (axis == 0) {
        si.uv = Vec2((si.p.z - mn.z) / (2.0f * ext.z), (si.p.y - mn.y) / (2.0f * ext.y));
        si.dpdu = Vec3(0.0f, 0.0f, 2.0f * ext.z * sign);
    } else if (axis == 1) {
        si.uv = Vec2((si.p.x - mn.x) / (2.0f * ext.x), (si.p.z - mn.z) / (2.0f * ext.z));
        si.dpdu = Vec3(2.0f * ext.x * sign, 0.0f, 0.0f);
    } else {
        si.uv = Vec2((si.p.x - mn.x) / (2.0f * ext.x), (si.p.y - mn.y) / (2.0f * ext.y));
        si.dpdu = Vec3(2.0f * ext.x * sign, 0.0f, 0.0f);
    }
}
// cube.cpp:83-146
float Cube::sampleSurface(const Vec3&, const Vec2& s, SurfaceInteraction& info) const {
    float areaX = 4.0f * ext.y * ext.z, areaY = 4.0f * ext.x * ext.z, areaZ = 4.0f * ext.x * ext.y;
    float total = 2.0f * (areaX + areaY + areaZ);
    float fp[6] = {areaX / total, areaX / total, areaY / total, areaY / total, areaZ / total, areaZ / total};
    Vec2 u = s;
    int face = 0;
    float c = 0.0f;
    for (int i = 0; i < 6; ++i) {
        c += fp[i];
        if (u.x < c || i == 5) { face = i; float prev = c - fp[i]; u.x = (u.x - prev) / fp[i]; break; }
    }
    float sign = (face % 2 == 0) ? 1.0f : -1.0f;
    if (face < 2) {
        info.p = Vec3(ext.x * sign, mn.y + u.x * (2.0f * ext.y), mn.z + u.y * (2.0f * ext.z));
        info.n = Vec3(sign, 0.0f, 0.0f);
        info.uv = Vec2((info.p.z - mn.z) / (2.0f * ext.z), (info.p.y - mn.y) / (2.0f * ext.y));
    } else if (face < 4) {
        info.p = Vec3(mn.x + u.x * (2.0f * ext.x), ext.y * sign, mn.z + u.y * (2.0f * ext.z));
        info.n = Vec3(0.0f, sign, 0.0f);
        info.uv = Vec2((info.p.x - mn.x) / (2.0f * ext.x), (info.p.z - mn.z) / (2.0f * ext.z));
    } else {
        info.p = Vec3(mn.x + u.x * (2.0f * ext.x), mn.y + u.y * (2.0f * ext.y), ext.z * sign);
        info.n = Vec3(0.0f, 0.0f, sign);
        info.uv = Vec2((info.p.x - mn.x) / (2.0f * ext.x), (info.p.y - mn.y) / (2.0f * ext.y));
    }
    return 1.0f / total;
}

// ---------------------------------------------------------------- primitive, scene BVH

// primitive.cpp:48-59 (worldToObject = the interpolated transform's inverse)
bool Primitive::rayIntersect(const Ray& rWorld, SurfaceInteraction& si, bool predicate, TraversalStats* st) const {
    Ray rLocal = anim.interpolate(rWorld.time).inverse().ray(rWorld);
    if (!shape->rayIntersect(rLocal, si, predicate, st)) return false;
    si.primitive = this;
    return true;
}
// primitive.cpp:61-72
void Primitive::fillInteraction(const Ray& rWorld, SurfaceInteraction& si) const {
    const Transform tw = anim.interpolate(rWorld.time);
    Ray rLocal = tw.inverse().ray(rWorld);
    shape->fillInteraction(rLocal, si);
    si.p = tw.point(si.p);
    si.n = Normalize(tw.normal(si.n));
    si.dpdu = Normalize(tw.vector(si.dpdu));
    si.time = rWorld.time;
}

// bvh.cpp:10-36
void Scene::buildTLAS() {
    if (prims.empty()) return;
    std::vector<BVHBuildInfo> bd;
    bd.reserve(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) {
        Bounds3 b = prims[i]->getWorldBounds();
        bd.push_back({b, b.pMin * 0.5f + b.pMax * 0.5f, (int)i});
    }
    BVHBuildResult r = buildBVH(bd);
    if (!r.nodes.empty()) bounds = r.nodes[0].bounds;
    std::vector<std::shared_ptr<Primitive>> ordered(prims.size());
    for (size_t i = 0; i < r.orderedIndices.size(); ++i) ordered[i] = prims[r.orderedIndices[i]];
    prims = std::move(ordered);
    if (!r.nodes.empty()) nodes4 = buildWide(r.nodes);
}

// bvh.cpp:38-66
bool Scene::rayIntersect(const Ray& ray, SurfaceInteraction& si, TraversalStats* st) const {
    si.t = std::numeric_limits<float>::max();
    auto leafFn = [&](int offset, int count) -> bool {
        bool hitLocal = false;
        for (int p = 0; p < count; ++p) {
            SurfaceInteraction its;
            if (prims[offset + p]->rayIntersect(ray, its, false, st)) {
                if (its.t < si.t) {
                    ray.tMax = its.t;
                    si = its;
                    hitLocal = true;
                }
            }
        }
        return hitLocal;
    };
    bool hit = traverseBVH4(nodes4, ray, false, leafFn, st);
    if (hit) si.primitive->fillInteraction(ray, si);
    return hit;
}
// bvh.cpp:38-66 with shadowRay=true (scene.cpp:68-71)
bool Scene::occluded(const Ray& ray, TraversalStats* st) const {
    auto leafFn = [&](int offset, int count) -> bool {
        for (int p = 0; p < count; ++p) {
            SurfaceInteraction its;
            if (prims[offset + p]->rayIntersect(ray, its, true, st)) return true;
        }
        return false;
    };
    return traverseBVH4(nodes4, ray, true, leafFn, st);
}

}  // namespace orc
