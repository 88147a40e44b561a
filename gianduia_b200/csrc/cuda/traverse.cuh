// Two-level BVH4 traversal on the device: one thread per ray, the traversal stack in
// shared memory (entry k of thread t at smem[k * BLOCK + t], bank-conflict free), hit
// children pushed farthest-first so the nearest is visited next.
//
// Arithmetic follows the reference bit for bit (the file is compiled without FMA
// contraction): the slab test of bvhTraversal.h:57-72 including its NaN behaviour
// (min/max return the second operand when a lane is NaN, as SSE minps/maxps do), the
// Moller-Trumbore test of mesh.cpp:259-291, the world-to-object ray transform of
// primitive.cpp:48-59 (object-space tMin reset to 1e-4, direction not renormalised),
// and the sphere / cube tests of sphere.cpp:15-39 and cube.cpp:16-46.
// Visit order differs from the reference (which pushes children in index order
// without sorting), so among hits at exactly equal t a different primitive may win.
#pragma once
#include "gnd/layout.h"

namespace gnd {

struct TRay {
    V3 o, d;
    float tmin, tmax;
};

struct THit {
    float t, u, v;
    int32_t inst;     // instance (primitive in scene-file order), -1 on a miss
    uint32_t slot;    // leaf-order triangle slot (meshes); 0xFFFFFFFF for analytic shapes
};

enum TraceError : int { kTraceOk = 0, kTraceStackOverflow = 1, kTraceIterLimit = 2, kTraceBadRef = 4 };

constexpr int kStackSize = 64;
constexpr uint32_t kSentinel = 0xFFFFFFFEu;
constexpr uint32_t kMaxIterations = 1u << 22;

__device__ __forceinline__ float4 ldg4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ uint4 ldgu4(const void* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

// Reference-exact lane min / max (SSE semantics).
__device__ __forceinline__ float lmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float lmax(float a, float b) { return a > b ? a : b; }

struct TraceCounters {
    uint32_t nodes, tris;
};

// Moller-Trumbore against the object-space ray (mesh.cpp:259-291). Returns true when the
// triangle is hit with tmin < t < tmax; writes t, u, v.
__device__ __forceinline__ bool triTest(const Tri* tp, V3 o, V3 d, float tmin, float tmax, float& t, float& u,
                                        float& v, uint32_t& prim) {
    float4 a = ldg4(&tp->v0x), b = ldg4(&tp->v1x), c = ldg4(&tp->v2x);
    float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
    float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
    float px = d.y * e2z - d.z * e2y;
    float py = d.z * e2x - d.x * e2z;
    float pz = d.x * e2y - d.y * e2x;
    float det = (e1x * px + e1y * py) + e1z * pz;
    bool ok = fabsf(det) > 1e-8f;
    float invDet = __frcp_rn(det);
    float tx = o.x - a.x, ty = o.y - a.y, tz = o.z - a.z;
    u = ((tx * px + ty * py) + tz * pz) * invDet;
    ok = ok && (u >= 0.0f) && (u <= 1.0f);
    float qx = ty * e1z - tz * e1y;
    float qy = tz * e1x - tx * e1z;
    float qz = tx * e1y - ty * e1x;
    v = ((d.x * qx + d.y * qy) + d.z * qz) * invDet;
    ok = ok && (v >= 0.0f) && (u + v <= 1.0f);
    t = ((e2x * qx + e2y * qy) + e2z * qz) * invDet;
    ok = ok && (t > tmin) && (t < tmax);
    prim = __float_as_uint(a.w);
    return ok;
}

// sphere.cpp:15-39 (object space)
__device__ __forceinline__ bool sphereTest(float radius, V3 o, V3 d, float tmin, float tmax, float& tHit) {
    float A = dot(d, d);
    float B = 2.0f * dot(o, d);
    float C = dot(o, o) - (radius * radius);
    float discrim = B * B - 4.0f * A * C;
    if (discrim < 0) return false;
    float rd = sqrtf(discrim);
    float t0 = (-B - rd) / (2.0f * A);
    float t1 = (-B + rd) / (2.0f * A);
    if (t0 > tmin && t0 < tmax) { tHit = t0; return true; }
    if (t1 > tmin && t1 < tmax) { tHit = t1; return true; }
    return false;
}

// cube.cpp:16-46 (object space, extents ex)
__device__ __forceinline__ bool cubeTest(V3 ex, V3 o, V3 d, float tmin, float tmax, float& tHit) {
    float t0 = 0.0f, t1 = tmax;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float inv = 1.0f / comp(d, i);
        float oi = comp(o, i), e = comp(ex, i);
        float tn = (-e - oi) * inv;
        float tf = (e - oi) * inv;
        if (tn > tf) { float s = tn; tn = tf; tf = s; }
        t0 = tn > t0 ? tn : t0;
        t1 = tf < t1 ? tf : t1;
        if (t0 > t1) return false;
    }
    float th = t0;
    if (th < tmin) {
        th = t1;
        if (th < tmin) return false;
    }
    tHit = th;
    return true;
}

// Trace one ray. ANY: stop at the first hit (occlusion query). SKIP_NULL: ignore
// instances whose material has no BSDF (index material) -- used by the path
// integrator's shadow rays. COUNT: accumulate node visits and triangle tests.
// `stk` points at this thread's first stack entry in shared memory; entries are
// BLOCK apart. Returns an error bitmask (0 on success).
template <int BLOCK, bool ANY, bool SKIP_NULL, bool COUNT>
__device__ __forceinline__ int traceRay(const SceneView& s, const TRay& ray, THit& hit, uint32_t* stk,
                                        TraceCounters* cnt, const uint8_t* nullMask) {
    hit.t = INFINITY;
    hit.u = hit.v = 0.f;
    hit.inst = -1;
    hit.slot = 0xFFFFFFFFu;
    if (s.tlasRoot == kEmpty) return kTraceOk;
    const V3 wo = ray.o, wd = ray.d;
    const float wtmin = ray.tmin;
    float tmax = ray.tmax;          // shrinks with every accepted hit
    float bestT = 3.402823466e38f;  // bvh.cpp:39 (FLT_MAX)
    V3 o = wo, d = wd;
    V3 inv = v3(__frcp_rn(wd.x), __frcp_rn(wd.y), __frcp_rn(wd.z));
    float tmin = wtmin;
    int curInst = -1;
    int sp = 0;
    stk[0] = s.tlasRoot;
    sp = 1;
    uint32_t iter = 0;
    int err = 0;
    while (sp > 0) {
        if (++iter > kMaxIterations) { err |= kTraceIterLimit; break; }
        uint32_t e = stk[(--sp) * BLOCK];
        if (e == kSentinel) {
            // leave the bottom-level tree: back to the world-space ray
            o = wo; d = wd;
            inv = v3(__frcp_rn(wd.x), __frcp_rn(wd.y), __frcp_rn(wd.z));
            tmin = wtmin;
            curInst = -1;
            continue;
        }
        if (!isLeaf(e)) {
            const Node4* nd = s.nodes + e;
            if (COUNT) cnt->nodes++;
            float4 lx = ldg4(nd->lox), hx = ldg4(nd->hix), ly = ldg4(nd->loy);
            float4 hy = ldg4(nd->hiy), lz = ldg4(nd->loz), hz = ldg4(nd->hiz);
            uint4 ch = ldgu4(nd->child);
            float key[4];
            uint32_t ref[4] = {ch.x, ch.y, ch.z, ch.w};
            const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, HX[4] = {hx.x, hx.y, hx.z, hx.w};
            const float LY[4] = {ly.x, ly.y, ly.z, ly.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w};
            const float LZ[4] = {lz.x, lz.y, lz.z, lz.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                float t1x = (LX[i] - o.x) * inv.x, t2x = (HX[i] - o.x) * inv.x;
                float t1y = (LY[i] - o.y) * inv.y, t2y = (HY[i] - o.y) * inv.y;
                float t1z = (LZ[i] - o.z) * inv.z, t2z = (HZ[i] - o.z) * inv.z;
                float tn = lmax(lmax(lmin(t1x, t2x), lmin(t1y, t2y)), lmax(lmin(t1z, t2z), tmin));
                float tf = lmin(lmin(lmax(t1x, t2x), lmax(t1y, t2y)), lmin(lmax(t1z, t2z), tmax));
                key[i] = (tn <= tf && ref[i] != kEmpty) ? tn : INFINITY;
            }
            // ascending sort network on (key, ref)
#define GND_CSWAP(a, b)                                                          \
    if (key[b] < key[a]) {                                                       \
        float tk = key[a]; key[a] = key[b]; key[b] = tk;                         \
        uint32_t tr = ref[a]; ref[a] = ref[b]; ref[b] = tr;                      \
    }
            GND_CSWAP(0, 1) GND_CSWAP(2, 3) GND_CSWAP(0, 2) GND_CSWAP(1, 3) GND_CSWAP(1, 2)
#undef GND_CSWAP
#pragma unroll
            for (int i = 3; i >= 0; --i) {
                if (key[i] != INFINITY) {
                    if (sp >= kStackSize) { err |= kTraceStackOverflow; break; }
                    stk[(sp++) * BLOCK] = ref[i];
                }
            }
            if (err) break;
            continue;
        }
        // leaf
        uint32_t first = leafFirst(e), count = leafCount(e);
        if (curInst >= 0) {
            // bottom level: triangles [first, first + count)
            for (uint32_t k = 0; k < count; ++k) {
                float t, u, v;
                uint32_t prim;
                if (COUNT) cnt->tris++;
                if (triTest(s.tris + first + k, o, d, tmin, tmax, t, u, v, prim)) {
                    if (ANY) { hit.t = t; hit.inst = curInst; hit.slot = first + k; return err; }
                    tmax = t;
                    bestT = t;
                    hit.t = t; hit.u = u; hit.v = v;
                    hit.inst = curInst;
                    hit.slot = first + k;
                }
            }
            continue;
        }
        // top level: instances tlasList[first .. first + count)
        for (uint32_t k = 0; k < count; ++k) {
            uint32_t id = __ldg(s.tlasList + first + k);
            if (SKIP_NULL && nullMask && nullMask[id]) continue;
            const InstTrav* it = s.instT + id;
            float4 r0 = ldg4(&it->w2o.r[0][0]), r1 = ldg4(&it->w2o.r[1][0]), r2 = ldg4(&it->w2o.r[2][0]);
            float4 meta = ldg4(&it->kind);
            uint32_t kind = __float_as_uint(meta.x);
            // primitive.cpp:49-50: rLocal = worldToObject(rWorld), tMin = Epsilon
            V3 lo, ld;
            lo.x = (r0.x * wo.x + r0.y * wo.y) + (r0.z * wo.z + r0.w);
            lo.y = (r1.x * wo.x + r1.y * wo.y) + (r1.z * wo.z + r1.w);
            lo.z = (r2.x * wo.x + r2.y * wo.y) + (r2.z * wo.z + r2.w);
            ld.x = (r0.x * wd.x + r0.y * wd.y) + (r0.z * wd.z + r0.w * 0.0f);
            ld.y = (r1.x * wd.x + r1.y * wd.y) + (r1.z * wd.z + r1.w * 0.0f);
            ld.z = (r2.x * wd.x + r2.y * wd.y) + (r2.z * wd.z + r2.w * 0.0f);
            if (kind == kShapeMesh) {
                uint32_t root = __float_as_uint(meta.y);
                if (root == kEmpty) continue;
                // remaining instances of this leaf come back after the bottom level
                if (k + 1 < count) {
                    if (sp >= kStackSize) { err |= kTraceStackOverflow; break; }
                    stk[(sp++) * BLOCK] = makeLeaf(first + k + 1, count - k - 1);
                }
                if (sp + 2 > kStackSize) { err |= kTraceStackOverflow; break; }
                stk[(sp++) * BLOCK] = kSentinel;
                stk[(sp++) * BLOCK] = root;
                o = lo; d = ld;
                inv = v3(__frcp_rn(ld.x), __frcp_rn(ld.y), __frcp_rn(ld.z));
                tmin = kEpsilon;
                curInst = (int)id;
                break;
            }
            float th;
            bool h;
            if (kind == kShapeSphere) {
                h = sphereTest(meta.z, lo, ld, kEpsilon, tmax, th);
            } else {
                float ez = __ldg(&s.instS[id].ext[2]);
                h = cubeTest(v3(meta.z, meta.w, ez), lo, ld, kEpsilon, tmax, th);
            }
            if (h && th < bestT) {
                if (ANY) { hit.t = th; hit.inst = (int)id; return err; }
                tmax = th;
                bestT = th;
                hit.t = th; hit.u = 0.f; hit.v = 0.f;
                hit.inst = (int)id;
                hit.slot = 0xFFFFFFFFu;
            }
        }
        if (err) break;
    }
    return err;
}

}  // namespace gnd
