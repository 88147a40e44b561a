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
#include "gnd/motion.h"

namespace gnd {

struct TRay {
    V3 o, d;
    float tmin, tmax;
    float time = 0.0f;   // shutter time; moves animated instances (primitive.cpp:48-50)
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

// Work counters of the counting variants: node visits and triangle tests per lane, and
// for the phases of the persistent loop (persistentTrace) the warp steps of each phase
// (counted by lane 0) and the lanes' leaf steps, so that lanes busy per step = lane steps
// / (32 x warp steps).
struct TraceCounters {
    uint32_t nodes, tris;
    uint32_t nodeWarpSteps, leafSteps, leafWarpSteps;
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

// World-to-object rows of animated instance `id` at `time` (primitive.cpp:49:
// m_objectToWorld.interpolate(time).inverse()); r0..r2 hold the start transform's rows on
// entry, which stay for time <= 0. Only the MOTION variants of the traversal call it
// (scenes with animated instances); rays at time 0 (user ray batches) need none.
__device__ __forceinline__ void animatedW2ORows(const SceneView& s, uint32_t id, float time, float4& r0, float4& r1, float4& r2) {
    if (time <= 0.0f) return;
    Xf34 w;
    if (time >= 1.0f) {
        w = s.motion[id].endW2O;
    } else {
        Xf34 m;
        motionCompose(s.motion[id], (time - 0.0f) / (1.0f - 0.0f), m, w);
    }
    r0 = make_float4(w.r[0][0], w.r[0][1], w.r[0][2], w.r[0][3]);
    r1 = make_float4(w.r[1][0], w.r[1][1], w.r[1][2], w.r[1][3]);
    r2 = make_float4(w.r[2][0], w.r[2][1], w.r[2][2], w.r[2][3]);
}

// Trace one ray. ANY: stop at the first hit (occlusion query). SKIP_NULL: ignore
// instances whose material has no BSDF (index material) -- used by the path
// integrator's shadow rays. COUNT: accumulate node visits and triangle tests.
// `stk` points at this thread's first stack entry in shared memory; entries are
// BLOCK apart. Returns an error bitmask (0 on success).
template <int BLOCK, bool ANY, bool SKIP_NULL, bool COUNT, bool MOTION = false>
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
            if (MOTION && (kind & kInstAnimated)) animatedW2ORows(s, id, ray.time, r0, r1, r2);
            kind &= ~kInstAnimated;
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

// ---------------------------------------------------------------- persistent traversal
// The same traversal as traceRay, restated as an incremental per-lane state machine for
// persistent warps: lanes that finish a ray fetch the next one (warp-aggregated atomic on
// a per-launch counter), and each round runs a node phase (every lane pops and tests
// inner nodes until it holds a leaf) followed by a leaf phase (one primitive per step),
// so the warp executes one code path at a time. Stack entries 0 .. SMEM-1 live in shared
// memory and deeper ones in a per-lane local array (SMEM is a template parameter, 32 by
// default), so shallow stacks never leave shared memory.
constexpr int kSmemStack = 32;
constexpr int kPStackMax = 128;   // entries per ray, shared + local

struct Trav {
    V3 wo, wd;          // world ray
    float time;         // shutter time (animated instances)
    V3 o, d, inv;       // current ray (world, or object space inside a bottom-level tree)
    float wtmin, tmin, tmax, bestT;
    int curInst;
    int sp;
    bool fast, wfast;   // current / world ray: nodeKeysFast applies (see there)
    uint32_t next;      // entry to visit next without a stack round trip, kEmpty when none
    uint32_t leaf;      // pending primitives (a leaf reference advanced past those done), kEmpty when none
    THit hit;           // t unused: a hit's distance is bestT (travHit)
};

// SMEM: entries kept in shared memory (the block's array holds SMEM * BLOCK words); the
// remaining kPStackMax - SMEM entries live in a per-lane local array.
template <int BLOCK, int SMEM = kSmemStack>
struct TStack {
    static_assert(SMEM > 0 && SMEM < kPStackMax, "shared part of the stack out of range");
    uint32_t* smem;                 // this lane's column in the block's shared array
    uint32_t local[kPStackMax - SMEM];
    __device__ __forceinline__ void put(int k, uint32_t v) {
        if (k < SMEM) smem[k * BLOCK] = v;
        else local[k - SMEM] = v;
    }
    __device__ __forceinline__ uint32_t get(int k) const { return k < SMEM ? smem[k * BLOCK] : local[k - SMEM]; }
};

// True when (bound - o) * inv cannot be NaN for any finite or infinite node bound: the
// origin is finite and every inverse direction component is finite and non-zero.
__device__ __forceinline__ bool slabFinite(const SceneView& s, V3 o, V3 inv) {
    const bool f = isfinite(o.x) && isfinite(o.y) && isfinite(o.z) && isfinite(inv.x) && isfinite(inv.y) &&
                   isfinite(inv.z) && inv.x != 0.0f && inv.y != 0.0f && inv.z != 0.0f;
    return s.fastBoxes && f;
}

__device__ __forceinline__ void travInit(Trav& t, const SceneView& s, const TRay& ray) {
    t.wo = ray.o; t.wd = ray.d;
    t.o = ray.o; t.d = ray.d;
    t.inv = v3(__frcp_rn(ray.d.x), __frcp_rn(ray.d.y), __frcp_rn(ray.d.z));
    t.fast = t.wfast = slabFinite(s, t.o, t.inv) && !isnan(ray.tmin) && !isnan(ray.tmax);
    t.wtmin = ray.tmin; t.tmin = ray.tmin; t.tmax = ray.tmax;
    t.time = ray.time;
    t.bestT = 3.402823466e38f;
    t.curInst = -1;
    t.leaf = kEmpty;
    t.next = kEmpty;
    t.hit.t = INFINITY; t.hit.u = t.hit.v = 0.f; t.hit.inst = -1; t.hit.slot = 0xFFFFFFFFu;
    t.sp = 0;
}

// Visit-order key of a hit child: the entry distance's bits with the child slot in the
// two lowest bits, so that unsigned comparison orders children nearest first (distances
// within 3 ulp fall back to slot order; a negative distance, possible only with a
// negative tMin, sorts by magnitude). Order affects only which of several hits at
// exactly equal t is reported, never whether or where a hit is found.
constexpr uint32_t kMissKey = 0xFFFFFFFFu;
__device__ __forceinline__ uint32_t packKey(float a, int slot) {
    return (__float_as_uint(a) & 0x7FFFFFFCu) | (uint32_t)slot;
}

// Child entry distances of one node for the current ray (bvhTraversal.h:57-72) as visit
// keys; kMissKey for a missed or empty child. nodeKeysExact is the reference's lane arithmetic with
// SSE min/max (the second operand when either is NaN), for any ray and any bounds.
__device__ __forceinline__ void nodeKeysExact(const Node4* nd, const Trav& t, const uint32_t ref[4], uint32_t key[4]) {
    float4 lx = ldg4(nd->lox), hx = ldg4(nd->hix);
    float t1[4] = {(lx.x - t.o.x) * t.inv.x, (lx.y - t.o.x) * t.inv.x, (lx.z - t.o.x) * t.inv.x, (lx.w - t.o.x) * t.inv.x};
    float t2[4] = {(hx.x - t.o.x) * t.inv.x, (hx.y - t.o.x) * t.inv.x, (hx.z - t.o.x) * t.inv.x, (hx.w - t.o.x) * t.inv.x};
    float tn[4], tf[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { tn[i] = lmin(t1[i], t2[i]); tf[i] = lmax(t1[i], t2[i]); }
    float4 ly = ldg4(nd->loy), hy = ldg4(nd->hiy);
    float u1[4] = {(ly.x - t.o.y) * t.inv.y, (ly.y - t.o.y) * t.inv.y, (ly.z - t.o.y) * t.inv.y, (ly.w - t.o.y) * t.inv.y};
    float u2[4] = {(hy.x - t.o.y) * t.inv.y, (hy.y - t.o.y) * t.inv.y, (hy.z - t.o.y) * t.inv.y, (hy.w - t.o.y) * t.inv.y};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        tn[i] = lmax(tn[i], lmin(u1[i], u2[i]));
        tf[i] = lmin(tf[i], lmax(u1[i], u2[i]));
    }
    float4 lz = ldg4(nd->loz), hz = ldg4(nd->hiz);
    float w1[4] = {(lz.x - t.o.z) * t.inv.z, (lz.y - t.o.z) * t.inv.z, (lz.z - t.o.z) * t.inv.z, (lz.w - t.o.z) * t.inv.z};
    float w2[4] = {(hz.x - t.o.z) * t.inv.z, (hz.y - t.o.z) * t.inv.z, (hz.z - t.o.z) * t.inv.z, (hz.w - t.o.z) * t.inv.z};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        // bvhTraversal.h:69-72: max(max(x, y), max(z, tMin)) <= min(min(x, y), min(z, tMax))
        float a = lmax(tn[i], lmax(lmin(w1[i], w2[i]), t.tmin));
        float b = lmin(tf[i], lmin(lmax(w1[i], w2[i]), t.tmax));
        key[i] = (a <= b && ref[i] != kEmpty) ? packKey(a, i) : kMissKey;
    }
}

// The same distances with less work, for rays and nodes where it gives the same values
// (t.fast: finite origin, finite non-zero inverse direction; fastBoxes: no NaN bound and
// lo <= hi for every non-empty child). Then no slab term is NaN, so min/max are the
// hardware ones, and because (bound - o) * inv is monotone in the bound, the smaller of
// the two planes of an axis is the lo plane when inv > 0 and the hi plane when inv < 0:
// the near and far planes are chosen once per axis from the direction's sign instead of
// by a min/max per child. Empty children (ref kEmpty) are discarded as before. The
// result may differ from nodeKeysExact only in the sign of a zero key, which no
// comparison sees.
__device__ __forceinline__ void nodeKeysFast(const Node4* nd, const Trav& t, const uint32_t ref[4], uint32_t key[4]) {
    const bool sx = t.inv.x < 0.0f, sy = t.inv.y < 0.0f, sz = t.inv.z < 0.0f;
    const float4 nx = ldg4(sx ? nd->hix : nd->lox), fx = ldg4(sx ? nd->lox : nd->hix);
    const float4 ny = ldg4(sy ? nd->hiy : nd->loy), fy = ldg4(sy ? nd->loy : nd->hiy);
    const float4 nz = ldg4(sz ? nd->hiz : nd->loz), fz = ldg4(sz ? nd->loz : nd->hiz);
    const float n0[4] = {nx.x, nx.y, nx.z, nx.w}, f0[4] = {fx.x, fx.y, fx.z, fx.w};
    const float n1[4] = {ny.x, ny.y, ny.z, ny.w}, f1[4] = {fy.x, fy.y, fy.z, fy.w};
    const float n2[4] = {nz.x, nz.y, nz.z, nz.w}, f2[4] = {fz.x, fz.y, fz.z, fz.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float tnx = (n0[i] - t.o.x) * t.inv.x, tfx = (f0[i] - t.o.x) * t.inv.x;
        const float tny = (n1[i] - t.o.y) * t.inv.y, tfy = (f1[i] - t.o.y) * t.inv.y;
        const float tnz = (n2[i] - t.o.z) * t.inv.z, tfz = (f2[i] - t.o.z) * t.inv.z;
        const float a = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, t.tmin));
        const float b = fminf(fminf(tfx, tfy), fminf(tfz, t.tmax));
        key[i] = (a <= b && ref[i] != kEmpty) ? packKey(a, i) : kMissKey;
    }
}

// Pops one entry: restores the world ray at a sentinel, tests an inner node and pushes its
// hit children nearest-last, or makes a leaf pending. Returns an error bitmask. Without
// ORDER (any-hit queries, whose answer does not depend on the visit order) the hit
// children are visited in slot order, which saves the sort.
template <int BLOCK, bool COUNT, int SMEM, bool ORDER = true>
__device__ __forceinline__ int travNodeStep(Trav& t, const SceneView& s, TStack<BLOCK, SMEM>& st, TraceCounters* cnt) {
    uint32_t e;
    if (t.next != kEmpty) {
        e = t.next;
        t.next = kEmpty;
    } else {
        e = st.get(--t.sp);
    }
    if (e == kSentinel) {
        t.o = t.wo; t.d = t.wd;
        t.inv = v3(__frcp_rn(t.wd.x), __frcp_rn(t.wd.y), __frcp_rn(t.wd.z));
        t.fast = t.wfast;
        t.tmin = t.wtmin;
        t.curInst = -1;
        return 0;
    }
    if (isLeaf(e)) {
        t.leaf = e;
        return 0;
    }
    const Node4* nd = s.nodes + e;
    if (COUNT) cnt->nodes++;
    uint32_t key[4];
    {
        const uint4 ch = ldgu4(nd->child);
        const uint32_t ref[4] = {ch.x, ch.y, ch.z, ch.w};
        if (t.fast) nodeKeysFast(nd, t, ref, key);
        else nodeKeysExact(nd, t, ref, key);
    }
    if (!ORDER) {
        const int nhit = (key[0] != kMissKey) + (key[1] != kMissKey) + (key[2] != kMissKey) + (key[3] != kMissKey);
        if (nhit == 0) return 0;
        if (t.sp + nhit - 1 > kPStackMax) return kTraceStackOverflow;
        uint32_t pending = kEmpty;
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            if (key[i] == kMissKey) continue;
            if (pending != kEmpty) st.put(t.sp++, pending);
            pending = __ldg(nd->child + i);
        }
        t.next = pending;
        return 0;
    }
    // ascending sort network on the packed keys (unsigned min / max)
#define GND_CSWAP(a, b)                                     \
    {                                                       \
        const uint32_t lo = min(key[a], key[b]);            \
        key[b] = max(key[a], key[b]);                       \
        key[a] = lo;                                        \
    }
    GND_CSWAP(0, 1) GND_CSWAP(2, 3) GND_CSWAP(0, 2) GND_CSWAP(1, 3) GND_CSWAP(1, 2)
#undef GND_CSWAP
    if (key[0] == kMissKey) return 0;
    const int npush = (key[1] != kMissKey) + (key[2] != kMissKey) + (key[3] != kMissKey);
    if (t.sp + npush > kPStackMax) return kTraceStackOverflow;
    // farther children on the stack (farthest deepest), the nearest visited next
#pragma unroll
    for (int i = 3; i >= 1; --i)
        if (key[i] != kMissKey) st.put(t.sp++, __ldg(nd->child + (key[i] & 3u)));
    t.next = __ldg(nd->child + (key[0] & 3u));
    return 0;
}

// Processes one primitive of the pending leaf. For ANY, a hit ends the ray (sp = 0).
template <int BLOCK, bool ANY, bool COUNT, int SMEM, bool MOTION>
__device__ __forceinline__ int travLeafStep(Trav& t, const SceneView& s, TStack<BLOCK, SMEM>& st, TraceCounters* cnt,
                                            const uint8_t* nullMask) {
    // the pending leaf's first primitive; the rest stays pending
    const uint32_t first = leafFirst(t.leaf), count = leafCount(t.leaf);
    t.leaf = count > 1u ? makeLeaf(first + 1u, count - 1u) : kEmpty;
    if (t.curInst >= 0) {
        float tt, u, v;
        uint32_t prim;
        if (COUNT) cnt->tris++;
        if (triTest(s.tris + first, t.o, t.d, t.tmin, t.tmax, tt, u, v, prim)) {
            t.tmax = tt;
            t.bestT = tt;
            t.hit.u = u; t.hit.v = v;
            t.hit.inst = t.curInst;
            t.hit.slot = first;
            if (ANY) { t.sp = 0; t.leaf = kEmpty; t.next = kEmpty; }
        }
        return 0;
    }
    uint32_t id = __ldg(s.tlasList + first);
    if (nullMask && nullMask[id]) return 0;
    const InstTrav* it = s.instT + id;
    float4 r0 = ldg4(&it->w2o.r[0][0]), r1 = ldg4(&it->w2o.r[1][0]), r2 = ldg4(&it->w2o.r[2][0]);
    float4 meta = ldg4(&it->kind);
    uint32_t kind = __float_as_uint(meta.x);
    if (MOTION && (kind & kInstAnimated)) animatedW2ORows(s, id, t.time, r0, r1, r2);
    kind &= ~kInstAnimated;
    V3 lo, ld;
    lo.x = (r0.x * t.wo.x + r0.y * t.wo.y) + (r0.z * t.wo.z + r0.w);
    lo.y = (r1.x * t.wo.x + r1.y * t.wo.y) + (r1.z * t.wo.z + r1.w);
    lo.z = (r2.x * t.wo.x + r2.y * t.wo.y) + (r2.z * t.wo.z + r2.w);
    ld.x = (r0.x * t.wd.x + r0.y * t.wd.y) + (r0.z * t.wd.z + r0.w * 0.0f);
    ld.y = (r1.x * t.wd.x + r1.y * t.wd.y) + (r1.z * t.wd.z + r1.w * 0.0f);
    ld.z = (r2.x * t.wd.x + r2.y * t.wd.y) + (r2.z * t.wd.z + r2.w * 0.0f);
    if (kind == kShapeMesh) {
        uint32_t root = __float_as_uint(meta.y);
        if (root == kEmpty) return 0;
        if (t.next != kEmpty) {
            // an entry found by speculative traversal before this leaf: keep it for later
            if (t.sp >= kPStackMax) return kTraceStackOverflow;
            st.put(t.sp++, t.next);
            t.next = kEmpty;
        }
        if (t.leaf != kEmpty) {
            // the rest of this leaf comes back after the bottom-level tree
            if (t.sp >= kPStackMax) return kTraceStackOverflow;
            st.put(t.sp++, t.leaf);
            t.leaf = kEmpty;
        }
        if (t.sp + 1 > kPStackMax) return kTraceStackOverflow;
        st.put(t.sp++, kSentinel);
        t.next = root;   // the bottom-level root is visited next
        t.o = lo; t.d = ld;
        t.inv = v3(__frcp_rn(ld.x), __frcp_rn(ld.y), __frcp_rn(ld.z));
        t.fast = t.wfast && slabFinite(s, lo, t.inv);
        t.tmin = kEpsilon;
        t.curInst = (int)id;
        return 0;
    }
    float th;
    bool h;
    if (kind == kShapeSphere) h = sphereTest(meta.z, lo, ld, kEpsilon, t.tmax, th);
    else h = cubeTest(v3(meta.z, meta.w, __ldg(&s.instS[id].ext[2])), lo, ld, kEpsilon, t.tmax, th);
    if (h && th < t.bestT) {
        t.tmax = th;
        t.bestT = th;
        t.hit.u = 0.f; t.hit.v = 0.f;
        t.hit.inst = (int)id;
        t.hit.slot = 0xFFFFFFFFu;
        if (ANY) { t.sp = 0; t.leaf = kEmpty; t.next = kEmpty; }
    }
    return 0;
}

// The hit a finished query reports: every accepted hit sets bestT to its distance.
__device__ __forceinline__ THit travHit(const Trav& t) {
    THit h = t.hit;
    h.t = t.hit.inst >= 0 ? t.bestT : INFINITY;
    return h;
}

// Warp-aggregated fetch of the next work index for lanes in `want`.
__device__ __forceinline__ uint32_t warpFetch(uint32_t* counter, bool want) {
    uint32_t mask = __ballot_sync(0xffffffffu, want);
    uint32_t base = 0;
    int lane = threadIdx.x & 31;
    if (mask) {
        int leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// Persistent traversal loop. Every lane of every warp runs it to the end (the block size
// is a multiple of 32 and no lane exits early). Src provides:
//   uint32_t count()                      number of rays
//   bool load(uint32_t i, TRay&, const SceneView*&, const uint8_t*& nullMask)
//   void store(uint32_t i, const THit&, const SceneView&)   (the query's scene)
// SLOT_ORDER_ANY: any-hit queries visit hit children in slot order instead of nearest
// first (faster for the bounded shadow segments of the path tracer; rays to infinity find
// an occluder sooner nearest first).
// leafBatch (1..32): the node phase ends as soon as that many lanes hold a leaf (32: when
// no lane can take another node step); lanes still traversing keep their state and go on
// in the next round. Only the interleaving of the lanes' steps changes.
template <int BLOCK, bool ANY, bool COUNT, int SMEM = kSmemStack, bool SPEC = false, bool MOTION = false,
          bool SLOT_ORDER_ANY = false, typename Src>
__device__ __forceinline__ int persistentTrace(Src& src, uint32_t* fetchCounter, uint32_t* smemStack, TraceCounters* cnt,
                                               uint32_t leafBatch = 32) {
    TStack<BLOCK, SMEM> st;
    st.smem = smemStack + threadIdx.x;
    Trav t;
    const SceneView* sv = nullptr;
    const uint8_t* nm = nullptr;
    bool active = false;
    bool drained = false;   // warp-uniform: the counter has passed n
    uint32_t idx = 0;
    int err = 0;
    const uint32_t n = src.count();
    uint32_t iter = 0;
    for (;;) {
        bool idle = !active && !drained;
        uint32_t got = warpFetch(fetchCounter, idle);
        if (__any_sync(0xffffffffu, idle && got >= n)) drained = true;
        if (idle && got < n) {
            idx = got;
            TRay r;
            // a source may decline an item (it belongs to another kernel of the launch)
            if (src.load(idx, r, sv, nm)) {
                travInit(t, *sv, r);
                t.next = sv->tlasRoot;   // kEmpty for a scene without primitives
                active = true;
                iter = 0;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        // node phase. Without SPEC a lane steps until it holds a leaf. With SPEC every lane
        // steps until it is blocked: a lane that holds a leaf keeps traversing ahead while
        // its next entry is an inner node of the same tree, and stops at the next leaf,
        // sentinel or an empty stack (more lanes busy per step, at the price of visits a
        // shorter tMax would have culled). Either way whether a lane steps depends only on
        // its own state, so each ray's sequence of visits, and its result, is the same
        // whatever the other rays of the warp do.
        for (;;) {
            const bool work = t.next != kEmpty || t.sp > 0;
            bool want = active && work;
            if (want && t.leaf != kEmpty) {
                if (!SPEC) {
                    want = false;
                } else {
                    const uint32_t peek = t.next != kEmpty ? t.next : st.get(t.sp - 1);
                    want = peek != kSentinel && !isLeaf(peek);
                }
            }
            if (!__any_sync(0xffffffffu, want)) break;
            if (leafBatch < 32u && (uint32_t)__popc(__ballot_sync(0xffffffffu, active && t.leaf != kEmpty)) >= leafBatch)
                break;
            if (COUNT && (threadIdx.x & 31) == 0) cnt->nodeWarpSteps++;
            if (want) {
                int e = travNodeStep<BLOCK, COUNT, SMEM, !(ANY && SLOT_ORDER_ANY)>(t, *sv, st, cnt);
                if (e || ++iter > kMaxIterations) {
                    err |= e ? e : (int)kTraceIterLimit;
                    t.sp = 0; t.leaf = kEmpty; t.next = kEmpty;
                }
            }
        }
        // leaf phase
        for (;;) {
            bool want = active && t.leaf != kEmpty;
            if (!__any_sync(0xffffffffu, want)) break;
            if (COUNT) {
                if ((threadIdx.x & 31) == 0) cnt->leafWarpSteps++;
                if (want) cnt->leafSteps++;
            }
            if (want) {
                int e = travLeafStep<BLOCK, ANY, COUNT, SMEM, MOTION>(t, *sv, st, cnt, nm);
                if (e) { err |= e; t.sp = 0; t.leaf = kEmpty; t.next = kEmpty; }
            }
        }
        if (active && t.sp == 0 && t.leaf == kEmpty && t.next == kEmpty) {
            src.store(idx, travHit(t), *sv);
            active = false;
        }
    }
    return err;
}

}  // namespace gnd
