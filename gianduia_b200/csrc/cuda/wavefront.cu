// Wavefront path tracer: the reference's `path` (path.cpp:12-181) and `volpath`
// (volPath.cpp:15-298) Li loops split into per-bounce kernels over a pool of path slots.
//
//   raygen  : camera sample per (pass, pixel) work item (integrator.h:92-125)
//   extend  : closest hit for every active path (two-level BVH4 traversal)
//   shade   : one bounce (medium sampling, emission with MIS, next-event estimation,
//             BSDF / phase sampling, Russian roulette); appends a shadow query and the
//             path to the next active list or to the done list
//   shadow  : occlusion (path) or transmittance through media and null surfaces
//             (volpath, volPath.cpp:261-291); adds the NEE contribution
//   retire  : film splat of finished paths (film.h:26-69) and, in batched mode, refill
//             of the freed slot with the next work item
//
// Every path draws its random numbers from its own PCG32 stream keyed exactly like the
// reference (pixel + pass * W * H), in one fixed draw order, so a path's result does
// not depend on which slot, pass or launch carries it. The film is accumulated in
// 2^-24 fixed point with integer atomics: sums are independent of completion order.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstring>

#include "raysort.cuh"
#include "shading.cuh"
#include "textures.cuh"
#include "traverse.cuh"
#include "wavefront.h"

namespace gnd {

constexpr int kBlock = 128;
constexpr float kFixScale = 16777216.0f;   // 2^24
constexpr float kFixMax = 1e11f;           // per-sample clamp before the fixed-point conversion
// Shade classes: integrator (0 path, 1 volpath) x class. Classes 0..3 follow the
// material type (matte, plastic, conductor, glass); class 4 holds misses and null-BSDF
// surfaces and is shaded by the kernel built with every lobe; class 5 (volpath only)
// holds paths inside a medium, whose medium sampling runs first in its own kernel.
constexpr int kMatClasses = 5;                       // surface classes 0..4
constexpr int kMediumClass = 5;
constexpr int kClassesPerInt = 6;
constexpr int kShadeClasses = 2 * kClassesPerInt;
constexpr uint32_t kFlagMediumDone = 2u;             // PathState::flags: medium sampled this bounce
static_assert(kQClass0 + kShadeClasses <= kQCount, "class counters exceed the counter block");


// ---------------------------------------------------------------- queue helpers
__device__ __forceinline__ uint32_t warpAppend(uint32_t* counter, bool pred) {
    uint32_t active = __activemask();
    uint32_t mask = __ballot_sync(active, pred);
    if (!pred) return 0xFFFFFFFFu;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// Block-aggregated queue operations for the short kernels whose appends and work grabs
// all reach the same counters at once (kRetire, kClassify): one atomic per counter per
// block of kAggBlock threads instead of one per warp. Every thread of the block calls
// them (block-uniform control flow); each starts with a barrier, so the shared scratch
// of the previous call is free.
constexpr int kAggBlock = 512;
constexpr int kAggWarps = kAggBlock / 32;

// Warp counts of `pred` -> this thread's offset among the block's predicated threads
// (warps in order, lanes in order) and the block total.
__device__ __forceinline__ uint32_t blockRank(uint32_t mask, uint32_t* sCnt, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sCnt[warp] = (uint32_t)__popc(mask);
    __syncthreads();
    uint32_t off = 0, tot = 0;
#pragma unroll
    for (uint32_t w = 0; w < (uint32_t)kAggWarps; ++w) {
        const uint32_t c = sCnt[w];
        off += w < warp ? c : 0u;
        tot += c;
    }
    total = tot;
    return off + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// Two appends with one atomic: threads with `a` take consecutive entries of the counter
// in the low half of `pair`, threads with `b` of the one in the high half.
struct AggScratch {
    uint32_t a[kAggWarps], b[kAggWarps];
    unsigned long long base;
};
__device__ __forceinline__ void blockAppend2(unsigned long long* pair, bool a, bool b, uint32_t& ia, uint32_t& ib,
                                             AggScratch& sc) {
    const uint32_t ma = __ballot_sync(0xffffffffu, a), mb = __ballot_sync(0xffffffffu, b);
    uint32_t ta, tb;
    const uint32_t ra = blockRank(ma, sc.a, ta);
    const uint32_t rb = blockRank(mb, sc.b, tb);
    if (threadIdx.x == 0) sc.base = (ta | tb) ? atomicAdd(pair, (unsigned long long)ta | ((unsigned long long)tb << 32)) : 0ull;
    __syncthreads();
    const unsigned long long base = sc.base;
    ia = (uint32_t)base + ra;
    ib = (uint32_t)(base >> 32) + rb;
}

struct KParams {
    const JobDev* jobs;
    PathState* paths;
    HitRec* hits;
    uint32_t* listIn;
    uint32_t* listOut;
    ShadowRec* shadow;
    uint32_t* done;
    uint32_t* cnt;                 // queue counters (kQIn ...)
    unsigned long long* totals;    // [0] extend rays, [1] shadow queries, [2] paths retired
    JobCtl* ctl;                   // per job: next work item, retired samples
    const uint32_t* active;        // active job indices (count in cnt[kQActive])
    uint32_t* freeIn;              // idle slots waiting for work
    uint32_t* freeOut;
    uint32_t* errWord;
    uint32_t* classLists;          // shade-class lists, `capacity` entries each
    float* slotTime;               // per path slot: the path's shutter time (ray.h: time)
    const uint32_t* extList;       // the active list in the order kExtend takes it (listIn,
                                   // or its copy reordered by ray key)
    uint32_t* rayKeys;             // ray reordering: key per active-list entry,
    uint32_t* rayBins;             // key histogram / bin offsets (kRayBins entries)
    uint32_t* raySorted;           // the reordered list
    const uint32_t* shadowOrder;   // order in which kShadowPath takes the shadow records, or null
    uint32_t leafBatch;            // closest-hit traversal: lanes holding a leaf that end the node phase (1..32)
    uint32_t shadowLeafBatch;      // the same for the shadow queries
    uint32_t capacity;
    uint32_t fifo;                 // 1: grabs walk the active list from its first job
};

// ---------------------------------------------------------------- surface interaction
struct SurfInt {
    V3 p, n, dpdu;
    V2 uv;
};

__device__ __forceinline__ V3 fallbackDpdu(V3 n) {
    if (fabsf(n.x) > fabsf(n.y)) return divs(v3(-n.z, 0.0f, n.x), sqrtf(n.x * n.x + n.z * n.z));
    return divs(v3(0.0f, n.z, -n.y), sqrtf(n.y * n.y + n.z * n.z));
}

__device__ __forceinline__ void sphereUV(SurfInt& si) {
    float phi = atan2f(si.n.x, si.n.z);
    if (phi < 0.0f) phi = (float)((double)phi + 2.0 * kPiD);
    float u = phi * kInv2Pi;
    float theta = acosf(clampf(si.n.y, -1.0f, 1.0f));
    si.uv = V2{u, theta * kInvPi};
    si.dpdu = v3((float)((double)(si.p.z * 2.0f) * kPiD), 0.0f, (float)((double)(-si.p.x * 2.0f) * kPiD));
}

// Object-space interaction of a mesh triangle (mesh.cpp:328-390).
__device__ __forceinline__ SurfInt meshInteraction(const SceneView& s, uint32_t slot, float u, float v) {
    SurfInt si;
    float4 a = ldg4(&s.tris[slot].v0x), b = ldg4(&s.tris[slot].v1x), c = ldg4(&s.tris[slot].v2x);
    V3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
    const TriAttr* at = s.attrs + slot;
    float4 A0 = ldg4(&at->n0x), A1 = ldg4(&at->n1y), A2 = ldg4(&at->n2z), A3 = ldg4(&at->v1_);
    uint32_t flags = (uint32_t)A3.w;
    float w = 1.0f - u - v;
    si.p = (p0 * w + p1 * u) + p2 * v;
    if (flags & 1u) {
        V3 n0 = v3(A0.x, A0.y, A0.z), n1 = v3(A0.w, A1.x, A1.y), n2 = v3(A1.z, A1.w, A2.x);
        si.n = normalize((n0 * w + n1 * u) + n2 * v);
    } else {
        si.n = normalize(cross(p1 - p0, p2 - p0));
    }
    if (flags & 2u) {
        V2 uv0{A2.y, A2.z}, uv1{A2.w, A3.x}, uv2{A3.y, A3.z};
        si.uv = V2{(uv0.x * w + uv1.x * u) + uv2.x * v, (uv0.y * w + uv1.y * u) + uv2.y * v};
        V3 dp1 = p1 - p0, dp2 = p2 - p0;
        V2 duv1{uv1.x - uv0.x, uv1.y - uv0.y}, duv2{uv2.x - uv0.x, uv2.y - uv0.y};
        float det = duv1.x * duv2.y - duv1.y * duv2.x;
        V3 dpdu;
        if (fabsf(det) < 1e-8f) dpdu = fallbackDpdu(si.n);
        else dpdu = (dp1 * duv2.y - dp2 * duv1.y) * (1.0f / det);
        si.dpdu = normalize(dpdu - si.n * dot(si.n, dpdu));
    } else {
        si.uv = V2{u, v};
        si.dpdu = normalize(fallbackDpdu(si.n));
    }
    return si;
}

// Primitive::fillInteraction (primitive.cpp:61-72) for the closest hit of world ray (o, d),
// with the instance's transforms o2w / w2o.
__device__ __forceinline__ SurfInt surfaceInteractionWith(const SceneView& s, const HitRec& h, V3 o, V3 d, const Xf34& o2w,
                                                          const Xf34& w2o) {
    const InstTrav& it = s.instT[h.inst];
    const InstShade& is = s.instS[h.inst];
    const uint32_t kind = it.kind & ~kInstAnimated;
    SurfInt si;
    if (kind == kShapeMesh) {
        si = meshInteraction(s, h.slot, h.u, h.v);
    } else {
        V3 lo = xfPoint(w2o, o), ld = xfVector(w2o, d);
        si.p = lo + ld * h.t;
        if (kind == kShapeSphere) {     // sphere.cpp:41-55
            si.n = normalize(si.p);
            sphereUV(si);
        } else {                        // cube.cpp:48-81
            V3 ex = v3(is.ext[0], is.ext[1], is.ext[2]);
            V3 dmin = si.p - (-ex), dmax = ex - si.p;
            float md = 3.402823466e38f;
            int axis = 0;
            float sign = 1.0f;
            for (int i = 0; i < 3; ++i) {
                if (comp(dmin, i) < md) { md = comp(dmin, i); axis = i; sign = -1.0f; }
                if (comp(dmax, i) < md) { md = comp(dmax, i); axis = i; sign = 1.0f; }
            }
            si.n = v3s(0.0f);
            if (axis == 0) si.n.x = sign; else if (axis == 1) si.n.y = sign; else si.n.z = sign;
            if (axis == 0) {
                si.uv = V2{(si.p.z - (-ex.z)) / (2.0f * ex.z), (si.p.y - (-ex.y)) / (2.0f * ex.y)};
                si.dpdu = v3(0.0f, 0.0f, 2.0f * ex.z * sign);
            } else if (axis == 1) {
                si.uv = V2{(si.p.x - (-ex.x)) / (2.0f * ex.x), (si.p.z - (-ex.z)) / (2.0f * ex.z)};
                si.dpdu = v3(2.0f * ex.x * sign, 0.0f, 0.0f);
            } else {
                si.uv = V2{(si.p.x - (-ex.x)) / (2.0f * ex.x), (si.p.y - (-ex.y)) / (2.0f * ex.y)};
                si.dpdu = v3(2.0f * ex.x * sign, 0.0f, 0.0f);
            }
        }
    }
    si.p = xfPoint(o2w, si.p);
    si.n = normalize(xfNormal(w2o, si.n));
    si.dpdu = normalize(xfVector(o2w, si.dpdu));
    return si;
}

// The same for an animated instance at shutter time `time` (Primitive::getToWorld,
// primitive.cpp:62 and 82-84). Out of line, so that static scenes keep their registers.
__device__ __noinline__ SurfInt surfaceInteractionMoving(const SceneView& s, const HitRec& h, V3 o, V3 d, float time) {
    Xf34 o2w, w2o;
    motionAt(s.motion[h.inst], s.instS[h.inst].o2w, s.instT[h.inst].w2o, time, o2w, w2o);
    return surfaceInteractionWith(s, h, o, d, o2w, w2o);
}

__device__ __forceinline__ SurfInt surfaceInteraction(const SceneView& s, const HitRec& h, V3 o, V3 d, float time) {
    if (s.instT[h.inst].kind & kInstAnimated) return surfaceInteractionMoving(s, h, o, d, time);
    return surfaceInteractionWith(s, h, o, d, s.instS[h.inst].o2w, s.instT[h.inst].w2o);
}

// ---------------------------------------------------------------- area emitters (area.cpp)
struct LightSample {
    V3 p, n;
    V2 uv;
    V3 Li;          // eval / pdf
    float pdf;      // solid angle; left 0 on the early return
    V3 sd;          // shadow direction
    float stmax;    // shadow tMax
    float stime;    // shadow ray time (ref.time; a point light's leaves it 0, pointlight.cpp:29)
    bool delta;     // point / spot / directional: no MIS against the BSDF (emitter.h)
};

// Shape::sampleSurface in object space; returns the area pdf.
__device__ __forceinline__ float sampleShape(const SceneView& s, int inst, V2 u, V3& p, V3& n, V2& uv) {
    const InstTrav& it = s.instT[inst];
    const InstShade& is = s.instS[inst];
    const uint32_t kind = it.kind & ~kInstAnimated;
    if (kind == kShapeMesh) {                            // mesh.cpp:396-434
        const MeshRec mr = s.meshes[is.meshId];
        if (mr.totalArea == 0.0f) return 0.0f;
        const float* cdf = s.cdf + mr.cdfOffset;
        uint32_t size = mr.numTris + 1;
        uint32_t lo = 0, hi = size;                      // std::lower_bound
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (cdf[mid] < u.x) lo = mid + 1; else hi = mid;
        }
        uint32_t tri = (lo < 1u ? 1u : (lo > size - 1 ? size - 1 : lo)) - 1;
        float pdfTri = cdf[tri + 1] - cdf[tri];
        float rx = clampf((u.x - cdf[tri]) / pdfTri, 0.0f, 1.0f);
        float sq = sqrtf(rx);
        float bu = 1.0f - sq;
        float bv = u.y * sq;
        uint32_t slot = s.origToLeaf[mr.origToLeaf + tri];
        SurfInt si = meshInteraction(s, slot, bu, bv);
        p = si.p;
        n = si.n;
        uv = si.uv;
        const TriAttr* at = s.attrs + slot;
        if (!(((uint32_t)at->flags) & 2u)) uv = V2{0.f, 0.f};
        return 1.0f / mr.totalArea;
    }
    if (kind == kShapeSphere) {                          // sphere.cpp:64-81
        float r = is.radius;
        V3 res = squareToUniformSphere(u);
        SurfInt si;
        si.p = res * r;
        si.n = normalize(si.p);
        sphereUV(si);
        p = si.p; n = si.n; uv = si.uv;
        return kInv4Pi / (r * r);
    }
    // cube.cpp:83-146
    V3 ex = v3(is.ext[0], is.ext[1], is.ext[2]);
    float aX = 4.0f * ex.y * ex.z, aY = 4.0f * ex.x * ex.z, aZ = 4.0f * ex.x * ex.y;
    float total = 2.0f * (aX + aY + aZ);
    float fp[6] = {aX / total, aX / total, aY / total, aY / total, aZ / total, aZ / total};
    float ux = u.x;
    int face = 0;
    float c = 0.0f;
    for (int i = 0; i < 6; ++i) {
        c += fp[i];
        if (ux < c || i == 5) { face = i; float prev = c - fp[i]; ux = (ux - prev) / fp[i]; break; }
    }
    float sign = (face % 2 == 0) ? 1.0f : -1.0f;
    if (face < 2) {
        p = v3(ex.x * sign, -ex.y + ux * (2.0f * ex.y), -ex.z + u.y * (2.0f * ex.z));
        n = v3(sign, 0.0f, 0.0f);
        uv = V2{(p.z - (-ex.z)) / (2.0f * ex.z), (p.y - (-ex.y)) / (2.0f * ex.y)};
    } else if (face < 4) {
        p = v3(-ex.x + ux * (2.0f * ex.x), ex.y * sign, -ex.z + u.y * (2.0f * ex.z));
        n = v3(0.0f, sign, 0.0f);
        uv = V2{(p.x - (-ex.x)) / (2.0f * ex.x), (p.z - (-ex.z)) / (2.0f * ex.z)};
    } else {
        p = v3(-ex.x + ux * (2.0f * ex.x), -ex.y + u.y * (2.0f * ex.y), ex.z * sign);
        n = v3(0.0f, 0.0f, sign);
        uv = V2{(p.x - (-ex.x)) / (2.0f * ex.x), (p.y - (-ex.y)) / (2.0f * ex.y)};
    }
    return 1.0f / total;
}

__device__ __forceinline__ float shapeAreaPdf(const SceneView& s, int inst) {
    const InstTrav& it = s.instT[inst];
    const InstShade& is = s.instS[inst];
    const uint32_t kind = it.kind & ~kInstAnimated;
    if (kind == kShapeMesh) {
        float ta = s.meshes[is.meshId].totalArea;
        return ta > 0.0f ? 1.0f / ta : 0.0f;
    }
    if (kind == kShapeSphere) return kInv4Pi / (is.radius * is.radius);
    V3 d = v3(is.ext[0], is.ext[1], is.ext[2]) - (-v3(is.ext[0], is.ext[1], is.ext[2]));
    return 1.0f / (2.0f * (d.x * d.y + d.x * d.z + d.y * d.z));
}

// AreaLight::eval (area.cpp:45-49)
__device__ __forceinline__ V3 emitterEval(const Emitter& e, V3 n, V2 uv, V3 w) {
    if (dot(n, w) > 0.0f) return evalTex(e.radiance, uv);
    return v3s(0.0f);
}
// A color slot at a surface point: texture trees in the EXT variants, constant and
// checkerboard slots everywhere.
template <bool EXT>
__device__ __forceinline__ V3 evalColor(const SceneView& s, const ColorTex& t, V3 p, V3 n, V3 dpdu, V2 uv) {
    if (EXT && t.kind == kTexNode) return evalTexTree(s, t.node, p, n, dpdu, uv);
    return evalTex(t, uv);
}
// Material::applyNormalOrBump (material.h:71-117): the normal map replaces n by its
// (x, y, z) in the (dpdu, n x dpdu, n) frame; the bump map tilts dpdu and dpdv by forward
// differences of the height (steps of 0.001 in p along dpdu / dpdv and in u / v). dpdu is
// re-orthogonalised against the new n. Everything after it (emission, light pdf, next
// event cosine, BSDF frame, medium choice) sees the new frame, as in the reference.
__device__ __noinline__ void applyNormalOrBump(const SceneView& s, const Material& m, SurfInt& si) {
    if (m.normalTex) {
        const V3 nm = evalTexTree(s, m.normalTex - 1, si.p, si.n, si.dpdu, si.uv);
        const V3 dpdv = normalize(cross(si.n, si.dpdu));
        const V3 pn = (si.dpdu * nm.x + dpdv * nm.y) + si.n * nm.z;
        si.n = normalize(pn);
        si.dpdu = normalize(si.dpdu - si.n * dot(si.n, si.dpdu));
    } else if (m.bumpTex) {
        const V3 dpdu = si.dpdu;
        const V3 dpdv = normalize(cross(si.n, dpdu));
        const float du = 0.001f, dv = 0.001f;
        const float hBase = evalTexTree(s, m.bumpTex - 1, si.p, si.n, si.dpdu, si.uv).x;
        const float hDu = evalTexTree(s, m.bumpTex - 1, si.p + dpdu * du, si.n, si.dpdu, V2{si.uv.x + du, si.uv.y}).x;
        const float hDv = evalTexTree(s, m.bumpTex - 1, si.p + dpdv * dv, si.n, si.dpdu, V2{si.uv.x, si.uv.y + dv}).x;
        float dhdu = (hDu - hBase) / du;
        float dhdv = (hDv - hBase) / dv;
        dhdu *= m.bumpScale;
        dhdv *= m.bumpScale;
        const V3 ndu = dpdu + si.n * dhdu;
        const V3 ndv = dpdv + si.n * dhdv;
        si.n = normalize(cross(ndu, ndv));
        si.dpdu = normalize(ndu - si.n * dot(si.n, ndu));
    }
}

// Material slots at a surface point; EXT: with texture trees.
template <bool EXT>
struct SlotTexAt {
    static constexpr bool kTrees = EXT;
    const SceneView& s;
    const SurfInt& si;
    __device__ __forceinline__ V3 operator()(const ColorTex& t) const { return evalColor<EXT>(s, t, si.p, si.n, si.dpdu, si.uv); }
    __device__ __forceinline__ V3 node(uint32_t root) const { return evalTexTree(s, root, si.p, si.n, si.dpdu, si.uv); }
};
template <bool EXT>
__device__ __forceinline__ V3 emitterEvalAt(const SceneView& s, const Emitter& e, V3 p, V3 n, V3 dpdu, V2 uv, V3 w) {
    if (dot(n, w) > 0.0f) return evalColor<EXT>(s, e.radiance, p, n, dpdu, uv);
    return v3s(0.0f);
}

// ---------------------------------------------------------------- environment map
// SphericalCoordinates (constants.h:80-85): (theta from +z, phi in [0, 2 pi))
__device__ __forceinline__ V2 sphericalCoordinates(V3 w) {
    const float z = w.z < -1.0f ? -1.0f : (1.0f < w.z ? 1.0f : w.z);   // std::clamp
    V2 r{acosf(z), atan2f(w.y, w.x)};
    if (r.y < 0.0f) r.y += 2.0f * kPi;
    return r;
}
// (u, v) of a direction in the lat-long image: phi / 2 pi and theta / pi, evaluated in
// double as the reference's float * M_1_PI expressions are (environment.cpp:31-35)
__device__ __forceinline__ V2 envUV(V2 sph) {
    constexpr double kInvPiD = 0.318309886183790671538;
    return V2{(float)((double)sph.y * kInvPiD * 0.5), (float)((double)sph.x * kInvPiD)};
}
// Film::getPixelBilinear (film.cpp:126-151): azimuth wraps, polar angle clamps
__device__ __forceinline__ V3 envTexel(const EnvView& e, int x, int y) {
    const float* t = e.texels + 3 * ((size_t)y * e.width + x);
    return v3(__ldg(t), __ldg(t + 1), __ldg(t + 2));
}
__device__ __forceinline__ V3 envBilinear(const EnvView& e, float u, float v) {
    const float x = u * (float)e.width - 0.5f, y = v * (float)e.height - 0.5f;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const float dx = x - (float)x0, dy = y - (float)y0;
    const int px0 = (x0 % e.width + e.width) % e.width;
    const int px1 = (px0 + 1) % e.width;
    const int py0 = min(max(y0, 0), e.height - 1), py1 = min(max(y0 + 1, 0), e.height - 1);
    const V3 c0 = envTexel(e, px0, py0) * (1.0f - dx) + envTexel(e, px1, py0) * dx;
    const V3 c1 = envTexel(e, px0, py1) * (1.0f - dx) + envTexel(e, px1, py1) * dx;
    return c0 * (1.0f - dy) + c1 * dy;
}
// EnvironmentMap::eval (environment.cpp:29-37)
__device__ __forceinline__ V3 envEval(const EnvView& e, V3 w) {
    const V2 uv = envUV(sphericalCoordinates(w));
    return envBilinear(e, uv.x, uv.y) * e.strength;
}
// Distribution1D::SampleContinuous (distribution.cpp:21-35)
__device__ __forceinline__ float dist1DSample(const float* func, const float* cdf, int n, float funcInt, float u, float& pdf,
                                              int& off) {
    int lo = 0, hi = n + 1;   // std::upper_bound over cdf[0..n]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (!(u < __ldg(cdf + mid))) lo = mid + 1;
        else hi = mid;
    }
    off = min(max(lo - 1, 0), n - 1);
    float du = u - __ldg(cdf + off);
    if ((__ldg(cdf + off + 1) - __ldg(cdf + off)) > 0.0f) du /= (__ldg(cdf + off + 1) - __ldg(cdf + off));
    pdf = (funcInt > 0.0f) ? __ldg(func + off) / funcInt : 0.0f;
    return ((float)off + du) / (float)n;
}
// EnvironmentMap::pdf (environment.cpp:75-89) for the unit direction wi from the
// reference point; Distribution2D::Pdf (distribution.cpp:76-80)
__device__ __forceinline__ float envPdf(const EnvView& e, V3 wi) {
    const V2 sph = sphericalCoordinates(wi);
    const float sinTheta = sinf(sph.x);
    if (sinTheta <= 0.0f) return 0.0f;
    const V2 uv = envUV(sph);
    const int iu = min(max((int)(uv.x * (float)e.width), 0), e.width - 1);
    const int iv = min(max((int)(uv.y * (float)e.height), 0), e.height - 1);
    const float mapPdf = __ldg(e.condFunc + (size_t)iv * e.width + iu) / e.margInt;
    return (float)((double)mapPdf / (2.0 * kPiD * kPiD * (double)sinTheta));
}
// EnvironmentMap::sample (environment.cpp:39-73)
__device__ __noinline__ void envSample(const EnvView& e, V3 ref, V2 u, LightSample& ls, float time) {
    ls.pdf = 0.0f;
    ls.Li = v3s(0.0f);
    ls.delta = false;
    ls.stime = time;
    float pdf0, pdf1;
    int v, off0;
    const float d1 = dist1DSample(e.margFunc, e.margCdf, e.height, e.margInt, u.y, pdf1, v);
    const float d0 = dist1DSample(e.condFunc + (size_t)v * e.width, e.condCdf + (size_t)v * (e.width + 1), e.width,
                                  __ldg(e.condInt + v), u.x, pdf0, off0);
    const float mapPdf = pdf0 * pdf1;
    if (mapPdf == 0.0f) return;
    const float theta = (float)((double)d1 * kPiD);
    const float phi = (float)((double)(d0 * 2.0f) * kPiD);
    const float cosTheta = cosf(theta), sinT = sinf(theta), cosPhi = cosf(phi), sinPhi = sinf(phi);
    const V3 wi = v3(sinT * cosPhi, sinT * sinPhi, cosTheta);   // SphericalDirection (constants.h:87-98)
    ls.p = ref + wi * 1e5f;
    ls.n = -wi;
    ls.uv = V2{0.0f, 0.0f};
    ls.sd = wi;
    ls.stmax = INFINITY;
    const float sinTheta = sinf(theta);
    if (sinTheta <= 0.0f) return;
    ls.pdf = (float)((double)mapPdf / (2.0 * kPiD * kPiD * (double)sinTheta));
    ls.Li = cdiv(envEval(e, wi), ls.pdf);
}

// ---------------------------------------------------------------- delta emitters
// PointLight::sample (pointlight.cpp:18-31), SpotLight::sample (spotlight.cpp:30-60),
// DirectionalLight::sample (directional.cpp:18-34)
__device__ __noinline__ void deltaSample(const Emitter& e, V3 ref, LightSample& ls, float time) {
    ls.delta = true;
    ls.pdf = 1.0f;
    ls.stime = e.type == kEmitPoint ? 0.0f : time;   // pointlight.cpp:29 uses info.time, never set
    ls.n = v3s(0.0f);
    ls.uv = V2{0.0f, 0.0f};
    const V3 col = v3(e.color[0], e.color[1], e.color[2]);
    if (e.type == kEmitDirectional) {
        const V3 wi = v3(e.dir[0], e.dir[1], e.dir[2]);
        ls.p = ref + wi * 1e5f;
        ls.sd = wi;
        ls.stmax = FLT_MAX;
        ls.Li = col;
        return;
    }
    const V3 pos = v3(e.pos[0], e.pos[1], e.pos[2]);
    const V3 I = col * kInv4Pi;
    ls.p = pos;
    if (e.type == kEmitPoint) {
        const float squaredDist = lengthSq(pos - ref);
        ls.sd = normalize(pos - ref);
        ls.stmax = length(pos - ref) - kEpsilon;
        ls.Li = cdiv(I, squaredDist);
        return;
    }
    const V3 wi = normalize(pos - ref);
    const float dist = length(pos - ref);
    const float squaredDist = dist * dist;
    ls.sd = wi;
    ls.stmax = dist - kEpsilon;
    const float cosTheta = dot(-wi, v3(e.dir[0], e.dir[1], e.dir[2]));
    if (cosTheta <= e.cosTotal) {
        ls.Li = v3s(0.0f);
        return;
    }
    float falloff = 1.0f;
    if (cosTheta < e.cosFalloff) {
        const float t = (cosTheta - e.cosTotal) / (e.cosFalloff - e.cosTotal);
        falloff = (t * t) * (3.0f - 2.0f * t);
    }
    ls.Li = cdiv(I * falloff, squaredDist);
}

// Emitter::sample for emitter ei of the scene's list: area lights below (area.cpp:51-88),
// the delta lights and the environment above
// `time` is the reference point's time (ref.time): the path's for surface next-event
// estimation, 0 for a volume scattering point (volPath.cpp:61-62 builds a fresh reference)
__device__ __forceinline__ void areaSample(const SceneView& s, const Emitter& e, V3 ref, V2 u, LightSample& ls, float time);
template <bool EXT>
__device__ __forceinline__ void areaSampleWith(const SceneView& s, const Emitter& e, V3 ref, V2 u, LightSample& ls, float time,
                                               const Xf34& o2w, const Xf34& w2o);
__device__ __forceinline__ void emitterSample(const SceneView& s, int ei, V3 ref, V2 u, LightSample& ls, float time) {
    const Emitter e = s.emitters[ei];
    if (e.type == kEmitArea) areaSample(s, e, ref, u, ls, time);
    else if (e.type == kEmitEnv) envSample(s.env, ref, u, ls, time);
    else deltaSample(e, ref, ls, time);
}
template <bool EXT>
__device__ __forceinline__ void emitterSampleT(const SceneView& s, int ei, V3 ref, V2 u, LightSample& ls, float time) {
    if (EXT) {
        emitterSample(s, ei, ref, u, ls, time);
        return;
    }
    const Emitter e = s.emitters[ei];
    areaSampleWith<false>(s, e, ref, u, ls, time, s.instS[e.instance].o2w, s.instT[e.instance].w2o);
}

// Environment light seen by an escaping ray, weighted against the previous bounce's pdf
// (path.cpp:42-55, volPath.cpp:124-141; the reference evaluates the environment's pdf
// from the origin towards o + 1e5 d)
__device__ __noinline__ V3 envMissRadiance(const SceneView& s, V3 o, V3 d, V3 tp, bool specular, float pdfPrev, float nL) {
    if (s.env.emitter < 0) return v3s(0.0f);
    const V3 Le = envEval(s.env, d);
    if (isBlack(Le)) return v3s(0.0f);
    float w = 1.0f;
    if (!specular) {
        const V3 p = o + d * 1e5f;
        const float ep = envPdf(s.env, normalize(p - v3s(0.0f)));
        const float pEnv = ep * (1.0f / nL);
        w = powerHeuristic(pdfPrev, pEnv);
    }
    return (tp * Le) * w;
}

// AreaLight::sample (area.cpp:51-88); the sampled point carries p, n and uv (no dpdu)
template <bool EXT>
__device__ __forceinline__ void areaSampleWith(const SceneView& s, const Emitter& e, V3 ref, V2 u, LightSample& ls, float time,
                                               const Xf34& o2w, const Xf34& w2o) {
    ls.delta = false;
    ls.stime = time;
    V3 lp, ln;
    V2 luv;
    float areaPdf = sampleShape(s, e.instance, u, lp, ln, luv);
    ls.p = xfPoint(o2w, lp);
    ls.n = normalize(xfNormal(w2o, ln));
    ls.uv = luv;
    Frame fr = frameFromNormal(ln);
    V3 t1 = xfVector(o2w, fr.x), t2 = xfVector(o2w, fr.y);
    float areaScale = length(cross(t1, t2));
    if (areaScale > 0.0f) areaPdf /= areaScale;
    ls.sd = normalize(ls.p - ref);
    ls.stmax = length(ls.p - ref) - kEpsilon;
    float dist = lengthSq(ref - ls.p);
    float cosTheta = dot(ls.n, -ls.sd);
    ls.pdf = 0.0f;
    ls.Li = v3s(0.0f);
    if (areaPdf <= kEpsilon || cosTheta <= kEpsilon) return;
    ls.pdf = areaPdf * dist / cosTheta;
    ls.Li = cdiv(emitterEvalAt<EXT>(s, e, ls.p, ls.n, v3s(0.0f), ls.uv, normalize(ref - ls.p)), ls.pdf);
}

// An animated area light at the reference point's time (m_primitive->getToWorld(ref.time),
// area.cpp:54); out of line like surfaceInteractionMoving.
__device__ __noinline__ void areaSampleMoving(const SceneView& s, const Emitter& e, V3 ref, V2 u, LightSample& ls, float time) {
    Xf34 o2w, w2o;
    motionAt(s.motion[e.instance], s.instS[e.instance].o2w, s.instT[e.instance].w2o, time, o2w, w2o);
    areaSampleWith<true>(s, e, ref, u, ls, time, o2w, w2o);
}

__device__ __forceinline__ void areaSample(const SceneView& s, const Emitter& e, V3 ref, V2 u, LightSample& ls, float time) {
    if (s.instT[e.instance].kind & kInstAnimated) areaSampleMoving(s, e, ref, u, ls, time);
    else areaSampleWith<true>(s, e, ref, u, ls, time, s.instS[e.instance].o2w, s.instT[e.instance].w2o);
}

// Emitter sampling in a kernel variant: without EXT every emitter is a static area light.
template <bool EXT>
__device__ __forceinline__ void emitterSampleT(const SceneView& s, int ei, V3 ref, V2 u, LightSample& ls, float time);

// AreaLight::pdf (area.cpp:90-119)
__device__ __forceinline__ float emitterPdf(const SceneView& s, int ei, V3 ref, V3 p, V3 n) {
    const Emitter e = s.emitters[ei];
    const InstShade& is = s.instS[e.instance];
    float areaPdf = shapeAreaPdf(s, e.instance);
    V3 ln = xfNormal(is.o2w, n);   // toLocal.normal: transpose(mat3(objectToWorld)) * n
    Frame fr = frameFromNormal(ln);
    V3 t1 = xfVector(is.o2w, fr.x), t2 = xfVector(is.o2w, fr.y);
    float areaScale = length(cross(t1, t2));
    if (areaScale > 0.0f) areaPdf /= areaScale;
    float dist = lengthSq(ref - p);
    V3 wi = normalize(p - ref);
    float cosTheta = dot(n, -wi);
    if (areaPdf <= kEpsilon || cosTheta <= kEpsilon) return 0.0f;
    return areaPdf * dist / cosTheta;
}

// scene.h:28-34
__device__ __forceinline__ int pickEmitter(int n, float rnd) {
    int idx = (int)floorf((float)n * rnd);
    return idx < n - 1 ? idx : n - 1;
}

// volPath.cpp:293-298
__device__ __forceinline__ int nextMedium(V3 wo, V3 wi, int cur, V3 n, int mIn, int mOut) {
    if (dot(wi, n) > 0.0f) return dot(wo, n) > 0.0f ? cur : mOut;
    return dot(wo, n) > 0.0f ? mIn : cur;
}

// ---------------------------------------------------------------- path state helpers
__device__ __forceinline__ void storeRng(PathState& ps, const Rng& r) {
    ps.rngLo = (uint32_t)r.state;
    ps.rngHi = (uint32_t)(r.state >> 32);
}
__device__ __forceinline__ Rng loadRng(const PathState& ps) {
    return Rng{((uint64_t)ps.rngHi << 32) | ps.rngLo};
}

// ---------------------------------------------------------------- camera
// Colour channel of a camera sample (integrator.h:103-121): -1 without chromatic
// aberration (thinLens.cpp:97-99), else 0/1/2 from the sample's channel number, with the
// wavelength offset +1/0/-1 the lens equations scale by.
__device__ __forceinline__ int cameraChannel(const Camera& cam, float chRnd, float& lambda) {
    lambda = 0.0f;
    if (cam.kind != kCamThinLens || (cam.caLateral == 0.0f && cam.caAxial == 0.0f)) return -1;
    if (chRnd < 0.333333f) { lambda = 1.0f; return 0; }
    if (chRnd < 0.666666f) return 1;
    lambda = -1.0f;
    return 2;
}

// Thin-lens camera ray in camera space (thinLens.cpp:33-91) for the film position (cx, cy)
// in [0,1]^2: barrel distortion, lateral / axial chromatic aberration, depth of field
// through a disk or polygon aperture. Returns the ray weight (cos^4 vignetting or 1).
// The shutter terms only change the sample time, which static transforms ignore.
__device__ __forceinline__ float thinLensRay(const Camera& cam, float cx, float cy, V2 lens, float lambda,
                                             V3& o, V3& dir) {
    const float ndcX = 2.0f * cx - 1.0f, ndcY = 2.0f * cy - 1.0f;
    const float r2 = ndcX * ndcX + ndcY * ndcY;
    const float distortion = 1.0f + cam.k1 * r2;
    const float distX = ndcX * distortion, distY = ndcY * distortion;
    const float scaleMod = cam.scale * (1.0f + cam.caLateral * lambda);
    dir = v3(distX * cam.aspect * scaleMod, distY * scaleMod, -1.0f);
    o = v3s(0.0f);
    if (cam.lensRadius > 0.0f) {
        const V2 pl = cam.blades >= 3 ? squareToUniformPolygon(lens, cam.blades) : squareToUniformDisk(lens);
        const float lx = pl.x * cam.lensRadius, ly = pl.y * cam.lensRadius;
        const float focalDistMod = cam.focalDistance * (1.0f + cam.caAxial * lambda);
        const float ft = focalDistMod / fabsf(dir.z);
        const V3 pFocus = o + dir * ft;
        o = v3(lx, ly, 0.0f);
        dir = pFocus - o;
    }
    dir = normalize(dir);
    if (!cam.vignetting) return 1.0f;
    const float cosTheta = fabsf(dir.z), cos2 = cosTheta * cosTheta;
    return cos2 * cos2;
}

// Camera weighting of a finished sample's radiance (integrator.h:130-135): the thin lens's
// ray weight, then with chromatic aberration only the sample's channel, times 3. `r` is the
// sample's generator right after the film position draw.
__device__ __forceinline__ V3 cameraWeigh(const Camera& cam, V3 L, Rng r, float fx, float fy, int W, int H) {
    const V2 lens = next2D(r);
    float lambda;
    const int ch = cameraChannel(cam, next1D(r), lambda);
    if (cam.vignetting) {
        V3 o, d;
        const float w = thinLensRay(cam, fx / (float)W, 1.0f - fy / (float)H, lens, lambda, o, d);
        L = L * w;
    }
    if (ch == 0) return v3(L.x * 3.0f, 0.0f, 0.0f);
    if (ch == 1) return v3(0.0f, L.y * 3.0f, 0.0f);
    if (ch == 2) return v3(0.0f, 0.0f, L.z * 3.0f);
    return L;
}

// Work item -> camera sample (integrator.h:88-125) in slot `slot`; returns the ray's
// shutter time, which every ray of the path keeps (ray.h: time; primitive.cpp:71).
template <bool EXT>
__device__ __forceinline__ float generatePath(const JobDev& j, uint32_t jobIdx, uint64_t item, PathState& ps) {
    int ww = j.wx1 - j.wx0;
    uint64_t npix = (uint64_t)ww * (uint64_t)(j.wy1 - j.wy0);
    uint32_t pass = (uint32_t)(item / npix) + (uint32_t)j.firstPass;
    uint32_t pix = (uint32_t)(item % npix);
    int x = j.wx0 + (int)(pix % (uint32_t)ww), y = j.wy0 + (int)(pix / (uint32_t)ww);
    uint64_t key = (uint64_t)y * (uint64_t)j.W + (uint64_t)x + (uint64_t)pass * ((uint64_t)j.W * (uint64_t)j.H);
    Rng r = rngSeed(key);
    V2 ps2 = next2D(r);
    float fx = (float)x + ps2.x, fy = (float)y + ps2.y;
    float cx = fx / (float)j.W, cy = 1.0f - fy / (float)j.H;
    const V2 lens = next2D(r);     // lens position
    const float chRnd = next1D(r); // chromatic aberration channel
    float time = next1D(r);        // shutter time
    const Camera& cam = j.view.camera;
    V3 o, d;
    if (EXT && cam.kind == kCamThinLens) {
        float lambda;
        cameraChannel(cam, chRnd, lambda);
        V3 oc, dc;
        thinLensRay(cam, cx, cy, lens, lambda, oc, dc);
        if (cam.rollingShutter) {   // thinLens.cpp:80-85
            const float scanline = 1.0f - cy;
            time = scanline * cam.scanDuration + (time * cam.exposureDuration);
        }
        Xf34 tw = cam.toWorld, unused;
        if (cam.animated) motionAt(cam.motion, cam.toWorld, cam.toWorld, time, tw, unused);
        o = xfPoint(tw, oc);
        d = xfVector(tw, dc);
    } else {
        // perspective.cpp:15-32
        float px = (2.0f * cx - 1.0f) * cam.aspect * cam.scale;
        float py = (2.0f * cy - 1.0f) * cam.scale;
        V3 dir = normalize(v3(px, py, -1.0f));
        if (EXT && cam.animated) {
            Xf34 tw, unused;
            motionAt(cam.motion, cam.toWorld, cam.toWorld, time, tw, unused);
            o = xfPoint(tw, v3s(0.0f));
            d = xfVector(tw, dir);
        } else {
            o = v3(cam.origin[0], cam.origin[1], cam.origin[2]);
            d = xfVector(cam.toWorld, dir);
        }
    }
    ps.ox = o.x; ps.oy = o.y; ps.oz = o.z; ps.pdfPrev = 1.0f;
    ps.dx = d.x; ps.dy = d.y; ps.dz = d.z;
    ps.lastX = o.x; ps.lastY = o.y; ps.lastZ = o.z;
    ps.tpr = ps.tpg = ps.tpb = 1.0f;
    ps.Lr = ps.Lg = ps.Lb = 0.0f;
    storeRng(ps, r);
    ps.pixel = pix;
    ps.pass = pass;
    ps.bounces = 0;
    ps.vsBounces = 0;
    ps.medium = -1;                        // camera rays start in vacuum (ray.h:18)
    ps.flags = 1u | (jobIdx << 8);         // specularBounce = true
    return time;
}

// ---------------------------------------------------------------- kernels
__global__ void kBeginIter(KParams p) {
    uint32_t* cnt = p.cnt;
    cnt[kQOut] = 0;
    cnt[kQShadow] = 0;
    cnt[kQDone] = 0;
    cnt[kQFetchA] = 0;
    cnt[kQFetchB] = 0;
    cnt[kQIter] += 1;   // iteration number: round-robin start of the job grabs
    for (int k = 0; k < kShadeClasses; ++k) cnt[kQClass0 + k] = 0;
    // Whether any active job has work items left to hand out (the hand-out limits change
    // only between launches). Without work the idle slots are carried over unchanged:
    // kRetire copies them to the front of the next free list, reserved here.
    uint32_t work = 0;
    const uint32_t na = cnt[kQActive];
    for (uint32_t t = 0; t < na && !work; ++t) {
        const uint32_t jid = p.active[t];
        if (p.ctl[jid].next < p.jobs[jid].workEnd) work = 1;
    }
    cnt[kQWork] = work;
    cnt[kQFreeOut] = work ? 0u : cnt[kQFree];
}

// Shade class of a path after its extend query (see kMatClasses): volpath paths inside a
// medium go to the medium class, others to their surface's class.
static_assert(kMatIndex == kMatClasses - 1, "the null-BSDF material type is the last surface class");
__device__ __forceinline__ uint32_t surfaceClass(const SceneView& s, int inst) {
    return inst >= 0 ? (uint32_t)__ldg(s.instClass + inst) : (uint32_t)(kMatClasses - 1);   // kMatIndex -> 4
}
__device__ __forceinline__ uint32_t shadeClass(const SceneView& s, bool vol, int medium, int inst) {
    const uint32_t c = (vol && medium >= 0) ? (uint32_t)kMediumClass : surfaceClass(s, inst);
    return (vol ? (uint32_t)kClassesPerInt : 0u) + c;
}
// Class of a path whose bounce ends it unchanged: a path_gpu ray that escapes a scene
// without an environment emitter (path.cpp: the escaped ray adds nothing and the path
// ends). kClassify appends it to the done list directly; the shade kernel would only
// have stored its state back unchanged.
constexpr uint32_t kClassDone = kShadeClasses;

// Closest-hit source/sink over the active list (extend). The store also records the
// path's shade class in the hit record, for kClassify.
struct ExtendSrc {
    const KParams* p;
    uint32_t n;
    uint32_t slot;
    int32_t medium;
    bool vol;
    __device__ uint32_t count() const { return n; }
    __device__ bool load(uint32_t i, TRay& r, const SceneView*& sv, const uint8_t*& nm) {
        slot = p->extList[i];
        const PathState* ps = p->paths + slot;
        float4 a = *reinterpret_cast<const float4*>(&ps->ox);
        float4 b = *reinterpret_cast<const float4*>(&ps->dx);
        uint4 c = *reinterpret_cast<const uint4*>(&ps->bounces);   // bounces, vsBounces, medium, flags
        const JobDev& jd = p->jobs[c.w >> 8];
        medium = (int32_t)c.z;
        vol = jd.integrator == 1;
        r.o = v3(a.x, a.y, a.z);
        r.d = v3(b.x, b.y, b.z);
        r.tmin = kEpsilon;
        r.tmax = INFINITY;
        r.time = p->slotTime[slot];
        sv = &jd.view;
        nm = nullptr;
        return true;
    }
    __device__ void store(uint32_t, const THit& h, const SceneView& sv) {
        HitRec hr;
        hr.t = h.t; hr.u = h.u; hr.v = h.v; hr.inst = h.inst; hr.slot = h.slot;
        hr.pad[0] = (h.inst < 0 && !vol && sv.env.emitter < 0) ? kClassDone : shadeClass(sv, vol, medium, h.inst);
        hr.pad[1] = hr.pad[2] = 0;
        p->hits[slot] = hr;
    }
};

// MOTION: the scene has animated instances (rays carry their shutter time)
// MINB: the blocks per SM the kernel is compiled to fit (8: 64 registers; 9 and 10 trade
// registers, with some spilled, for more resident warps; gnd_tune trav_blocks)
template <bool COUNT, int SMEM, bool SPEC, bool MOTION = false, int MINB = 8>
__global__ void __launch_bounds__(kBlock, MINB) kExtend(KParams p) {
    __shared__ uint32_t stack[SMEM * kBlock];
    const uint32_t n = p.cnt[kQIn];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.totals[0], (unsigned long long)n);
    TraceCounters cnt{0, 0, 0, 0, 0};
    ExtendSrc src{&p, n, 0};
    int err = persistentTrace<kBlock, false, COUNT, SMEM, SPEC, MOTION>(src, p.cnt + kQFetchA, stack, &cnt, p.leafBatch);
    if (COUNT) {
        unsigned long long nn = cnt.nodes, nt = cnt.tris, nw = cnt.nodeWarpSteps, ls = cnt.leafSteps, lw = cnt.leafWarpSteps;
        for (int o = 16; o > 0; o >>= 1) {
            nn += __shfl_down_sync(0xffffffffu, nn, o);
            nt += __shfl_down_sync(0xffffffffu, nt, o);
            nw += __shfl_down_sync(0xffffffffu, nw, o);
            ls += __shfl_down_sync(0xffffffffu, ls, o);
            lw += __shfl_down_sync(0xffffffffu, lw, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&p.totals[3], nn);
            atomicAdd(&p.totals[5], nw);
            atomicAdd(&p.totals[6], ls);
            atomicAdd(&p.totals[7], lw);
            atomicAdd(&p.totals[4], nt);
        }
    }
    if (err) atomicOr(p.errWord, (uint32_t)err);
}

// ---------------------------------------------------------------- ray reordering
// Counting sort of the active list (or of the shadow queries) by ray key (raysort.cuh)
// before the traversal kernel that takes them. Only the order in which the kernel takes
// the paths changes; what each path computes does not depend on it.
// Keys and their histogram (one atomic per distinct key per warp) of the active list
// (SHADOW false: entry i is path slot listIn[i]) or of the shadow queries (SHADOW true:
// entry i is shadow record i).
template <bool SHADOW>
__global__ void __launch_bounds__(kBlock) kRayKeys(KParams p) {
    const uint32_t n = SHADOW ? p.cnt[kQShadow] : p.cnt[kQIn];
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * kBlock + (threadIdx.x & ~31u); base < n; base += gridDim.x * kBlock) {
        const uint32_t i = base + lane;
        uint32_t key = 0xFFFFFFFFu;
        if (i < n) {
            float4 a, b;
            uint32_t slot;
            if (SHADOW) {
                const ShadowRec* sr = p.shadow + i;
                a = *reinterpret_cast<const float4*>(&sr->ox);
                b = *reinterpret_cast<const float4*>(&sr->dx);
                slot = __float_as_uint(b.w);
            } else {
                slot = p.listIn[i];
                a = *reinterpret_cast<const float4*>(&p.paths[slot].ox);
                b = *reinterpret_cast<const float4*>(&p.paths[slot].dx);
            }
            const uint32_t job = p.paths[slot].flags >> 8;
            key = rayKey(p.jobs[job].view, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z));
            p.rayKeys[i] = key;
        }
        const uint32_t grp = __match_any_sync(0xffffffffu, key);
        if (i < n && (int)lane == __ffs(grp) - 1) atomicAdd(&p.rayBins[key], (uint32_t)__popc(grp));
    }
}

// Scatter into key order (lanes of one warp with the same key keep their relative order);
// the bins are left zeroed for the next iteration's histogram.
template <bool SHADOW>
__global__ void __launch_bounds__(kBlock) kRayScatter(KParams p) {
    const uint32_t n = SHADOW ? p.cnt[kQShadow] : p.cnt[kQIn];
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * kBlock + (threadIdx.x & ~31u); base < n; base += gridDim.x * kBlock) {
        const uint32_t i = base + lane;
        const uint32_t key = i < n ? p.rayKeys[i] : 0xFFFFFFFFu;
        const uint32_t grp = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(grp) - 1;
        uint32_t pos = 0;
        if (i < n && (int)lane == leader) pos = atomicAdd(&p.rayBins[key], (uint32_t)__popc(grp));
        pos = __shfl_sync(grp, pos, leader);
        if (i < n) p.raySorted[pos + (uint32_t)__popc(grp & ((1u << lane) - 1u))] = SHADOW ? i : p.listIn[i];
    }
}


// Active list -> per-class lists (and kClassDone -> the done list): per block, the warps'
// groups of one class take consecutive places (shared-memory counts), then one atomic per
// class per block.
__global__ void __launch_bounds__(kAggBlock, 4) kClassify(KParams p, uint32_t* classLists) {
    constexpr int kLists = kShadeClasses + 1;   // the class lists and the done list
    __shared__ uint32_t sCount[kLists], sBase[kLists];
    const uint32_t n = p.cnt[kQIn];
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t bb = blockIdx.x * kAggBlock; bb < n; bb += gridDim.x * kAggBlock) {   // block-uniform
        const uint32_t i = bb + threadIdx.x;
        const bool valid = i < n;
        uint32_t cls = 0xFFFFFFFFu, slot = 0;
        if (valid) {
            slot = p.listIn[i];
            cls = p.hits[slot].pad[0];   // written by the extend store (shadeClass or kClassDone)
        }
        __syncthreads();   // the previous iteration's reads of sBase are over
        if (threadIdx.x < (unsigned)kLists) sCount[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t grp = __match_any_sync(0xffffffffu, cls);
        const int leader = __ffs(grp) - 1;
        uint32_t off = 0;
        if (valid && (int)lane == leader) off = atomicAdd(&sCount[cls], (uint32_t)__popc(grp));
        off = __shfl_sync(0xffffffffu, off, leader);
        __syncthreads();
        if (threadIdx.x < (unsigned)kLists) {
            const uint32_t c = sCount[threadIdx.x];
            uint32_t* counter = threadIdx.x < (unsigned)kShadeClasses ? &p.cnt[kQClass0 + threadIdx.x] : &p.cnt[kQDone];
            sBase[threadIdx.x] = c ? atomicAdd(counter, c) : 0u;
        }
        __syncthreads();
        if (valid) {
            const uint32_t at = sBase[cls] + off + (uint32_t)__popc(grp & ((1u << lane) - 1u));
            if (cls < (uint32_t)kShadeClasses) classLists[(size_t)cls * p.capacity + at] = slot;
            else p.done[at] = slot;
        }
    }
}

// One bounce of path (VOL = false) or volpath (VOL = true) for the slots of one shade
// class; M is the set of lobes the class can meet (every lobe for class 4). With
// M = kLobesNone the kernel serves the medium class: it samples the medium, finishes the
// bounce of paths that scatter in it, and hands each other path on to its surface
// class (medium sampling marked done) for a surface kernel later in the iteration.
// EXT: some job of the launch uses the rarer features (SceneView::ext); without them the
// kernel keeps the area-light, static-transform code only.
template <bool VOL, uint32_t M, bool EXT>
__global__ void __launch_bounds__(kBlock) kShade(KParams p, const uint32_t* list, const uint32_t* count) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        uint32_t slot = list[i];
        PathState ps = p.paths[slot];
        const HitRec h = p.hits[slot];
        const float time = EXT ? p.slotTime[slot] : 0.0f;
        const uint32_t jobIdx = ps.flags >> 8;
        const JobDev& j = p.jobs[jobIdx];
        const SceneView& s = j.view;
        Rng rng = loadRng(ps);
        V3 o = v3(ps.ox, ps.oy, ps.oz), d = v3(ps.dx, ps.dy, ps.dz);
        V3 tp = v3(ps.tpr, ps.tpg, ps.tpb), L = v3(ps.Lr, ps.Lg, ps.Lb);
        V3 last = v3(ps.lastX, ps.lastY, ps.lastZ);
        uint32_t bounces = ps.bounces & 0xFFFFu, nullB = ps.bounces >> 16;
        uint32_t volB = ps.vsBounces & 0xFFFFu, surfB = ps.vsBounces >> 16;
        bool specular = (ps.flags & 1u) != 0;
        float pdfPrev = ps.pdfPrev;
        int medium = ps.medium;
        const float nL = (float)s.numEmitters;
        bool cont = false, terminate = false, emitShadow = false, handOff = false;
        ShadowRec sr;
        const bool hit = h.inst >= 0;

        do {
            if (VOL && (M == kLobesAll || M == kLobesNone) && medium >= 0 && !(ps.flags & kFlagMediumDone)) {
                // medium->sample (homogeneous.cpp:32-63); the ray's tMax is the hit distance
                const Medium m = s.media[medium];
                float rtmax = hit ? h.t : INFINITY;
                float u0 = next1D(rng);
                float u1 = next1D(rng);
                int ch = min((int)(u0 * 3.0f), 2);
                float sig = ch == 0 ? m.sigT[0] : (ch == 1 ? m.sigT[1] : m.sigT[2]);
                float dist = -logf(1.0f - u1) / sig;
                float t = fminf_(dist, rtmax);
                bool sampled = t < rtmax;
                V3 tr = v3(expf(-m.sigT[0] * t), expf(-m.sigT[1] * t), expf(-m.sigT[2] * t));
                V3 pc = sampled ? v3(m.sigT[0], m.sigT[1], m.sigT[2]) * tr : tr;
                float pdf = (pc.x + pc.y + pc.z) / 3.0f;
                if (pdf == 0.0f) tp = tp * v3s(0.0f);
                else tp = tp * cdiv(tr, pdf);
                if (sampled) {
                    // volumetric scattering event (volPath.cpp:47-112)
                    V3 mp = o + d * t;
                    V3 wo = -d;
                    tp = tp * v3(m.sigS[0], m.sigS[1], m.sigS[2]);
                    if (isBlack(tp)) { terminate = true; break; }
                    float lightSelectPdf = 1.0f / nL;
                    int ei = pickEmitter(s.numEmitters, next1D(rng));
                    LightSample ls;
                    emitterSampleT<EXT>(s, ei, mp, next2D(rng), ls, 0.0f);
                    V3 Li = ls.Li * (1.0f / lightSelectPdf);
                    if (ls.pdf > 1e-6f && !isBlack(Li)) {
                        V3 wi = normalize(ls.p - mp);
                        float g = hgClampG(m.g);
                        float phasePdf = phaseHG(dot(wo, wi), g);
                        if (phasePdf > 1e-6f) {
                            float pl = ls.pdf * lightSelectPdf;
                            float wl = powerHeuristic(pl, ls.delta ? 0.0f : phasePdf);
                            V3 c = ((tp * phasePdf) * Li) * wl;   // Tr applied by the shadow pass
                            sr.ox = mp.x; sr.oy = mp.y; sr.oz = mp.z; sr.tmax = ls.stmax;
                            sr.dx = ls.sd.x; sr.dy = ls.sd.y; sr.dz = ls.sd.z; sr.slot = slot;
                            sr.cr = c.x; sr.cg = c.y; sr.cb = c.z; sr.medium = medium;
                            sr.lx = ls.p.x; sr.ly = ls.p.y; sr.lz = ls.p.z; sr.pad = __float_as_uint(ls.stime);
                            emitShadow = true;
                        }
                    }
                    V3 wi;
                    pdfPrev = hgSample(hgClampG(m.g), wo, wi, next2D(rng));
                    specular = false;
                    last = mp;
                    o = mp;
                    d = wi;
                    if (volB > 6) {
                        float q = fmaxf_(0.05f, fminf_(luminance(tp), 0.99f));
                        if (next1D(rng) > q) { terminate = true; break; }
                        tp = tp * (1.0f / q);
                    }
                    bounces++;
                    volB = min(volB + 1, 0xFFFFu);
                    cont = true;
                    break;
                }
            }
            if (M == kLobesNone) {
                // no scattering: the path reaches its surface (or escapes)
                if (!hit) {
                    if (EXT) L = L + envMissRadiance(s, o, d, tp, specular, pdfPrev, nL);
                    terminate = true;
                } else {
                    handOff = true;
                }
                break;
            }
            const int curMedium = medium;
            if (!hit) {
                if (EXT) L = L + envMissRadiance(s, o, d, tp, specular, pdfPrev, nL);
                terminate = true;
                break;
            }
            SurfInt si = EXT ? surfaceInteraction(s, h, o, d, time)
                             : surfaceInteractionWith(s, h, o, d, s.instS[h.inst].o2w, s.instT[h.inst].w2o);
            const InstShade& is = s.instS[h.inst];
            const Material mat = s.materials[is.material];
            if (EXT && (mat.normalTex | mat.bumpTex)) applyNormalOrBump(s, mat, si);
            Bsdf bsdf;
            const bool hasBsdf = makeLobeT<M>(mat, SlotTexAt<EXT>{s, si}, bsdf.lobe);
            if (is.emitter >= 0) {
                bool skip = (bounces == 0 && !hasBsdf);
                if (!skip) {
                    const Emitter e = s.emitters[is.emitter];
                    V3 Le = emitterEvalAt<EXT>(s, e, si.p, si.n, si.dpdu, si.uv, -d);
                    if (!isBlack(Le)) {
                        float w = 1.0f;
                        if (!specular) {
                            float lightPdf = emitterPdf(s, is.emitter, last, si.p, si.n);
                            float pl = lightPdf * (1.0f / nL);
                            w = powerHeuristic(pdfPrev, pl);
                        }
                        L = L + (tp * Le) * w;
                    }
                }
            }
            if (!hasBsdf) {
                // pass-through boundary (path.cpp:87-92, volPath.cpp:171-177)
                if (nullB++ > 100) { terminate = true; break; }
                if (VOL) {
                    medium = is.hasMedia ? (dot(d, si.n) > 0.0f ? is.mediumOut : is.mediumIn) : -1;
                }
                o = si.p;
                cont = true;
                break;
            }
            bsdf.fr = shadingFrame(si.n, si.dpdu);
            // next event estimation (path.cpp:104-151, volPath.cpp:193-220)
            float lightSelectPdf = 1.0f / nL;
            int ei = pickEmitter(s.numEmitters, next1D(rng));
            LightSample ls;
            emitterSampleT<EXT>(s, ei, si.p, next2D(rng), ls, time);
            V3 Li = ls.Li * (1.0f / lightSelectPdf);
            if (ls.pdf > 1e-6f && !isBlack(Li)) {
                V3 wi = normalize(ls.p - si.p);
                float bp = bsdfPdf<M>(bsdf, -d, wi);
                V3 f = bsdfF<M>(bsdf, -d, wi);
                if (!isBlack(f) && bp > 1e-6f) {
                    float pl = ls.pdf * lightSelectPdf;
                    float wl = powerHeuristic(pl, ls.delta ? 0.0f : bp);
                    V3 c = (((tp * f) * Li) * fabsf(dot(si.n, wi))) * wl;
                    int smed = -1;
                    if (VOL) smed = nextMedium(-d, ls.sd, curMedium, si.n, is.hasMedia ? is.mediumIn : -1, is.hasMedia ? is.mediumOut : -1);
                    sr.ox = si.p.x; sr.oy = si.p.y; sr.oz = si.p.z; sr.tmax = ls.stmax;
                    sr.dx = ls.sd.x; sr.dy = ls.sd.y; sr.dz = ls.sd.z; sr.slot = slot;
                    sr.cr = c.x; sr.cg = c.y; sr.cb = c.z; sr.medium = smed;
                    sr.lx = ls.p.x; sr.ly = ls.p.y; sr.lz = ls.p.z; sr.pad = __float_as_uint(ls.stime);
                    emitShadow = true;
                }
            }
            // BSDF sampling (path.cpp:153-172, volPath.cpp:222-245)
            V2 u2 = next2D(rng);
            float u1 = next1D(rng);
            V3 wi;
            uint32_t type = 0;
            V3 fcos = bsdfSample<M>(bsdf, -d, wi, u2, u1, pdfPrev, type);
            if (isBlack(fcos) || pdfPrev <= 1e-6f) { terminate = true; break; }
            specular = (type & kSpecular) != 0;
            tp = tp * fcos;
            if (VOL) {
                V3 incident = -d;
                last = si.p;
                o = si.p;
                medium = nextMedium(incident, wi, curMedium, si.n, is.hasMedia ? is.mediumIn : -1, is.hasMedia ? is.mediumOut : -1);
                d = wi;
                if (surfB > 2) {
                    float q = fmaxf_(0.05f, fminf_(luminance(tp), 0.99f));
                    if (next1D(rng) > q) { terminate = true; break; }
                    tp = tp * (1.0f / q);
                }
                surfB = min(surfB + 1, 0xFFFFu);
            } else {
                if (bounces > 2) {
                    float q = fmaxf_(0.05f, fminf_(luminance(tp), 0.99f));
                    if (next1D(rng) > q) { terminate = true; break; }
                    tp = tp * (1.0f / q);
                }
                last = si.p;
                o = si.p;
                d = wi;
            }
            bounces++;
            cont = true;
        } while (false);

        if (cont && bounces >= (uint32_t)j.maxDepth) { cont = false; terminate = true; }
        ps.ox = o.x; ps.oy = o.y; ps.oz = o.z; ps.pdfPrev = pdfPrev;
        ps.dx = d.x; ps.dy = d.y; ps.dz = d.z;
        ps.tpr = tp.x; ps.tpg = tp.y; ps.tpb = tp.z;
        ps.Lr = L.x; ps.Lg = L.y; ps.Lb = L.z;
        ps.lastX = last.x; ps.lastY = last.y; ps.lastZ = last.z;
        storeRng(ps, rng);
        ps.bounces = (bounces & 0xFFFFu) | (min(nullB, 0xFFFFu) << 16);
        ps.vsBounces = (volB & 0xFFFFu) | (surfB << 16);
        ps.medium = medium;
        ps.flags = (ps.flags & ~(1u | kFlagMediumDone)) | (specular ? 1u : 0u) | (handOff ? kFlagMediumDone : 0u);
        p.paths[slot] = ps;
        if (M == kLobesNone) {
            // hand-off to the surface class (warp-aggregated per class)
            const uint32_t hc = handOff ? (uint32_t)kClassesPerInt + surfaceClass(s, h.inst) : 0xFFFFFFFFu;
            const uint32_t grp = __match_any_sync(__activemask(), hc);
            if (handOff) {
                const int leader = __ffs(grp) - 1;
                const int lane = threadIdx.x & 31;
                uint32_t b = 0;
                if (lane == leader) b = atomicAdd(&p.cnt[kQClass0 + hc], (uint32_t)__popc(grp));
                b = __shfl_sync(grp, b, leader);
                p.classLists[(size_t)hc * p.capacity + b + (uint32_t)__popc(grp & ((1u << lane) - 1u))] = slot;
            }
        }
        uint32_t k = warpAppend(&p.cnt[kQShadow], emitShadow);
        if (emitShadow) p.shadow[k] = sr;
        uint32_t c = warpAppend(&p.cnt[kQOut], cont);
        if (cont) p.listOut[c] = slot;
        uint32_t dn = warpAppend(&p.cnt[kQDone], terminate);
        if (terminate) p.done[dn] = slot;
    }
}

// Shadow queries of `path`. The reference traces closest hits and treats the segment as
// occluded when the first surface has a BSDF (path.cpp:124-140; after a null-BSDF first
// hit the next segment's tMax is ~0, so the segment counts as clear). ANY = true is the
// plain any-hit query, exact when no job in the launch has null-BSDF materials; ANY =
// false is the closest hit plus the material check.
template <bool ANY>
struct ShadowSrc {
    const KParams* p;
    uint32_t n;
    bool mixed;
    uint32_t rec;   // the shadow record of the query in flight (its path slot and job are read again at the store)
    __device__ uint32_t count() const { return n; }
    __device__ bool load(uint32_t i, TRay& r, const SceneView*& sv, const uint8_t*& nmOut) {
        rec = p->shadowOrder ? p->shadowOrder[i] : i;
        const ShadowRec* sr = p->shadow + rec;
        float4 a = *reinterpret_cast<const float4*>(&sr->ox);
        float4 b = *reinterpret_cast<const float4*>(&sr->dx);
        const uint32_t slot = __float_as_uint(b.w);
        r.o = v3(a.x, a.y, a.z);
        r.tmax = a.w;
        r.d = v3(b.x, b.y, b.z);
        r.tmin = kEpsilon;
        r.time = __uint_as_float(sr->pad);
        const JobDev& j = p->jobs[p->paths[slot].flags >> 8];
        if (mixed && j.integrator != 0) return false;
        sv = &j.view;
        nmOut = nullptr;
        return true;
    }
    __device__ void store(uint32_t i, const THit& h, const SceneView&) {
        const ShadowRec* sr = p->shadow + rec;
        const uint32_t slot = sr->slot;
        PathState* ps = p->paths + slot;
        bool clear = h.inst < 0 || (!ANY && p->jobs[ps->flags >> 8].nullMask[h.inst]);
        if (clear) {
            float4 c = *reinterpret_cast<const float4*>(&sr->cr);
            ps->Lr = ps->Lr + c.x;
            ps->Lg = ps->Lg + c.y;
            ps->Lb = ps->Lb + c.z;
        }
    }
};

template <bool ANY, int SMEM, bool SPEC, bool MOTION = false, int MINB = 8>
__global__ void __launch_bounds__(kBlock, MINB) kShadowPath(KParams p, bool mixed) {
    __shared__ uint32_t stack[SMEM * kBlock];
    const uint32_t n = p.cnt[kQShadow];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.totals[1], (unsigned long long)n);
    ShadowSrc<ANY> src{&p, n, mixed, 0};
    int err = persistentTrace<kBlock, ANY, false, SMEM, SPEC, MOTION, true>(src, p.cnt + kQFetchB, stack, nullptr,
                                                                            p.shadowLeafBatch);
    if (err) atomicOr(p.errWord, (uint32_t)err);
}

// Shadow queries of `volpath`: evaluateTr (volPath.cpp:261-291), a loop of closest hits
// through null-BSDF boundaries multiplying the transmittance of each medium segment.
template <bool VOL, bool MOTION = false>
__global__ void __launch_bounds__(kBlock) kShadow(KParams p, bool mixed) {
    __shared__ uint32_t stack[kStackSize * kBlock];
    uint32_t* stk = stack + threadIdx.x;
    const uint32_t n = p.cnt[kQShadow];
    if (!mixed && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.totals[1], (unsigned long long)n);
    int err = 0;
    for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const ShadowRec sr = p.shadow[i];
        const uint32_t slot = sr.slot;
        const uint32_t jobIdx = p.paths[slot].flags >> 8;
        const JobDev& j = p.jobs[jobIdx];
        if (mixed && j.integrator != 1) continue;
        const SceneView& s = j.view;
        TRay r;
        r.o = v3(sr.ox, sr.oy, sr.oz);
        r.d = v3(sr.dx, sr.dy, sr.dz);
        r.tmin = kEpsilon;
        r.tmax = sr.tmax;
        r.time = __uint_as_float(sr.pad);
        V3 c = v3(sr.cr, sr.cg, sr.cb);
        bool clear;
        if (!VOL) {
            THit h;
            if (j.hasNull) {
                err |= traceRay<kBlock, false, false, false, MOTION>(s, r, h, stk, nullptr, nullptr);
                clear = h.inst < 0 || j.nullMask[h.inst];
            } else {
                err |= traceRay<kBlock, true, false, false, MOTION>(s, r, h, stk, nullptr, nullptr);
                clear = h.inst < 0;
            }
        } else {
            V3 Tr = v3s(1.0f);
            int medium = sr.medium;
            V3 lightP = v3(sr.lx, sr.ly, sr.lz);
            clear = true;
            for (int seg = 0; seg < 256; ++seg) {
                THit h;
                err |= traceRay<kBlock, false, false, false, MOTION>(s, r, h, stk, nullptr, nullptr);
                bool hit = h.inst >= 0;
                if (medium >= 0) {
                    float segT = hit ? h.t : r.tmax;
                    Tr = Tr * mediumTr(s.media[medium], segT);
                }
                if (isBlack(Tr)) { clear = false; break; }
                if (!hit) break;
                if (!j.nullMask[h.inst]) { clear = false; break; }
                HitRec hr;
                hr.t = h.t; hr.u = h.u; hr.v = h.v; hr.inst = h.inst; hr.slot = h.slot;
                SurfInt si = MOTION ? surfaceInteraction(s, hr, r.o, r.d, r.time)
                                    : surfaceInteractionWith(s, hr, r.o, r.d, s.instS[h.inst].o2w, s.instT[h.inst].w2o);
                const InstShade& is = s.instS[h.inst];
                // volPath.cpp:277: computeScatteringFunctions applies the material's normal or
                // bump map before the medium is chosen by the side the ray leaves through
                if (s.ext) {
                    const Material& mat = s.materials[is.material];
                    if (mat.normalTex | mat.bumpTex) applyNormalOrBump(s, mat, si);
                }
                medium = is.hasMedia ? (dot(r.d, si.n) > 0.0f ? is.mediumOut : is.mediumIn) : -1;
                r.o = si.p;
                r.tmin = kEpsilon;
                r.tmax = length(si.p - lightP) - kEpsilon;
                if (seg == 255) { clear = false; err |= 16; }
            }
            c = c * Tr;
        }
        if (clear) {
            PathState* ps = p.paths + slot;
            ps->Lr = ps->Lr + c.x;
            ps->Lg = ps->Lg + c.y;
            ps->Lb = ps->Lb + c.z;
        }
    }
    if (err) atomicOr(p.errWord, (uint32_t)err);
}

__device__ __forceinline__ unsigned long long toFixed(float x) {
    x = fminf_(fmaxf_(x, 0.0f), kFixMax);
    return (unsigned long long)__float2ll_rn(x * kFixScale);
}

// film.h:26-69 splat of one finished sample (NaN/Inf zeroed as integrator.h:137-141).
template <bool EXT>
__device__ __forceinline__ void filmSplat(const JobDev& j, const PathState& ps) {
    V3 L = v3(ps.Lr, ps.Lg, ps.Lb);
    int ww = j.wx1 - j.wx0;
    int x = j.wx0 + (int)(ps.pixel % (uint32_t)ww), y = j.wy0 + (int)(ps.pixel / (uint32_t)ww);
    uint64_t key = (uint64_t)y * (uint64_t)j.W + (uint64_t)x + (uint64_t)ps.pass * ((uint64_t)j.W * (uint64_t)j.H);
    Rng r = rngSeed(key);
    V2 s2 = next2D(r);
    float fx = (float)x + s2.x, fy = (float)y + s2.y;
    if (EXT && j.view.camera.kind == kCamThinLens) L = cameraWeigh(j.view.camera, L, r, fx, fy, j.W, j.H);
    if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = v3s(0.0f);
    int x0 = max(0, (int)ceilf(fx - j.frx - 0.5f));
    int x1 = min(j.W - 1, (int)floorf(fx + j.frx - 0.5f));
    int y0 = max(0, (int)ceilf(fy - j.fry - 0.5f));
    int y1 = min(j.H - 1, (int)floorf(fy + j.fry - 0.5f));
    for (int py = y0; py <= y1; ++py) {
        for (int px = x0; px <= x1; ++px) {
            float ox = fx - ((float)px + 0.5f), oy = fy - ((float)py + 0.5f);
            float w;
            if (j.filter == 0) {
                w = (fabsf(ox) <= j.frx && fabsf(oy) <= j.fry) ? 1.0f : 0.0f;
            } else {
                float gx = fmaxf_(0.0f, expf(-j.falpha * ox * ox) - j.fexpX);
                float gy = fmaxf_(0.0f, expf(-j.falpha * oy * oy) - j.fexpY);
                w = gx * gy;
            }
            if (w > 0.0f) {
                size_t idx = (size_t)py * (size_t)j.W + (size_t)px;
                atomicAdd(&j.filmSum[idx * 4 + 0], toFixed(L.x * w));
                atomicAdd(&j.filmSum[idx * 4 + 1], toFixed(L.y * w));
                atomicAdd(&j.filmSum[idx * 4 + 2], toFixed(L.z * w));
                atomicAdd(&j.filmSum[idx * 4 + 3], toFixed(w));
                atomicAdd(&j.filmSq[idx * 3 + 0], L.x * L.x * w);
                atomicAdd(&j.filmSq[idx * 3 + 1], L.y * L.y * w);
                atomicAdd(&j.filmSq[idx * 3 + 2], L.z * L.z * w);
            }
        }
    }
}

// Per-sample film record for the 0.5-radius box filter. A sample at film position
// (fx, fy) with neither coordinate a whole number adds weight 1 to exactly its own pixel
// (floor fx, floor fy): that is the one pixel filmSplat's loop bounds and |offset| <= 0.5
// test select (film.h:26-69). Such a sample is stored as (L.r, L.g, L.b, 1) at its work
// item and added to the film later by kFilmFromSamples; a sample on a whole coordinate
// (it also reaches a neighbouring pixel) is splatted with atomics as before.
//
// With the Gaussian filter every sample is recorded, with its film position within its
// pixel (fx - x, fy - y: exact, as fx lies in [x, x + 1]), and kFilmFromSamplesGauss
// gathers the records of each pixel's neighbourhood.
template <bool EXT>
__device__ __forceinline__ void sampleRecord(const JobDev& j, const PathState& ps) {
    const int ww = j.wx1 - j.wx0;
    const int x = j.wx0 + (int)(ps.pixel % (uint32_t)ww), y = j.wy0 + (int)(ps.pixel / (uint32_t)ww);
    const uint64_t key = (uint64_t)y * (uint64_t)j.W + (uint64_t)x + (uint64_t)ps.pass * ((uint64_t)j.W * (uint64_t)j.H);
    Rng r = rngSeed(key);
    const V2 s2 = next2D(r);
    const float fx = (float)x + s2.x, fy = (float)y + s2.y;
    if (j.filter == 0 && (fx == floorf(fx) || fy == floorf(fy))) {
        filmSplat<EXT>(j, ps);
        return;
    }
    V3 L = v3(ps.Lr, ps.Lg, ps.Lb);
    if (EXT && j.view.camera.kind == kCamThinLens) L = cameraWeigh(j.view.camera, L, r, fx, fy, j.W, j.H);
    if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = v3s(0.0f);
    const uint64_t npix = (uint64_t)ww * (uint64_t)(j.wy1 - j.wy0);
    const uint64_t item = (uint64_t)(ps.pass - (uint32_t)j.firstPass) * npix + ps.pixel;
    j.samples[item] = make_float4(L.x, L.y, L.z, 1.0f);
    if (j.filter != 0) j.sampleOff[item] = make_float2(fx - (float)x, fy - (float)y);
}

// The Gaussian film from per-sample records: one thread per film pixel that the window's
// samples can reach (the window grown by the filter radius, inside the film). For every
// recorded sample of the pixels around it, the same test and weight as filmSplat: the
// pixel must lie in the sample's [ceil(f - r - 0.5), floor(f + r - 0.5)] range on both
// axes (film.h:37-40), w = max(0, exp(-a dx^2) - e_x) * max(0, exp(-a dy^2) - e_y)
// (filter.h:43-47), and w > 0. The fixed-point sums equal the atomic splat's; the float
// sum of wL^2 is taken in a fixed order (source pixel, then pass).
__global__ void kFilmFromSamplesGauss(JobDev j, uint32_t passes) {
    const int ww = j.wx1 - j.wx0, wh = j.wy1 - j.wy0;
    const uint64_t npix = (uint64_t)ww * (uint64_t)wh;
    // a sample of pixel sx lies at fx in [sx, sx + 1], so the pixels it reaches satisfy
    // |px - sx| <= floor(r + 0.5) (the largest bound, floor(fx + r - 0.5), at fx = sx + 1)
    const int Rx = (int)floorf(j.frx + 0.5f), Ry = (int)floorf(j.fry + 0.5f);
    const int tx0 = max(0, j.wx0 - Rx), tx1 = min(j.W, j.wx1 + Rx);
    const int ty0 = max(0, j.wy0 - Ry), ty1 = min(j.H, j.wy1 + Ry);
    const uint64_t tw = (uint64_t)max(tx1 - tx0, 0), nt = tw * (uint64_t)max(ty1 - ty0, 0);
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nt; q += (uint64_t)gridDim.x * blockDim.x) {
        const int px = tx0 + (int)(q % tw), py = ty0 + (int)(q / tw);
        unsigned long long sr = 0, sg = 0, sb = 0, sw = 0;
        float qr = 0.0f, qg = 0.0f, qb = 0.0f;
        for (int sy = max(py - Ry, j.wy0); sy <= min(py + Ry, j.wy1 - 1); ++sy) {
            for (int sx = max(px - Rx, j.wx0); sx <= min(px + Rx, j.wx1 - 1); ++sx) {
                const uint64_t src = (uint64_t)(sy - j.wy0) * (uint64_t)ww + (uint64_t)(sx - j.wx0);
                for (uint32_t k = 0; k < passes; ++k) {
                    const uint64_t item = (uint64_t)k * npix + src;
                    const float4 rec = j.samples[item];
                    if (rec.w == 0.0f) continue;
                    const float2 off = j.sampleOff[item];
                    const float fx = (float)sx + off.x, fy = (float)sy + off.y;
                    if (px < max(0, (int)ceilf(fx - j.frx - 0.5f)) || px > min(j.W - 1, (int)floorf(fx + j.frx - 0.5f))) continue;
                    if (py < max(0, (int)ceilf(fy - j.fry - 0.5f)) || py > min(j.H - 1, (int)floorf(fy + j.fry - 0.5f))) continue;
                    const float ox = fx - ((float)px + 0.5f), oy = fy - ((float)py + 0.5f);
                    const float gx = fmaxf_(0.0f, expf(-j.falpha * ox * ox) - j.fexpX);
                    const float gy = fmaxf_(0.0f, expf(-j.falpha * oy * oy) - j.fexpY);
                    const float w = gx * gy;
                    if (!(w > 0.0f)) continue;
                    sr += toFixed(rec.x * w);
                    sg += toFixed(rec.y * w);
                    sb += toFixed(rec.z * w);
                    sw += toFixed(w);
                    qr += rec.x * rec.x * w;
                    qg += rec.y * rec.y * w;
                    qb += rec.z * rec.z * w;
                }
            }
        }
        const size_t idx = (size_t)py * (size_t)j.W + (size_t)px;
        j.filmSum[idx * 4 + 0] += sr;
        j.filmSum[idx * 4 + 1] += sg;
        j.filmSum[idx * 4 + 2] += sb;
        j.filmSum[idx * 4 + 3] += sw;
        j.filmSq[idx * 3 + 0] += qr;
        j.filmSq[idx * 3 + 1] += qg;
        j.filmSq[idx * 3 + 2] += qb;
    }
}

// Adds the per-sample records of `passes` passes into the job's film: one thread per
// window pixel, records in pass order. The fixed-point sums equal what filmSplat's atomics
// add (integer sums do not depend on order); the float sum of wL^2 is taken in pass order.
// Records never written (samples splatted directly, or not rendered) have w = 0.
__global__ void kFilmFromSamples(JobDev j, uint32_t passes) {
    const int ww = j.wx1 - j.wx0;
    const uint64_t npix = (uint64_t)ww * (uint64_t)(j.wy1 - j.wy0);
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < npix; q += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long sr = 0, sg = 0, sb = 0, sw = 0;
        float qr = 0.0f, qg = 0.0f, qb = 0.0f;
        for (uint32_t k = 0; k < passes; ++k) {
            const float4 rec = j.samples[(uint64_t)k * npix + q];
            if (rec.w == 0.0f) continue;
            sr += toFixed(rec.x);
            sg += toFixed(rec.y);
            sb += toFixed(rec.z);
            sw += toFixed(1.0f);
            qr += rec.x * rec.x;
            qg += rec.y * rec.y;
            qb += rec.z * rec.z;
        }
        const int x = j.wx0 + (int)(q % (uint64_t)ww), y = j.wy0 + (int)(q / (uint64_t)ww);
        const size_t idx = (size_t)y * (size_t)j.W + (size_t)x;
        j.filmSum[idx * 4 + 0] += sr;
        j.filmSum[idx * 4 + 1] += sg;
        j.filmSum[idx * 4 + 2] += sb;
        j.filmSum[idx * 4 + 3] += sw;
        j.filmSq[idx * 3 + 0] += qr;
        j.filmSq[idx * 3 + 1] += qg;
        j.filmSq[idx * 3 + 2] += qb;
    }
}

// ---------------------------------------------------------------- retire / refill
// Threads in `want` take work items from the active jobs: one thread per block walks the
// active list from a per-block round-robin start (the first job with FIFO admission) and
// takes one contiguous range per job until the block is served (at most four jobs per
// grab); threads left over stay idle this iteration. One atomic per job per block.
struct GrabScratch {
    uint32_t cnt[kAggWarps];
    uint32_t job[4], n[4];
    unsigned long long first[4];
};
__device__ __forceinline__ bool blockGrab(const KParams& p, bool want, uint32_t& jobOut, uint64_t& itemOut, GrabScratch& g) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    uint32_t total;
    uint32_t r = blockRank(mask, g.cnt, total);
    if (threadIdx.x == 0) {
        uint32_t remaining = total;
        int ns = 0;
        if (remaining > 0) {
            const uint32_t na = p.cnt[kQActive];
            const uint32_t start = p.fifo ? 0u : blockIdx.x + p.cnt[kQIter];
            for (uint32_t t = 0; t < na && remaining > 0 && ns < 4; ++t) {
                const uint32_t jid = p.active[(start + t) % na];
                const unsigned long long end = p.jobs[jid].workEnd;
                if (*(volatile unsigned long long*)&p.ctl[jid].next >= end) continue;
                const unsigned long long got = atomicAdd(&p.ctl[jid].next, (unsigned long long)remaining);
                if (got >= end) continue;
                const uint32_t avail = (uint32_t)min((unsigned long long)remaining, end - got);
                g.job[ns] = jid; g.first[ns] = got; g.n[ns] = avail;
                ++ns;
                remaining -= avail;
            }
        }
        for (int k = ns; k < 4; ++k) g.n[k] = 0;
    }
    __syncthreads();
    if (!want) return false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (r < g.n[k]) { jobOut = g.job[k]; itemOut = g.first[k] + r; return true; }
        r -= g.n[k];
    }
    return false;
}

// Per-job retired counts of one block iteration: the warps' groups add into a small
// shared table (one entry per job met), flushed with one atomic per job; a job that finds
// the table full adds directly.
constexpr int kRetireJobSlots = 8;
struct RetireScratch {
    uint32_t job[kRetireJobSlots];
    uint32_t n[kRetireJobSlots];
};
__device__ __forceinline__ void blockRetired(const KParams& p, uint32_t jobIdx, RetireScratch& rs) {
    const uint32_t lane = threadIdx.x & 31u;
    __syncthreads();   // the previous flush is over
    if (threadIdx.x < (unsigned)kRetireJobSlots) { rs.job[threadIdx.x] = 0xFFFFFFFFu; rs.n[threadIdx.x] = 0; }
    __syncthreads();
    const uint32_t grp = __match_any_sync(0xffffffffu, jobIdx);
    if (jobIdx != 0xFFFFFFFFu && (int)lane == __ffs(grp) - 1) {
        bool placed = false;
        for (int k = 0; k < kRetireJobSlots && !placed; ++k) {
            const uint32_t old = atomicCAS(&rs.job[k], 0xFFFFFFFFu, jobIdx);
            if (old == 0xFFFFFFFFu || old == jobIdx) {
                atomicAdd(&rs.n[k], (uint32_t)__popc(grp));
                placed = true;
            }
        }
        if (!placed) atomicAdd(&p.ctl[jobIdx].retired, (unsigned long long)__popc(grp));
    }
    __syncthreads();
    if (threadIdx.x < (unsigned)kRetireJobSlots && rs.job[threadIdx.x] != 0xFFFFFFFFu)
        atomicAdd(&p.ctl[rs.job[threadIdx.x]].retired, (unsigned long long)rs.n[threadIdx.x]);
}

// Finished paths (done list): film splat and per-job retired count. Finished and idle
// slots (free list) then take new work items; slots left without work join the next
// free list. The loop is block-uniform (all threads of a block iterate together).
template <bool EXT>
__global__ void __launch_bounds__(kAggBlock, 3) kRetire(KParams p) {
    __shared__ GrabScratch sGrab;
    __shared__ AggScratch sApp;
    __shared__ RetireScratch sRet;
    const uint32_t nd = p.cnt[kQDone], nf = p.cnt[kQFree];
    const bool work = p.cnt[kQWork] != 0;
    // with work left, finished and idle slots take work items; without, only finished
    // paths are retired and the idle slots are copied over
    const uint32_t total = work ? nd + nf : nd;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.totals[2], (unsigned long long)nd);
    if (!work)
        for (uint32_t i = blockIdx.x * kAggBlock + threadIdx.x; i < nf; i += gridDim.x * kAggBlock) p.freeOut[i] = p.freeIn[i];
    for (uint32_t bb = blockIdx.x * kAggBlock; bb < total; bb += gridDim.x * kAggBlock) {
        const uint32_t i = bb + threadIdx.x;
        const bool valid = i < total;
        const bool isDone = i < nd;
        const uint32_t slot = valid ? (isDone ? p.done[i] : p.freeIn[i - nd]) : 0u;
        uint32_t jobIdx = 0xFFFFFFFFu;
        if (valid && isDone) {
            PathState ps = p.paths[slot];
            jobIdx = ps.flags >> 8;
            const JobDev& jd = p.jobs[jobIdx];
            if (jd.samples) sampleRecord<EXT>(jd, ps);
            else filmSplat<EXT>(jd, ps);
        }
        if (bb < nd) blockRetired(p, jobIdx, sRet);   // block-uniform: done slots come first
        uint32_t gj = 0;
        uint64_t item = 0;
        bool got = false;
        if (work) got = blockGrab(p, valid, gj, item, sGrab);   // `work` is uniform over the grid
        if (got) {
            PathState ps;
            const float t = generatePath<EXT>(p.jobs[gj], gj, item, ps);
            if (EXT) p.slotTime[slot] = t;
            p.paths[slot] = ps;
        }
        const bool idle = valid && !got;
        uint32_t k, f;
        blockAppend2(reinterpret_cast<unsigned long long*>(p.cnt + kQOut), got, idle, k, f, sApp);
        if (got) p.listOut[k] = slot;
        if (idle) p.freeOut[f] = slot;
    }
}

__global__ void kEndIter(uint32_t* cnt) {
    cnt[kQIn] = cnt[kQOut];
    cnt[kQFree] = cnt[kQFreeOut];
}

// Fixed-point film -> float film [H*W][7] (sum wL rgb, sum w, sum wL^2 rgb).
__global__ void kFilmResolve(const unsigned long long* __restrict__ sum, const float* __restrict__ sq, float* __restrict__ out,
                             size_t npix) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < npix; q += (size_t)gridDim.x * blockDim.x) {
        float* o = out + q * 7;
        for (int k = 0; k < 4; ++k) o[k] = (float)((double)sum[q * 4 + k] * (1.0 / 16777216.0));
        for (int k = 0; k < 3; ++k) o[4 + k] = sq[q * 3 + k];
    }
}

// Every slot idle: free list = [0, n).
__global__ void kResetPool(uint32_t* freeList, uint32_t n, uint32_t* cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) freeList[i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int k = 0; k < kQCount; ++k)
            if (k != kQActive) cnt[k] = 0;
        cnt[kQFree] = n;
    }
}

// One shade launch per material class of one integrator (empty classes exit at once).
template <bool VOL, bool EXT>
static void launchShade(const KParams& kp, uint32_t* classLists, int grid, cudaStream_t st) {
    const size_t cap = kp.capacity;
    const int c0 = VOL ? kClassesPerInt : 0;
    uint32_t* cnt = kp.cnt + kQClass0 + c0;
    uint32_t* lists = classLists + (size_t)c0 * cap;
    static_assert(kMatMatte == 0 && kMatPlastic == 1 && kMatConductor == 2 && kMatGlass == 3,
                  "material classes follow the material type codes");
    // medium sampling first: its hand-offs join the surface classes shaded below
    if (VOL) kShade<true, kLobesNone, EXT><<<grid, kBlock, 0, st>>>(kp, lists + kMediumClass * cap, cnt + kMediumClass);
    kShade<VOL, kLobesMatte, EXT><<<grid, kBlock, 0, st>>>(kp, lists + 0 * cap, cnt + 0);
    kShade<VOL, kLobesPlastic, EXT><<<grid, kBlock, 0, st>>>(kp, lists + 1 * cap, cnt + 1);
    kShade<VOL, kLobesConductor, EXT><<<grid, kBlock, 0, st>>>(kp, lists + 2 * cap, cnt + 2);
    kShade<VOL, kLobesGlass, EXT><<<grid, kBlock, 0, st>>>(kp, lists + 3 * cap, cnt + 3);
    kShade<VOL, kLobesAll, EXT><<<grid, kBlock, 0, st>>>(kp, lists + 4 * cap, cnt + 4);
}

// ---------------------------------------------------------------- host driver
Wavefront::Wavefront(Context* c) : ctx_(c) {
    counters_.alloc(kQCount * sizeof(uint32_t));
    GND_CUDA(cudaMemset(counters_.ptr, 0, kQCount * sizeof(uint32_t)));
    totals_.alloc(8 * sizeof(unsigned long long));
    jobTab_.alloc(kMaxJobs * sizeof(JobDev));
    ctl_.alloc(kMaxJobs * sizeof(JobCtl));
    active_.alloc(kMaxJobs * sizeof(uint32_t));
    GND_CUDA(cudaMemset(ctl_.ptr, 0, kMaxJobs * sizeof(JobCtl)));
    GND_CUDA(cudaMallocHost(&snaps_, 2 * sizeof(Snapshot)));
    std::memset(snaps_, 0, 2 * sizeof(Snapshot));
    for (cudaEvent_t& e : snapEv_) GND_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    GND_CUDA(cudaEventCreate(&evStart_));
    GND_CUDA(cudaEventCreate(&evEnd_));
}

cudaEvent_t Wavefront::nextEvent() {
    if (evUsed_ == evPool_.size()) {
        cudaEvent_t e = nullptr;
        GND_CUDA(cudaEventCreate(&e));
        evPool_.push_back(e);
    }
    return evPool_[evUsed_++];
}

uint64_t Wavefront::poolBytes() const {
    uint64_t b = slotBytes() * cap_ + filmOut_.bytes;
    for (const HostJob& j : jobs_)
        if (!j.used) b += j.filmSum.bytes + j.filmSq.bytes;
    return b;
}
Wavefront::~Wavefront() {
    for (cudaEvent_t e : evPool_) cudaEventDestroy(e);
    if (evStart_) cudaEventDestroy(evStart_);
    if (evEnd_) cudaEventDestroy(evEnd_);
    if (pinnedFilm_) cudaFreeHost(pinnedFilm_);
    clearGraphs();
    for (cudaEvent_t e : snapEv_)
        if (e) cudaEventDestroy(e);
    if (snaps_) cudaFreeHost(snaps_);
}

void Wavefront::ensureCapacity(size_t slots) {
    if (slots <= cap_) return;
    clearGraphs();   // the captured launches hold the old buffers
    paths_.alloc(slots * sizeof(PathState));
    times_.alloc(slots * sizeof(float));
    hits_.alloc(slots * sizeof(HitRec));
    listA_.alloc(slots * sizeof(uint32_t));
    listB_.alloc(slots * sizeof(uint32_t));
    freeA_.alloc(slots * sizeof(uint32_t));
    freeB_.alloc(slots * sizeof(uint32_t));
    shadow_.alloc(slots * sizeof(ShadowRec));
    done_.alloc(slots * sizeof(uint32_t));
    classes_.alloc(slots * kShadeClasses * sizeof(uint32_t));
    rayKeys_.alloc(slots * sizeof(uint32_t));
    raySorted_.alloc(slots * sizeof(uint32_t));
    if (!rayBins_.ptr) {
        rayBins_.alloc(kRayBins * sizeof(uint32_t));
        GND_CUDA(cudaMemset(rayBins_.ptr, 0, kRayBins * sizeof(uint32_t)));
    }
    cap_ = slots;
}

void Wavefront::reset(size_t slots) {
    ensureCapacity(std::max<size_t>(slots, 1));
    cudaStream_t st = ctx_->stream;
    cur_ = 0;
    kResetPool<<<ctx_->numSMs * 4, 256, 0, st>>>(freeA_.as<uint32_t>(), (uint32_t)slots, counters_.as<uint32_t>());
    ++launches_;
    GND_CUDA(cudaGetLastError());
    GND_CUDA(cudaMemsetAsync(totals_.ptr, 0, 8 * sizeof(unsigned long long), st));
}

uint64_t Wavefront::jobBytes() const {
    uint64_t b = 0;
    for (const HostJob& j : jobs_)
        if (j.used) b += j.bytes;
    return b;
}

void Wavefront::setPriorities(const std::vector<std::pair<int, uint64_t>>& keys) {
    auto order = [&]() {
        std::vector<int> ids;
        for (int j = 0; j < kMaxJobs; ++j)
            if (jobs_[j].used) ids.push_back(j);
        std::sort(ids.begin(), ids.end(), [&](int a, int b) {
            return jobs_[a].prio != jobs_[b].prio ? jobs_[a].prio < jobs_[b].prio : jobs_[a].seq < jobs_[b].seq;
        });
        return ids;
    };
    const std::vector<int> before = order();
    for (const auto& k : keys)
        if (k.first >= 0 && k.first < kMaxJobs && jobs_[k.first].used) jobs_[k.first].prio = k.second;
    if (order() != before) syncActive();
}

bool Wavefront::busy() const {
    for (const HostJob& j : jobs_)
        if (j.used) return true;
    return false;
}

void Wavefront::syncActive() {
    uint32_t ids[kMaxJobs];
    uint32_t n = 0;
    for (int j = 0; j < kMaxJobs; ++j)
        if (jobs_[j].used) ids[n++] = (uint32_t)j;
    std::sort(ids, ids + n, [&](uint32_t a, uint32_t b) {
        return jobs_[a].prio != jobs_[b].prio ? jobs_[a].prio < jobs_[b].prio : jobs_[a].seq < jobs_[b].seq;
    });
    cudaStream_t st = ctx_->stream;
    if (n) GND_CUDA(cudaMemcpyAsync(active_.ptr, ids, n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    GND_CUDA(cudaMemcpyAsync(counters_.as<uint32_t>() + kQActive, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    // the staging arrays are on the stack: wait for the copies before returning
    GND_CUDA(cudaStreamSynchronize(st));
    activeDirty_ = false;
}

int Wavefront::admit(const DeviceScene& ds, int W, int H, int spp, int firstPass, int maxDepth, int integrator,
                     const int window[4], uint64_t releaseItems) {
    int j = -1;
    for (int k = 0; k < kMaxJobs; ++k)
        if (!jobs_[k].used) { j = k; break; }
    if (j < 0) throw Error(GND_ERR_BUDGET, "job table full");
    if (W <= 0 || H <= 0) throw Error(GND_ERR_INVALID, "job has no film size");
    if (ds.view.numEmitters <= 0) throw Error(GND_ERR_INVALID, "the path integrators need at least one emitter");
    int wx0 = 0, wy0 = 0, wx1 = W, wy1 = H;
    if (window && (window[0] | window[1] | window[2] | window[3])) {
        wx0 = window[0]; wy0 = window[1]; wx1 = window[2]; wy1 = window[3];
        if (wx0 < 0 || wy0 < 0 || wx1 > W || wy1 > H || wx0 >= wx1 || wy0 >= wy1) throw Error(GND_ERR_INVALID, "bad pixel window");
    }
    HostJob& hj = jobs_[j];
    cudaStream_t st = ctx_->stream;
    const size_t npixAll = (size_t)W * H;
    // film buffers stay allocated between jobs of the slot and are reused when large enough
    hj.filmSum.ensure(npixAll * 4 * sizeof(unsigned long long));
    hj.filmSq.ensure(npixAll * 3 * sizeof(float));
    GND_CUDA(cudaMemsetAsync(hj.filmSum.ptr, 0, npixAll * 4 * sizeof(unsigned long long), st));
    GND_CUDA(cudaMemsetAsync(hj.filmSq.ptr, 0, npixAll * 3 * sizeof(float), st));
    hj.bytes = npixAll * (4 * sizeof(unsigned long long) + 3 * sizeof(float));
    JobDev& jd = hj.dev;
    jd = JobDev{};
    jd.view = ds.view;
    jd.view.camera.width = W;
    jd.view.camera.height = H;
    jd.view.camera.aspect = W / (float)H;   // perspective.cpp:20 (getAspectRatio)
    jd.nullMask = ds.nullMask.as<uint8_t>();
    jd.filmSum = hj.filmSum.as<unsigned long long>();
    jd.filmSq = hj.filmSq.as<float>();
    jd.W = W; jd.H = H; jd.maxDepth = maxDepth; jd.integrator = integrator;
    jd.wx0 = wx0; jd.wy0 = wy0; jd.wx1 = wx1; jd.wy1 = wy1;
    jd.filter = ds.filter;
    jd.frx = ds.filter == 0 ? 0.5f : ds.filterRadius[0];
    jd.fry = ds.filter == 0 ? 0.5f : ds.filterRadius[1];
    jd.falpha = ds.filterAlpha;
    jd.fexpX = std::exp(-jd.falpha * jd.frx * jd.frx);   // filter.h:39-40
    jd.fexpY = std::exp(-jd.falpha * jd.fry * jd.fry);
    jd.hasNull = ds.hasNullMaterials ? 1 : 0;
    jd.firstPass = firstPass;
    hj.total = (uint64_t)(wx1 - wx0) * (uint64_t)(wy1 - wy0) * (uint64_t)spp;
    hj.released = std::min<uint64_t>(releaseItems, hj.total);
    hj.retired = 0;
    jd.workBegin = 0;
    jd.workEnd = hj.released;
    hj.used = true;
    hj.seq = seqNext_++;
    hj.prio = hj.seq;
    GND_CUDA(cudaMemcpyAsync(jobTab_.as<JobDev>() + j, &jd, sizeof(JobDev), cudaMemcpyHostToDevice, st));
    GND_CUDA(cudaMemsetAsync(ctl_.as<JobCtl>() + j, 0, sizeof(JobCtl), st));
    syncActive();
    return j;
}

void Wavefront::release(int j, uint64_t upTo) {
    HostJob& hj = jobs_[j];
    hj.released = std::min(upTo, hj.total);
    hj.dev.workEnd = hj.released;
    GND_CUDA(cudaMemcpyAsync(&jobTab_.as<JobDev>()[j].workEnd, &hj.dev.workEnd, sizeof(uint64_t), cudaMemcpyHostToDevice,
                             ctx_->stream));
    GND_CUDA(cudaStreamSynchronize(ctx_->stream));
}

uint64_t Wavefront::retired(int j) {
    JobCtl c;
    GND_CUDA(cudaMemcpyAsync(&c, ctl_.as<JobCtl>() + j, sizeof(JobCtl), cudaMemcpyDeviceToHost, ctx_->stream));
    GND_CUDA(cudaStreamSynchronize(ctx_->stream));
    jobs_[j].retired = c.retired;
    return c.retired;
}

void Wavefront::readRetired(std::vector<uint64_t>& out) {
    JobCtl c[kMaxJobs];
    GND_CUDA(cudaMemcpyAsync(c, ctl_.ptr, sizeof(c), cudaMemcpyDeviceToHost, ctx_->stream));
    GND_CUDA(cudaStreamSynchronize(ctx_->stream));
    out.resize(kMaxJobs);
    for (int j = 0; j < kMaxJobs; ++j) {
        out[j] = c[j].retired;
        if (jobs_[j].used) jobs_[j].retired = c[j].retired;
    }
}

void Wavefront::readCtl(std::vector<JobCtl>& out) {
    out.resize(kMaxJobs);
    GND_CUDA(cudaMemcpyAsync(out.data(), ctl_.ptr, kMaxJobs * sizeof(JobCtl), cudaMemcpyDeviceToHost, ctx_->stream));
    GND_CUDA(cudaStreamSynchronize(ctx_->stream));
    for (int j = 0; j < kMaxJobs; ++j)
        if (jobs_[j].used) jobs_[j].retired = out[j].retired;
}

void Wavefront::useSampleRecords(int j, uint64_t items) {
    cudaStream_t st = ctx_->stream;
    samples_.ensure(items * sizeof(float4));
    GND_CUDA(cudaMemsetAsync(samples_.ptr, 0, items * sizeof(float4), st));
    HostJob& hj = jobs_[j];
    hj.dev.samples = samples_.as<float4>();
    hj.dev.sampleOff = nullptr;
    if (hj.dev.filter != 0) {
        sampleOff_.ensure(items * sizeof(float2));
        hj.dev.sampleOff = sampleOff_.as<float2>();
    }
    // pageable sources: the copies are staged before the call returns
    GND_CUDA(cudaMemcpyAsync(&jobTab_.as<JobDev>()[j].samples, &hj.dev.samples, sizeof(float4*), cudaMemcpyHostToDevice, st));
    GND_CUDA(cudaMemcpyAsync(&jobTab_.as<JobDev>()[j].sampleOff, &hj.dev.sampleOff, sizeof(float2*), cudaMemcpyHostToDevice, st));
}

void Wavefront::filmFromSamples(int j, uint64_t items) {
    const JobDev& jd = jobs_[j].dev;
    const uint64_t npix = (uint64_t)(jd.wx1 - jd.wx0) * (uint64_t)(jd.wy1 - jd.wy0);
    if (!jd.samples || npix == 0) return;
    const uint32_t passes = (uint32_t)(items / npix);
    if (jd.filter != 0) {
        const int grid = (int)std::min<uint64_t>(((uint64_t)jd.W * jd.H + 255) / 256, (uint64_t)ctx_->numSMs * 16);
        kFilmFromSamplesGauss<<<std::max(grid, 1), 256, 0, ctx_->stream>>>(jd, passes);
        ++launches_;
        GND_CUDA(cudaGetLastError());
        return;
    }
    const int grid = (int)std::min<uint64_t>((npix + 255) / 256, (uint64_t)ctx_->numSMs * 16);
    kFilmFromSamples<<<std::max(grid, 1), 256, 0, ctx_->stream>>>(jd, passes);
    ++launches_;
    GND_CUDA(cudaGetLastError());
}

void Wavefront::stop(int j) {
    HostJob& hj = jobs_[j];
    hj.dev.workEnd = 0;
    GND_CUDA(cudaMemsetAsync(&jobTab_.as<JobDev>()[j].workEnd, 0, sizeof(uint64_t), ctx_->stream));
}

const float* Wavefront::resolvePinned(int j) {
    HostJob& hj = jobs_[j];
    const size_t npix = (size_t)hj.dev.W * hj.dev.H;
    const size_t bytes = npix * 7 * sizeof(float);
    filmOut_.ensure(bytes);
    if (pinnedFilmBytes_ < bytes) {
        if (pinnedFilm_) GND_CUDA(cudaFreeHost(pinnedFilm_));
        pinnedFilm_ = nullptr;
        pinnedFilmBytes_ = 0;
        GND_CUDA(cudaMallocHost(&pinnedFilm_, bytes));
        pinnedFilmBytes_ = bytes;
    }
    cudaStream_t st = ctx_->stream;
    int grid = (int)std::min<size_t>((npix + 255) / 256, (size_t)ctx_->numSMs * 8);
    kFilmResolve<<<std::max(grid, 1), 256, 0, st>>>(hj.filmSum.as<unsigned long long>(), hj.filmSq.as<float>(),
                                                    filmOut_.as<float>(), npix);
    ++launches_;
    GND_CUDA(cudaGetLastError());
    GND_CUDA(cudaMemcpyAsync(pinnedFilm_, filmOut_.ptr, bytes, cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaStreamSynchronize(st));
    return pinnedFilm_;
}

void Wavefront::resolve(int j, float* filmHost) {
    const float* f = resolvePinned(j);
    std::memcpy(filmHost, f, (size_t)jobs_[j].dev.W * jobs_[j].dev.H * 7 * sizeof(float));
}

void Wavefront::finish(int j, float* filmHost) {
    HostJob& hj = jobs_[j];
    const size_t n = (size_t)hj.dev.W * hj.dev.H * 7;
    if (filmHost) {
        const float* f = resolvePinned(j);
        for (size_t q = 0; q < n; ++q) filmHost[q] += f[q];
    }
    drop(j);
}

void Wavefront::finishFixed(int j, uint64_t* sum, float* sq) {
    HostJob& hj = jobs_[j];
    const size_t npix = (size_t)hj.dev.W * hj.dev.H;
    std::vector<unsigned long long> fs(npix * 4);
    std::vector<float> fq(npix * 3);
    GND_CUDA(cudaMemcpyAsync(fs.data(), hj.filmSum.ptr, fs.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             ctx_->stream));
    GND_CUDA(cudaMemcpyAsync(fq.data(), hj.filmSq.ptr, fq.size() * sizeof(float), cudaMemcpyDeviceToHost, ctx_->stream));
    GND_CUDA(cudaStreamSynchronize(ctx_->stream));
    for (size_t q = 0; q < fs.size(); ++q) sum[q] += fs[q];   // modulo 2^64
    if (sq)
        for (size_t q = 0; q < fq.size(); ++q) sq[q] += fq[q];
    drop(j);
}

void Wavefront::drop(int j) {
    HostJob& hj = jobs_[j];
    hj.used = false;   // its film buffers are kept for the next job of the slot
    hj.bytes = 0;
    syncActive();
}

// The plain traversal kernels compiled for MINB blocks per SM.
template <int SMEM, int MINB>
static void launchWide(const KParams& kp, int mix, bool hasNull, int travGrid, cudaStream_t st, cudaEvent_t ea,
                       cudaEvent_t eb, int stage) {
    if (stage == 0) {
        if (ea) GND_CUDA(cudaEventRecord(ea, st));
        kExtend<false, SMEM, false, false, MINB><<<travGrid, kBlock, 0, st>>>(kp);
        if (eb) GND_CUDA(cudaEventRecord(eb, st));
    } else if (mix & 1) {
        if (hasNull) kShadowPath<false, SMEM, false, false, MINB><<<travGrid, kBlock, 0, st>>>(kp, mix == 3);
        else kShadowPath<true, SMEM, false, false, MINB><<<travGrid, kBlock, 0, st>>>(kp, mix == 3);
    }
}

// The traversal kernels for one shared-stack size and speculation setting; bps: blocks
// per SM (the grid is bps per SM; 9 and 10 select the kernels compiled for them, for
// static scenes without speculation or visit counting).
template <int SMEM, bool SPEC>
static void launchTraversal(const KParams& kp, int mix, bool hasNull, bool count, int travGrid, cudaStream_t st,
                            cudaEvent_t ea, cudaEvent_t eb, int stage, bool motion, int bps) {
    if (!motion && !count && !SPEC && bps > 8) {
        if (bps == 9) launchWide<SMEM, 9>(kp, mix, hasNull, travGrid, st, ea, eb, stage);
        else launchWide<SMEM, 10>(kp, mix, hasNull, travGrid, st, ea, eb, stage);
        return;
    }
    if (bps > 8) travGrid = travGrid / bps * 8;   // the 64-register kernels fit 8 blocks per SM
    if (motion) {
        // animated instances: the MOTION kernels (no speculation, no visit counters)
        if (stage == 0) {
            if (ea) GND_CUDA(cudaEventRecord(ea, st));
            kExtend<false, SMEM, false, true><<<travGrid, kBlock, 0, st>>>(kp);
            if (eb) GND_CUDA(cudaEventRecord(eb, st));
        } else if (mix & 1) {
            if (hasNull) kShadowPath<false, SMEM, false, true><<<travGrid, kBlock, 0, st>>>(kp, mix == 3);
            else kShadowPath<true, SMEM, false, true><<<travGrid, kBlock, 0, st>>>(kp, mix == 3);
        }
        return;
    }
    if (stage == 0) {
        if (ea) GND_CUDA(cudaEventRecord(ea, st));
        // the instrumented variant counts the visits of plain nearest-first order: the
        // algorithmic work of a ray, independent of speculation
        if (count) kExtend<true, SMEM, false><<<travGrid, kBlock, 0, st>>>(kp);
        else kExtend<false, SMEM, SPEC><<<travGrid, kBlock, 0, st>>>(kp);
        if (eb) GND_CUDA(cudaEventRecord(eb, st));
    } else if (mix & 1) {
        if (hasNull) kShadowPath<false, SMEM, SPEC><<<travGrid, kBlock, 0, st>>>(kp, mix == 3);
        else kShadowPath<true, SMEM, SPEC><<<travGrid, kBlock, 0, st>>>(kp, mix == 3);
    }
}

template <int SMEM>
static void launchTraversal(const KParams& kp, int mix, bool hasNull, bool count, int travGrid, cudaStream_t st,
                            cudaEvent_t ea, cudaEvent_t eb, int stage, bool spec, bool motion, int bps) {
    if (spec) launchTraversal<SMEM, true>(kp, mix, hasNull, count, travGrid, st, ea, eb, stage, motion, bps);
    else launchTraversal<SMEM, false>(kp, mix, hasNull, count, travGrid, st, ea, eb, stage, motion, bps);
}

void Wavefront::setTune(const Tune& t) {
    if (t != tune_) {
        clearGraphs();
        tune_ = t;
    }
}

void Wavefront::enqueueIteration(KParams kp, int par, int mix, bool hasNull, int profile, cudaStream_t st) {
    const int grid = ctx_->numSMs * 8;
    const int bps = std::min(std::max(tune_.travBlocks, 1), 10);
    const int travGrid = ctx_->numSMs * bps;
    const bool sort = tune_.sort != 0 || mix == 3;   // an unsorted launch serves one integrator
    uint32_t* lists[2] = {listA_.as<uint32_t>(), listB_.as<uint32_t>()};
    uint32_t* frees[2] = {freeA_.as<uint32_t>(), freeB_.as<uint32_t>()};
    kp.listIn = lists[par];
    kp.listOut = lists[par ^ 1];
    kp.freeIn = frees[par];
    kp.freeOut = frees[par ^ 1];
    kBeginIter<<<1, 1, 0, st>>>(kp);
    kp.extList = kp.listIn;
    if (tune_.raySort & 1) {
        kRayKeys<false><<<grid, kBlock, 0, st>>>(kp);
        kRayScan<<<1, 1024, 0, st>>>(kp.rayBins);
        kRayScatter<false><<<grid, kBlock, 0, st>>>(kp);
        kRayClear<<<64, 1024, 0, st>>>(kp.rayBins);
        kp.extList = kp.raySorted;
    }
    cudaEvent_t ea = nullptr, eb = nullptr;
    if (profile & 1) {
        ea = nextEvent();
        eb = nextEvent();
        evs_.push_back(ea);
        evs_.push_back(eb);
    }
    const bool count = (profile & 2) != 0;
    if (tune_.smem == 16) launchTraversal<16>(kp, mix, hasNull, count, travGrid, st, ea, eb, 0, tune_.specExtend != 0, motion_, bps);
    else launchTraversal<32>(kp, mix, hasNull, count, travGrid, st, ea, eb, 0, tune_.specExtend != 0, motion_, bps);
    if (sort) {
        uint32_t* cls = classes_.as<uint32_t>();
        kClassify<<<ctx_->numSMs * 4, kAggBlock, 0, st>>>(kp, cls);   // latency-bound: a full SM of warps
        if (mix & 1) {
            if (ext_) launchShade<false, true>(kp, cls, grid, st);
            else launchShade<false, false>(kp, cls, grid, st);
        }
        if (mix & 2) {
            if (ext_) launchShade<true, true>(kp, cls, grid, st);
            else launchShade<true, false>(kp, cls, grid, st);
        }
    } else if (mix == 2) {
        if (ext_) kShade<true, kLobesAll, true><<<grid, kBlock, 0, st>>>(kp, kp.listIn, kp.cnt + kQIn);
        else kShade<true, kLobesAll, false><<<grid, kBlock, 0, st>>>(kp, kp.listIn, kp.cnt + kQIn);
    } else {
        if (ext_) kShade<false, kLobesAll, true><<<grid, kBlock, 0, st>>>(kp, kp.listIn, kp.cnt + kQIn);
        else kShade<false, kLobesAll, false><<<grid, kBlock, 0, st>>>(kp, kp.listIn, kp.cnt + kQIn);
    }
    kp.shadowOrder = nullptr;
    if ((tune_.raySort & 2) && (mix & 1)) {
        // the keys and the reordered list of the extend stage are free again
        kRayKeys<true><<<grid, kBlock, 0, st>>>(kp);
        kRayScan<<<1, 1024, 0, st>>>(kp.rayBins);
        kRayScatter<true><<<grid, kBlock, 0, st>>>(kp);
        kRayClear<<<64, 1024, 0, st>>>(kp.rayBins);
        kp.shadowOrder = kp.raySorted;
    }
    if (tune_.smem == 16) launchTraversal<16>(kp, mix, hasNull, false, travGrid, st, nullptr, nullptr, 1, tune_.specShadow != 0, motion_, bps);
    else launchTraversal<32>(kp, mix, hasNull, false, travGrid, st, nullptr, nullptr, 1, tune_.specShadow != 0, motion_, bps);
    if (mix & 2) {
        if (motion_) kShadow<true, true><<<grid, kBlock, 0, st>>>(kp, mix == 3);
        else kShadow<true><<<grid, kBlock, 0, st>>>(kp, mix == 3);
    }
    // 12 blocks per SM: its register limit
    if (ext_) kRetire<true><<<ctx_->numSMs * 3, kAggBlock, 0, st>>>(kp);
    else kRetire<false><<<ctx_->numSMs * 3, kAggBlock, 0, st>>>(kp);
    kEndIter<<<1, 1, 0, st>>>(kp.cnt);
    GND_CUDA(cudaGetLastError());
}

void Wavefront::clearGraphs() {
    for (GraphEntry& g : graphs_) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
}

cudaGraphExec_t Wavefront::pairGraph(const KParams& kp, int par, int mix, bool hasNull, cudaStream_t st) {
    const bool fifo = kp.fifo != 0;
    for (const GraphEntry& g : graphs_)
        if (g.par == par && g.mix == mix && g.hasNull == hasNull && g.fifo == fifo && g.motion == motion_ && g.ext == ext_)
            return g.exec;
    cudaGraph_t graph = nullptr;
    GND_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
        enqueueIteration(kp, par, mix, hasNull, 0, st);
        enqueueIteration(kp, par ^ 1, mix, hasNull, 0, st);
    } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    GND_CUDA(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) throw Error(GND_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    graphs_.push_back(GraphEntry{par, mix, hasNull, fifo, motion_, ext_, exec});
    return exec;
}

uint32_t Wavefront::step(int iters, int mix, bool hasNull, int profile, Result& acc) {
    enqueueRound(iters, mix, hasNull, profile, acc, 0);
    const Snapshot& sn = waitRound(0);
    for (int j = 0; j < kMaxJobs; ++j)
        if (jobs_[j].used) jobs_[j].retired = sn.ctl[j].retired;
    return sn.inflight;
}

const Wavefront::Snapshot& Wavefront::waitRound(int slot) {
    GND_CUDA(cudaEventSynchronize(snapEv_[slot]));
    return snaps_[slot];
}

void Wavefront::enqueueRound(int iters, int mix, bool hasNull, int profile, Result& acc, int slot) {
    Context* c = ctx_;
    cudaStream_t st = c->stream;
    motion_ = false;   // the traversal variant for animated instances, when a job needs it
    ext_ = false;      // the shade / retire variants for the rarer features
    for (int j = 0; j < kMaxJobs; ++j) {
        if (!jobs_[j].used) continue;
        if (jobs_[j].dev.view.motion) motion_ = true;
        if (jobs_[j].dev.view.ext) ext_ = true;
    }
    KParams kp{};
    kp.jobs = jobTab_.as<JobDev>();
    kp.paths = paths_.as<PathState>();
    kp.slotTime = times_.as<float>();
    kp.hits = hits_.as<HitRec>();
    kp.shadow = shadow_.as<ShadowRec>();
    kp.done = done_.as<uint32_t>();
    kp.cnt = counters_.as<uint32_t>();
    kp.totals = totals_.as<unsigned long long>();
    kp.ctl = ctl_.as<JobCtl>();
    kp.active = active_.as<uint32_t>();
    kp.errWord = c->errWord.as<uint32_t>();
    kp.capacity = (uint32_t)cap_;
    kp.classLists = classes_.as<uint32_t>();
    kp.leafBatch = (uint32_t)tune_.leafBatch;
    kp.shadowLeafBatch = (uint32_t)tune_.shadowLeafBatch;
    kp.rayKeys = rayKeys_.as<uint32_t>();
    kp.rayBins = rayBins_.as<uint32_t>();
    kp.raySorted = raySorted_.as<uint32_t>();
    kp.fifo = fifo_ ? 1u : 0u;
    // begin, extend, retire, end; classify + 5 shade kernels per integrator when sorting (one
    // shade kernel otherwise); 1 shadow kernel per integrator
    const bool sort = tune_.sort != 0 || mix == 3;
    const int nint = (mix & 1 ? 1 : 0) + (mix & 2 ? 1 : 0);
    const int perIter = 4 + nint + (sort ? 1 + 5 * nint + ((mix & 2) ? 1 : 0) : 1) +   // + the medium kernel
                        ((tune_.raySort & 1) ? 4 : 0) + ((tune_.raySort & 2) && (mix & 1) ? 4 : 0);
    int it = 0;
    while (it < iters) {
        if (tune_.graphs && profile == 0 && iters - it >= 2) {
            GND_CUDA(cudaGraphLaunch(pairGraph(kp, cur_, mix, hasNull, st), st));
            it += 2;
            acc.iterations += 2;
            launches_ += 2 * perIter;
        } else {
            enqueueIteration(kp, cur_, mix, hasNull, profile, st);
            cur_ ^= 1;
            ++it;
            acc.iterations++;
            launches_ += perIter;
        }
    }
    GND_CUDA(cudaMemcpyAsync(&snaps_[slot].inflight, kp.cnt + kQIn, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaMemcpyAsync(&snaps_[slot].err, kp.errWord, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaMemcpyAsync(&snaps_[slot].retiredAll, kp.totals + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaMemcpyAsync(snaps_[slot].ctl, ctl_.ptr, kMaxJobs * sizeof(JobCtl), cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaEventRecord(snapEv_[slot], st));
}

Wavefront::Result Wavefront::render(DeviceScene& ds, int W, int H, int spp, int firstPass, int maxDepth, int integrator,
                                    const int window[4], bool batched, int profile, float* filmHost, gnd_progress_fn cb,
                                    void* user, uint64_t* fixedSum, float* fixedSq) {
    Context* c = ctx_;
    cudaStream_t st = c->stream;
    int wx0 = 0, wy0 = 0, wx1 = W, wy1 = H;
    if (window && (window[0] | window[1] | window[2] | window[3])) {
        wx0 = window[0]; wy0 = window[1]; wx1 = window[2]; wy1 = window[3];
    }
    const uint64_t npix = (uint64_t)std::max(0, wx1 - wx0) * (uint64_t)std::max(0, wy1 - wy0);
    const uint64_t total = npix * (uint64_t)std::max(spp, 0);
    if (npix > (1ull << 31)) throw Error(GND_ERR_INVALID, "window too large");
    Result res;
    if (total == 0) return res;
    // the pool: one pass for plain renders, up to 4M in-flight paths for batched ones
    setTune(ds.tune);
    const int poolLog2 = std::min(std::max(tune_.poolLog2, 16), 26);
    const size_t slots =
        batched ? (size_t)std::min<uint64_t>(total, std::max<uint64_t>(npix, 1ull << poolLog2)) : (size_t)npix;
    for (int j = 0; j < kMaxJobs; ++j)
        if (jobs_[j].used) throw Error(GND_ERR_INVALID, "the engine is serving jobs; render through the server");
    const uint64_t launches0 = launches_;
    reset(slots);
    const int j = admit(ds, W, H, spp, firstPass, maxDepth, integrator, window, batched ? total : npix);
    const int mix = integrator == 1 ? 2 : 1;
    // batched renders keep per-sample records instead of film atomics (at most 2^30
    // records: 16 GiB, and 8 GiB more of film positions with the Gaussian filter)
    const bool records = batched && tune_.sampleFilm && total <= (1ull << 30);
    if (records) {
        try {
            useSampleRecords(j, total);
        } catch (...) {
            drop(j);
            throw;
        }
    }
    cudaEvent_t e0 = evStart_, e1 = evEnd_;
    GND_CUDA(cudaEventRecord(e0, st));
    int pass = 0;
    const int itersPerStep = 2;
    const int64_t iterCap = (int64_t)(maxDepth + 110) * (spp + 2) * 4 + 4096;
    bool cancelled = false;
    try {
        if (batched) {
            // every work item is released: rounds of kRoundIters iterations, one queued
            // ahead of the one whose counters the host is reading
            const int kRoundIters = std::min(std::max(tune_.roundIters & ~1, 2), 64);
            int64_t k = 0, stopAt = -1;
            enqueueRound(kRoundIters, mix, ds.hasNullMaterials, profile, res, 0);
            for (;;) {
                enqueueRound(kRoundIters, mix, ds.hasNullMaterials, profile, res, (int)((k + 1) & 1));
                const Snapshot& sn = waitRound((int)(k & 1));
                const uint64_t r = sn.ctl[j].retired;
                const uint32_t inflight = sn.inflight;
                if (r >= total && inflight == 0) break;
                // after a cancel, only rounds queued after the stop show the final state
                if (cancelled && k > stopAt && inflight == 0) break;
                if (c->cancel && !cancelled) {
                    stop(j);            // queued behind round k + 1
                    stopAt = k + 1;
                    cancelled = true;
                }
                if (res.iterations > iterCap) throw Error(GND_ERR_DEVICE_CHECK, "path iteration limit reached");
                ++k;
            }
            GND_CUDA(cudaStreamSynchronize(st));   // the round queued ahead has nothing left to do
            if (records) filmFromSamples(j, total);
        }
        while (!batched) {
            uint32_t inflight = step(itersPerStep, mix, ds.hasNullMaterials, profile, res);
            uint64_t r = retired(j);
            if (!batched) {
                while (pass < spp && r >= (uint64_t)(pass + 1) * npix) {
                    ++pass;
                    res.passesDone = pass;
                    if (cb) {
                        // film so far, as the reference's per-pass resolve + callback
                        const size_t n = (size_t)W * H;
                        std::vector<unsigned long long> fs(n * 4);
                        std::vector<float> fq(n * 3), pf(n * 7);
                        GND_CUDA(cudaMemcpyAsync(fs.data(), jobs_[j].filmSum.ptr, fs.size() * 8, cudaMemcpyDeviceToHost, st));
                        GND_CUDA(cudaMemcpyAsync(fq.data(), jobs_[j].filmSq.ptr, fq.size() * 4, cudaMemcpyDeviceToHost, st));
                        GND_CUDA(cudaStreamSynchronize(st));
                        for (size_t q = 0; q < n; ++q) {
                            for (int k = 0; k < 4; ++k) pf[q * 7 + k] = (float)((double)fs[q * 4 + k] / 16777216.0);
                            for (int k = 0; k < 3; ++k) pf[q * 7 + 4 + k] = fq[q * 3 + k];
                        }
                        cb(user, firstPass + pass - 1, pf.data(), W, H);
                    }
                    if (pass < spp && !c->cancel) release(j, (uint64_t)(pass + 1) * npix);
                }
                if (c->cancel && !cancelled) cancelled = true;
            }
            if (r >= total && inflight == 0) break;
            if (cancelled && inflight == 0) break;
            if (res.iterations > iterCap) throw Error(GND_ERR_DEVICE_CHECK, "path iteration limit reached");
        }
    } catch (...) {
        drop(j);
        throw;
    }
    if (batched) res.passesDone = cancelled ? (int)(retired(j) / std::max<uint64_t>(npix, 1)) : spp;
    GND_CUDA(cudaEventRecord(e1, st));
    unsigned long long tot[8];
    GND_CUDA(cudaMemcpyAsync(tot, totals_.ptr, sizeof(tot), cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    for (size_t k = 0; k + 1 < evs_.size(); k += 2) {
        float em = 0.f;
        cudaEventElapsedTime(&em, evs_[k], evs_[k + 1]);
        res.extendMs += em;
    }
    evs_.clear();
    evUsed_ = 0;
    try {
        c->checkKernelErrors("render");
    } catch (...) {
        drop(j);
        throw;
    }
    if (fixedSum) finishFixed(j, fixedSum, fixedSq);
    else finish(j, filmHost);
    res.paths = (int64_t)tot[2];
    res.rays = (int64_t)(tot[0] + tot[1]);
    res.extendRays = (int64_t)tot[0];
    res.shadowRays = (int64_t)tot[1];
    res.extendNodes = (int64_t)tot[3];
    res.extendTris = (int64_t)tot[4];
    res.extendNodeWarpSteps = (int64_t)tot[5];
    res.extendLeafSteps = (int64_t)tot[6];
    res.extendLeafWarpSteps = (int64_t)tot[7];
    res.ms = ms;
    res.launches = (int64_t)(launches_ - launches0);
    return res;
}

}  // namespace gnd

using namespace gnd;

extern "C" {

namespace {
// gnd_gpu_render / gnd_gpu_render_fixed: the film goes to `film` or, in fixed-point form,
// to `sum` and `sq`.
void renderCall(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_render_params* prm, float* film, uint64_t* sum, float* sq,
                gnd_render_stats* stats) {
    Context* c = ctxOf(ctxh);
    if (!film && !sum) throw Error(GND_ERR_INVALID, "null film buffer");
    c->bind();
    std::lock_guard<FairMutex> lk(c->mu);
    DeviceScene& ds = c->scene(id);
    gnd_render_params p{};
    p.integrator = -1;
    if (prm) p = *prm;
    int spp = p.spp > 0 ? p.spp : ds.spp;
    int maxDepth = p.max_depth > 0 ? p.max_depth : ds.maxDepth;
    int integ = p.integrator >= 0 ? p.integrator : ds.integrator;
    if (integ != 0 && integ != 1) throw Error(GND_ERR_INVALID, "integrator must be 0 (path_gpu) or 1 (volpath_gpu)");
    if (maxDepth > 65535) maxDepth = 65535;
    if (!c->wave) c->wave = std::make_unique<Wavefront>(c);
    c->cancel = false;
    const int W = p.width > 0 ? p.width : ds.width, H = p.height > 0 ? p.height : ds.height;
    if ((uint64_t)W * (uint64_t)H > (1ull << 31)) throw Error(GND_ERR_INVALID, "film too large");
    Wavefront::Result r = c->wave->render(ds, W, H, spp, p.first_pass, maxDepth, integ, p.window, p.batched != 0,
                                          p.profile, film, p.batched ? nullptr : p.callback, p.user, sum, sq);
    gnd_render_stats rs{};
    rs.paths = r.paths;
    rs.rays = r.rays;
    rs.passes_done = r.passesDone;
    rs.ms = r.ms;
    rs.extend_rays = r.extendRays;
    rs.shadow_rays = r.shadowRays;
    rs.extend_nodes = r.extendNodes;
    rs.extend_tris = r.extendTris;
    rs.extend_node_warp_steps = r.extendNodeWarpSteps;
    rs.extend_leaf_steps = r.extendLeafSteps;
    rs.extend_leaf_warp_steps = r.extendLeafWarpSteps;
    rs.extend_ms = r.extendMs;
    rs.iterations = r.iterations;
    rs.launches = r.launches;
    c->countRender(rs);
    if (stats) *stats = rs;
    if (c->cancel && r.passesDone < spp) throw Error(GND_ERR_CANCELLED, "render cancelled");
}
}  // namespace

gnd_status gnd_gpu_render(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_render_params* prm, float* film, gnd_render_stats* stats) {
    return guarded([&]() {
        if (!film) throw Error(GND_ERR_INVALID, "null film buffer");
        renderCall(ctxh, id, prm, film, nullptr, nullptr, stats);
    });
}

gnd_status gnd_gpu_render_fixed(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_render_params* prm, uint64_t* sum, float* sq,
                                gnd_render_stats* stats) {
    return guarded([&]() {
        if (!sum || !sq) throw Error(GND_ERR_INVALID, "null film buffer");
        renderCall(ctxh, id, prm, nullptr, sum, sq, stats);
    });
}

static Tune tuneFromC(const gnd_tune& t) {
    if (t.pool_log2 < 16 || t.pool_log2 > 26) throw Error(GND_ERR_INVALID, "pool_log2 must be in 16..26");
    if (t.round_iters < 2 || t.round_iters > 64 || (t.round_iters & 1)) throw Error(GND_ERR_INVALID, "round_iters must be even, 2..64");
    if (t.trav_blocks < 1 || t.trav_blocks > 10) throw Error(GND_ERR_INVALID, "trav_blocks must be in 1..10");
    if (t.material_sort != 0 && t.material_sort != 1) throw Error(GND_ERR_INVALID, "material_sort must be 0 or 1");
    if (t.stack_smem != 16 && t.stack_smem != 32) throw Error(GND_ERR_INVALID, "stack_smem must be 16 or 32");
    if (t.graphs != 0 && t.graphs != 1) throw Error(GND_ERR_INVALID, "graphs must be 0 or 1");
    if (t.sample_film != 0 && t.sample_film != 1) throw Error(GND_ERR_INVALID, "sample_film must be 0 or 1");
    if (t.spec_extend != 0 && t.spec_extend != 1) throw Error(GND_ERR_INVALID, "spec_extend must be 0 or 1");
    if (t.spec_shadow != 0 && t.spec_shadow != 1) throw Error(GND_ERR_INVALID, "spec_shadow must be 0 or 1");
    if (t.ray_sort < 0 || t.ray_sort > 7) throw Error(GND_ERR_INVALID, "ray_sort must be in 0..7");
    if (t.leaf_batch < 1 || t.leaf_batch > 32) throw Error(GND_ERR_INVALID, "leaf_batch must be in 1..32");
    if (t.trace_leaf_batch < 1 || t.trace_leaf_batch > 32) throw Error(GND_ERR_INVALID, "trace_leaf_batch must be in 1..32");
    if (t.shadow_leaf_batch < 1 || t.shadow_leaf_batch > 32) throw Error(GND_ERR_INVALID, "shadow_leaf_batch must be in 1..32");
    if (t.trace_blocks < 1 || t.trace_blocks > 10) throw Error(GND_ERR_INVALID, "trace_blocks must be in 1..10");
    Tune r;
    r.poolLog2 = t.pool_log2;
    r.roundIters = t.round_iters;
    r.travBlocks = t.trav_blocks;
    r.sort = t.material_sort;
    r.smem = t.stack_smem;
    r.graphs = t.graphs;
    r.sampleFilm = t.sample_film;
    r.specExtend = t.spec_extend;
    r.specShadow = t.spec_shadow;
    r.raySort = t.ray_sort;
    r.leafBatch = t.leaf_batch;
    r.traceLeafBatch = t.trace_leaf_batch;
    r.shadowLeafBatch = t.shadow_leaf_batch;
    r.traceBlocks = t.trace_blocks;
    return r;
}

static gnd_tune tuneToC(const Tune& t) {
    gnd_tune r;
    r.pool_log2 = t.poolLog2;
    r.round_iters = t.roundIters;
    r.trav_blocks = t.travBlocks;
    r.material_sort = t.sort;
    r.stack_smem = t.smem;
    r.graphs = t.graphs;
    r.sample_film = t.sampleFilm;
    r.spec_extend = t.specExtend;
    r.spec_shadow = t.specShadow;
    r.ray_sort = t.raySort;
    r.leaf_batch = t.leafBatch;
    r.trace_leaf_batch = t.traceLeafBatch;
    r.shadow_leaf_batch = t.shadowLeafBatch;
    r.trace_blocks = t.traceBlocks;
    return r;
}

gnd_status gnd_gpu_get_tune(gnd_gpu_ctx* ctxh, gnd_scene_id id, gnd_tune* out) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!out) throw Error(GND_ERR_INVALID, "null tune");
        std::lock_guard<FairMutex> lk(c->mu);
        *out = tuneToC(c->scene(id).tune);
    });
}

gnd_status gnd_gpu_set_tune(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_tune* t) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!t) throw Error(GND_ERR_INVALID, "null tune");
        const Tune v = tuneFromC(*t);
        std::lock_guard<FairMutex> lk(c->mu);
        c->scene(id).tune = v;
    });
}

gnd_status gnd_gpu_serve_tune(gnd_gpu_ctx* ctxh, const gnd_tune* t) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!t) throw Error(GND_ERR_INVALID, "null tune");
        Tune v = tuneFromC(*t);
        v.sort = 1;   // served jobs of both integrators share launches: always sorted
        std::lock_guard<FairMutex> lk(c->mu);
        c->serveTune = v;
    });
}

gnd_status gnd_gpu_autotune(gnd_gpu_ctx* ctxh, gnd_scene_id id, int32_t spp, int32_t budgetMs, gnd_tune* best,
                            double* mpaths) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        DeviceScene& ds = c->scene(id);
        if (!c->wave) c->wave = std::make_unique<Wavefront>(c);
        if (spp <= 0) spp = 8;
        const int maxDepth = std::min(ds.maxDepth, 65535);
        const auto t0 = std::chrono::steady_clock::now();
        auto spentMs = [&]() {
            return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        };
        // a candidate: one render to capture graphs and size the pool, one timed on the device
        auto trial = [&](const Tune& t) {
            ds.tune = t;
            double v = 0.0;
            for (int r = 0; r < 2; ++r) {
                Wavefront::Result res = c->wave->render(ds, ds.width, ds.height, spp, 0, maxDepth, ds.integrator, nullptr,
                                                        true, 0, nullptr, nullptr, nullptr);
                if (r == 1 && res.ms > 0.0) v = (double)res.paths / res.ms / 1e3;
            }
            c->checkKernelErrors("autotune");
            return v;
        };
        Tune cur = ds.tune;
        double bestV = trial(cur);
        struct Knob {
            int Tune::*field;
            std::vector<int> values;
        };
        const std::vector<Knob> knobs = {
            {&Tune::travBlocks, {8, 9, 10, 6, 4}}, {&Tune::smem, {32, 16}},          {&Tune::sort, {1, 0}},
            {&Tune::poolLog2, {22, 21, 23, 24, 20}}, {&Tune::roundIters, {8, 16, 4}}, {&Tune::graphs, {1, 0}},
            {&Tune::sampleFilm, {1, 0}}, {&Tune::specExtend, {1, 0}}, {&Tune::specShadow, {1, 0}},
            {&Tune::raySort, {1, 3, 0}}, {&Tune::leafBatch, {16, 8, 24, 32}}, {&Tune::shadowLeafBatch, {16, 8, 24, 32}},
        };
        for (int sweep = 0; sweep < 2; ++sweep) {
            bool changed = false;
            for (const Knob& k : knobs) {
                for (int v : k.values) {
                    if (spentMs() > budgetMs) break;
                    // the render knobs only: ray_sort keeps its ray-batch bit (bit 2)
                    const int value = k.field == &Tune::raySort ? (v | (cur.raySort & 4)) : v;
                    if (cur.*(k.field) == value) continue;
                    Tune t = cur;
                    t.*(k.field) = value;
                    double m = trial(t);
                    bool take = m > bestV * 1.02;
                    if (!take && m > bestV * 1.003) {
                        // up to 2% faster: measured twice more, alternating with the current
                        // settings, and taken when faster over the three pairs (some knobs
                        // are worth about 1% on some scenes; one pair cannot tell that
                        // from noise)
                        double sc = bestV, sm = m;
                        for (int r = 0; r < 2; ++r) {
                            sc += trial(cur);
                            sm += trial(t);
                        }
                        take = sm > sc * 1.005;
                        m = sm / 3.0;
                        if (!take) bestV = sc / 3.0;
                    }
                    if (take) {
                        bestV = m;
                        cur = t;
                        changed = true;
                    }
                }
            }
            if (!changed || spentMs() > budgetMs) break;
        }
        ds.tune = cur;
        if (best) *best = tuneToC(cur);
        if (mpaths) *mpaths = bestV;
    });
}

gnd_status gnd_gpu_cancel(gnd_gpu_ctx* ctxh) {
    return guarded([&]() { ctxOf(ctxh)->cancel = true; });
}

}  // extern "C"
