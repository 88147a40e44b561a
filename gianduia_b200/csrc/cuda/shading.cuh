// Device shading library of the radiance path: PCG32 sampler, warps, Fresnel, GGX,
// the BxDF lobes of the in-scope materials, surface interactions, area emitters and
// homogeneous media. Each function restates the reference function cited beside it in
// the same operation order (the file is compiled without FMA contraction); the
// transcendental functions are CUDA's (last-ulp differences from libm are expected).
#pragma once
#include "gnd/layout.h"

namespace gnd {

// ---------------------------------------------------------------- sampler
// pcg32.h:5-32 with stream 1 (inc = 3) and independent.cpp:22-44 seeding
struct Rng {
    uint64_t state;
};
__device__ __forceinline__ uint64_t splitMix64(uint64_t z) {
    z = z + 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
constexpr uint64_t kPcgMult = 6364136223846793005ULL;
constexpr uint64_t kPcgInc = 3ULL;
__device__ __forceinline__ uint32_t pcgNext(Rng& r) {
    uint64_t old = r.state;
    r.state = old * kPcgMult + kPcgInc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return __funnelshift_r(xs, xs, rot);
}
__device__ __forceinline__ Rng rngSeed(uint64_t key) {
    // seed(initstate = splitMix64(key), initseq = 1): state = ((0*M + inc) + init)*M + inc
    Rng r;
    r.state = kPcgInc + splitMix64(key);
    r.state = r.state * kPcgMult + kPcgInc;
    return r;
}
// ldexp((float)u, -32): exact power-of-two scaling of the rounded conversion
__device__ __forceinline__ float next1D(Rng& r) { return __uint2float_rn(pcgNext(r)) * 2.3283064365386962890625e-10f; }
// x first, then y (the order this implementation fixes for Point2f(next, next))
__device__ __forceinline__ V2 next2D(Rng& r) {
    float a = next1D(r);
    float b = next1D(r);
    return V2{a, b};
}

// ---------------------------------------------------------------- warps (warp.cpp)
__device__ __forceinline__ V2 squareToUniformDisk(V2 s) {
    float px = 2.0f * s.x - 1.0f, py = 2.0f * s.y - 1.0f;
    if (fabsf(px) < kEpsilon && fabsf(py) < kEpsilon) return V2{0.f, 0.f};
    float r, theta;
    if (fabsf(px) > fabsf(py)) {
        r = px;
        theta = (float)((kPiD / 4.0) * (double)(py / px));
    } else {
        r = py;
        theta = (float)((kPiD / 2.0) - (kPiD / 4.0) * (double)(px / py));
    }
    return V2{r * cosf(theta), r * sinf(theta)};
}
// warp.cpp:86-113: a regular polygon with one corner at the top, sampled by picking one of
// its `blades` triangles around the centre with s.x and a point in it
__device__ __forceinline__ V2 squareToUniformPolygon(V2 s, int blades) {
    if (blades < 3) return squareToUniformDisk(s);
    const float bladeFloat = s.x * (float)blades;
    const int bladeIdx = min((int)bladeFloat, blades - 1);
    const float u0 = bladeFloat - (float)bladeIdx, u1 = s.y;
    const float deltaTheta = 2.0f * kPi / (float)blades;
    const float offset = kPi / 2.0f;
    const float theta1 = (float)bladeIdx * deltaTheta + offset;
    const float theta2 = (float)(bladeIdx + 1) * deltaTheta + offset;
    const float c1 = cosf(theta1), s1 = sinf(theta1), c2 = cosf(theta2), s2 = sinf(theta2);
    const float r = sqrtf(u0);
    return V2{r * ((1.0f - u1) * c1 + u1 * c2), r * ((1.0f - u1) * s1 + u1 * s2)};
}
__device__ __forceinline__ V3 squareToUniformSphere(V2 s) {
    // squareToUniformSphereCap(s, -1): theta = acos(1 - 2 s.x), phi = 2 pi s.y (double)
    float theta = acosf(1.0f - (1.0f - (-1.0f)) * s.x);
    float phi = (float)(2.0 * kPiD * (double)s.y);
    float st = sinf(theta);
    return v3(st * cosf(phi), st * sinf(phi), cosf(theta));
}
__device__ __forceinline__ V3 squareToCosineHemisphere(V2 s) {
    V2 d = squareToUniformDisk(s);
    float r = d.x * d.x + d.y * d.y;
    return v3(d.x, d.y, sqrtf(1.0f - r));
}
__device__ __forceinline__ float cosineHemispherePdf(V3 v) {
    if (v.z <= 0.0f || fabsf(1.0f - lengthSq(v)) > kEpsilon) return 0.0f;
    return kInvPi * v.z;
}

// ---------------------------------------------------------------- Fresnel (fresnel.h)
__device__ __forceinline__ float frDielectric(float cosI, float etaExt, float etaInt) {
    if (etaExt == etaInt) return 0.0f;
    cosI = clampf(cosI, -1.f, 1.f);
    if (cosI < 0.f) {
        float t = etaExt; etaExt = etaInt; etaInt = t;
        cosI = -cosI;
    }
    float sinI = sqrtf(fmaxf_(0.f, 1.f - cosI * cosI));
    float sinT = etaExt / etaInt * sinI;
    if (sinT >= 1.f) return 1.f;
    float cosT = sqrtf(fmaxf_(0.f, 1.f - sinT * sinT));
    float rPar = ((etaInt * cosI) - (etaExt * cosT)) / ((etaInt * cosI) + (etaExt * cosT));
    float rPerp = ((etaExt * cosI) - (etaInt * cosT)) / ((etaExt * cosI) + (etaInt * cosT));
    return (rPar * rPar + rPerp * rPerp) / 2.f;
}
__device__ __forceinline__ bool refract(V3 wi, V3 n, float eta, V3& wt) {
    float cosI = dot(n, wi);
    float sin2I = fmaxf_(0.f, 1.f - cosI * cosI);
    float sin2T = eta * eta * sin2I;
    if (sin2T >= 1.f) return false;
    float cosT = sqrtf(1.f - sin2T);
    wt = -wi * eta + n * (eta * cosI - cosT);
    return true;
}
__device__ __forceinline__ float frConductorChannel(float cosI, float etaI, float etaT, float k) {
    float c2 = cosI * cosI;
    float s2 = fmaxf_(0.0f, 1.f - c2);
    float eta = etaT / etaI, etak = k / etaI;
    float eta2 = eta * eta, etak2 = etak * etak;
    float t0 = eta2 - etak2 - s2;
    float a2b2 = sqrtf(t0 * t0 + 4.f * eta2 * etak2);
    float t1 = a2b2 + c2;
    float a = sqrtf(fmaxf_(0.0f, 0.5f * (a2b2 + t0)));
    float t2 = 2.f * fabsf(cosI) * a;
    float Rs = (t1 - t2) / (t1 + t2);
    float t3 = c2 * a2b2 + s2 * s2;
    float t4 = t2 * s2;
    float Rp = Rs * (t3 - t4) / (t3 + t4);
    return 0.5f * (Rp + Rs);
}

// ---------------------------------------------------------------- GGX (microfacet.cpp)
__device__ __forceinline__ float roughnessToAlpha(float r) {
    r = fmaxf_(r, 1e-3f);
    return r * r;
}
struct Ggx {
    float a;   // isotropic, alpha clamped to 1e-4
};
__device__ __forceinline__ Ggx makeGgx(float alpha) { return Ggx{fmaxf_(1e-4f, alpha)}; }
__device__ __forceinline__ float ggxD(const Ggx& g, V3 wh) {
    if (fabsf(wh.z) < kEpsilon) return 0.0f;
    float d = (wh.x * wh.x) / (g.a * g.a) + (wh.y * wh.y) / (g.a * g.a) + (wh.z * wh.z);
    return 1.0f / (kPi * g.a * g.a * d * d);
}
__device__ __forceinline__ float ggxG1(const Ggx& g, V3 w) {
    if (fabsf(w.z) < kEpsilon) return 0.0f;
    float a2tan2 = (w.x * w.x * g.a * g.a + w.y * w.y * g.a * g.a) / (w.z * w.z);
    float lambda = 0.5f * (-1.0f + sqrtf(1.0f + a2tan2));
    return 1.0f / (1.0f + lambda);
}
__device__ __forceinline__ float ggxG(const Ggx& g, V3 wo, V3 wi) { return ggxG1(g, wo) * ggxG1(g, wi); }
__device__ __forceinline__ V3 ggxSampleWh(const Ggx& g, V3 wo, V2 u) {
    bool flip = wo.z < 0.0f;
    V3 woh = flip ? -wo : wo;
    V3 Vh = normalize(v3(g.a * woh.x, g.a * woh.y, woh.z));
    float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    V3 T1 = lensq > 0.0f ? divs(v3(-Vh.y, Vh.x, 0.0f), sqrtf(lensq)) : v3(1.0f, 0.0f, 0.0f);
    V3 T2 = cross(Vh, T1);
    float r = sqrtf(u.x);
    float phi = 2.0f * kPi * u.y;
    float t1 = r * cosf(phi);
    float t2 = r * sinf(phi);
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(fmaxf_(0.0f, 1.0f - t1 * t1)) + s * t2;
    V3 Nh = (T1 * t1 + T2 * t2) + Vh * sqrtf(fmaxf_(0.0f, 1.0f - t1 * t1 - t2 * t2));
    V3 wh = normalize(v3(g.a * Nh.x, g.a * Nh.y, fmaxf_(0.0f, Nh.z)));
    if (flip) wh = -wh;
    return wh;
}
__device__ __forceinline__ float ggxPdf(const Ggx& g, V3 wo, V3 wh) {
    if (wo.z * wh.z < 0.0f) return 0.0f;
    float cosO = fabsf(wo.z);
    if (cosO == 0.0f) return 0.0f;
    float dotOH = fabsf(dot(wo, wh));
    return ggxD(g, wh) * ggxG1(g, wo) * dotOH / cosO;
}

// ---------------------------------------------------------------- textures
// checkerboard.h:36-48 / constant.h:19-21
__device__ __forceinline__ V3 evalTex(const ColorTex& t, V2 uv) {
    if (t.kind == 0) return v3(t.v1[0], t.v1[1], t.v1[2]);
    float x = uv.x / t.scale[0], y = uv.y / t.scale[1];
    x -= t.delta[0];
    y -= t.delta[1];
    int s = (int)floorf(x), tt = (int)floorf(y);
    return ((s + tt) % 2 == 0) ? v3(t.v1[0], t.v1[1], t.v1[2]) : v3(t.v2[0], t.v2[1], t.v2[2]);
}

// ---------------------------------------------------------------- BxDF lobes
enum BxDFBits : uint32_t {
    kRefl = 1, kTrans = 2, kDiffuse = 4, kGlossy = 8, kSpecular = 16
};

// One material instance at a shading point (every in-scope material builds one lobe).
struct Lobe {
    uint32_t kind;      // 0 Lambertian, 1 SpecularReflection(conductor), 2 FresnelSpecular,
                        // 3 MicrofacetReflection(conductor), 4 MicrofacetFresnel,
                        // 5 SmoothPlastic, 6 RoughPlastic
    V3 a, b;            // R / Kd | T / Ks
    V3 ceta, ck;        // conductor eta, k
    float eta;          // glass / plastic eta
    Ggx ggx;
};

__device__ __forceinline__ V3 condFresnel(const Lobe& l, float c) {
    return v3(frConductorChannel(c, 1.0f, l.ceta.x, l.ck.x), frConductorChannel(c, 1.0f, l.ceta.y, l.ck.y),
              frConductorChannel(c, 1.0f, l.ceta.z, l.ck.z));
}

// reflection.cpp:103-121
__device__ __forceinline__ V3 mfReflF(const Lobe& l, V3 wo, V3 wi) {
    if (wo.z * wi.z <= 0.0f) return v3s(0.f);
    float cosO = fabsf(wo.z), cosI = fabsf(wi.z);
    if (cosO == 0.0f || cosI == 0.0f) return v3s(0.f);
    V3 wh = wo + wi;
    if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return v3s(0.f);
    wh = normalize(wh);
    if (wh.z < 0.0f) wh = -wh;
    if (dot(wo, wh) * wo.z < 0.0f || dot(wi, wh) * wi.z < 0.0f) return v3s(0.f);
    V3 F = condFresnel(l, dot(wi, wh));
    float D = ggxD(l.ggx, wh);
    float G = ggxG(l.ggx, wo, wi);
    return cdiv(((l.a * D) * G) * F, 4.0f * cosI * cosO);
}
// reflection.cpp:140-146
__device__ __forceinline__ float mfReflPdf(const Lobe& l, V3 wo, V3 wi) {
    if (wo.z * wi.z <= 0.0f) return 0.0f;
    V3 wh = normalize(wo + wi);
    if (wh.z < 0.0f) wh = -wh;
    return ggxPdf(l.ggx, wo, wh) / (4.0f * dot(wo, wh));
}
// reflection.cpp:151-191
__device__ __forceinline__ V3 mfFresF(const Lobe& l, V3 wo, V3 wi) {
    bool reflect = wo.z * wi.z > 0.0f;
    bool entering = wo.z > 0.0f;
    float etaI = entering ? 1.0f : l.eta;
    float etaT = entering ? l.eta : 1.0f;
    V3 wh = reflect ? normalize(wo + wi) : normalize(wo * etaI + wi * etaT);
    if (wh.z * wo.z < 0.0f) wh = -wh;
    float dotO = dot(wo, wh), dotI = dot(wi, wh);
    if (reflect) {
        if (dotO <= 0.0f || dotI <= 0.0f) return v3s(0.f);
    } else {
        if (dotO <= 0.0f || dotI >= 0.0f) return v3s(0.f);
    }
    float F = frDielectric(dotO, etaI, etaT);
    float D = ggxD(l.ggx, wh);
    float G = ggxG(l.ggx, wo, wi);
    if (reflect) return cdiv(((l.a * D) * G) * F, 4.0f * fabsf(wo.z * wi.z));
    if (dotO * dotI > 0.0f) return v3s(0.f);
    float denom = (etaI * dotO + etaT * dotI);
    denom *= denom;
    float factor = fabsf(dotO * dotI) / fabsf(wo.z * wi.z);
    return cdiv(((((l.b * factor) * (etaI * etaI)) * D) * G) * (1.0f - F), denom);
}
// reflection.cpp:227-253
__device__ __forceinline__ float mfFresPdf(const Lobe& l, V3 wo, V3 wi) {
    bool reflect = wo.z * wi.z > 0.0f;
    bool entering = wo.z > 0.0f;
    float etaI = entering ? 1.0f : l.eta;
    float etaT = entering ? l.eta : 1.0f;
    V3 wh = reflect ? normalize(wo + wi) : normalize(wo * etaI + wi * etaT);
    if (wh.z * wo.z < 0.0f) wh = -wh;
    float dotO = dot(wo, wh), dotI = dot(wi, wh);
    float F = frDielectric(dotO, etaI, etaT);
    float pwh = ggxPdf(l.ggx, wo, wh);
    if (reflect) return F * pwh / (4.0f * fabsf(dotO));
    if (dotO * dotI > 0.0f) return 0.0f;
    float denom = (etaI * dotO + etaT * dotI);
    float dwh = (etaT * etaT * fabsf(dotI)) / (denom * denom);
    return (1.0f - F) * pwh * dwh;
}
// reflection.cpp:258-264
__device__ __forceinline__ V3 smoothPlasticF(const Lobe& l, V3 wo, V3 wi) {
    if (wo.z < kEpsilon || wi.z < kEpsilon) return v3s(0.f);
    float Fo = frDielectric(wo.z, 1.0f, l.eta), Fi = frDielectric(wi.z, 1.0f, l.eta);
    return ((l.a * kInvPiD) * (1.0f - Fo)) * (1.0f - Fi);
}
// reflection.cpp:295-313
__device__ __forceinline__ V3 roughPlasticF(const Lobe& l, V3 wo, V3 wi) {
    if (wo.z < kEpsilon || wi.z < kEpsilon) return v3s(0.f);
    float Fo = frDielectric(wo.z, 1.0f, l.eta), Fi = frDielectric(wi.z, 1.0f, l.eta);
    V3 diffuse = ((l.a * kInvPiD) * (1.0f - Fo)) * (1.0f - Fi);
    V3 wh = normalize(wo + wi);
    if (wh.z < 0.0f) wh = -wh;
    if (dot(wo, wh) * wo.z < 0.0f || dot(wi, wh) * wi.z < 0.0f) return v3s(0.f);
    float Fh = frDielectric(dot(wo, wh), 1.0f, l.eta);
    float D = ggxD(l.ggx, wh);
    float G = ggxG(l.ggx, wo, wi);
    V3 spec = cdiv(((l.b * D) * G) * Fh, 4.0f * wo.z * wi.z);
    return diffuse + spec;
}
// reflection.cpp:337-348
__device__ __forceinline__ float roughPlasticPdf(const Lobe& l, V3 wo, V3 wi) {
    if (wo.z < kEpsilon || wi.z < kEpsilon) return 0.0f;
    V3 wh = normalize(wo + wi);
    if (wh.z < 0.0f) wh = -wh;
    float ps = frDielectric(wo.z, 1.0f, l.eta);
    float pdfSpec = ggxPdf(l.ggx, wo, wh) / (4.0f * dot(wo, wh));
    float pdfDiff = cosineHemispherePdf(wi);
    return ps * pdfSpec + (1.0f - ps) * pdfDiff;
}

// Lobe kinds a kernel may meet, as a bitmask over Lobe::kind. Kernels specialised to one
// material class pass its mask so the other lobes' code is not compiled in.
constexpr uint32_t kLobesAll = 0x7Fu;
constexpr uint32_t kLobesNone = 0u;   // the medium-only shade kernel: no surface lobes
constexpr uint32_t kLobesMatte = 1u << 0;
constexpr uint32_t kLobesConductor = (1u << 1) | (1u << 3);
constexpr uint32_t kLobesGlass = (1u << 2) | (1u << 4);
constexpr uint32_t kLobesPlastic = (1u << 5) | (1u << 6);

// BxDF::f in the local frame
template <uint32_t M = kLobesAll>
__device__ __forceinline__ V3 lobeF(const Lobe& l, V3 wo, V3 wi) {
    if ((M & (1u << 0)) && l.kind == 0) return l.a * kInvPi;              // reflection.cpp:8-10
    if ((M & (1u << 3)) && l.kind == 3) return mfReflF(l, wo, wi);
    if ((M & (1u << 4)) && l.kind == 4) return mfFresF(l, wo, wi);
    if ((M & (1u << 5)) && l.kind == 5) return smoothPlasticF(l, wo, wi);
    if ((M & (1u << 6)) && l.kind == 6) return roughPlasticF(l, wo, wi);
    return v3s(0.f);                                                      // delta lobes
}
// BxDF::pdf in the local frame
template <uint32_t M = kLobesAll>
__device__ __forceinline__ float lobePdf(const Lobe& l, V3 wo, V3 wi) {
    if ((M & (1u << 0)) && l.kind == 0) return cosineHemispherePdf(wi);
    if ((M & (1u << 3)) && l.kind == 3) return mfReflPdf(l, wo, wi);
    if ((M & (1u << 4)) && l.kind == 4) return mfFresPdf(l, wo, wi);
    if ((M & (1u << 5)) && l.kind == 5) {                                 // reflection.cpp:286-290
        if (wo.z < kEpsilon || wi.z < kEpsilon) return 0.0f;
        float Fo = frDielectric(wo.z, 1.0f, l.eta);
        return (1.0f - Fo) * cosineHemispherePdf(wi);
    }
    if ((M & (1u << 6)) && l.kind == 6) return roughPlasticPdf(l, wo, wi);
    return 0.0f;
}
// BxDF::sample in the local frame. Returns f; pdf left untouched on the paths where the
// reference leaves it unwritten (caller initialises it to 0).
template <uint32_t M = kLobesAll>
__device__ __forceinline__ V3 lobeSample(const Lobe& l, V3 wo, V3& wi, V2 u, float uc, float& pdf, uint32_t& type) {
    const uint32_t kind = l.kind;
    {
        if ((M & (1u << 0)) && kind == 0) {   // reflection.cpp:12-27
            if (wo.z <= 0.0f) { pdf = 0.0f; return v3s(0.f); }
            wi = squareToCosineHemisphere(u);
            pdf = cosineHemispherePdf(wi);
            type = kRefl | kDiffuse;
            return l.a * kInvPi;
        }
        if ((M & (1u << 1)) && kind == 1) {   // reflection.cpp:40-47
            wi = v3(-wo.x, -wo.y, wo.z);
            pdf = 1.0f;
            type = kRefl | kSpecular;
            return l.a * condFresnel(l, wo.z);
        }
        if ((M & (1u << 2)) && kind == 2) {   // reflection.cpp:61-93
            float F = frDielectric(wo.z, 1.0f, l.eta);
            if (u.x < F) {
                wi = v3(-wo.x, -wo.y, wo.z);
                type = kSpecular | kRefl;
                pdf = F;
                return l.a * F;
            }
            bool entering = wo.z > 0;
            float etaI = entering ? 1.0f : l.eta;
            float etaT = entering ? l.eta : 1.0f;
            V3 n = v3(0.f, 0.f, entering ? 1.f : -1.f);
            V3 wr;
            if (!refract(wo, n, etaI / etaT, wr)) return v3s(0.f);
            wi = wr;
            type = kSpecular | kTrans;
            pdf = 1.f - F;
            float r = etaI / etaT;
            return ((l.b * r) * r) * (1.0f - F);
        }
        if ((M & (1u << 3)) && kind == 3) {   // reflection.cpp:123-138
            if (fabsf(wo.z) < kEpsilon) { pdf = 0.0f; return v3s(0.f); }
            V3 wh = ggxSampleWh(l.ggx, wo, u);
            float dotO = dot(wo, wh);
            if (dotO <= 0.0f) { pdf = 0.0f; return v3s(0.f); }
            wi = -wo + (wh * 2.0f) * dotO;
            if (wo.z * wi.z <= 0.0f) { pdf = 0.0f; return v3s(0.f); }
            pdf = mfReflPdf(l, wo, wi);
            type = kRefl | kGlossy;
            return mfReflF(l, wo, wi);
        }
        if ((M & (1u << 4)) && kind == 4) {   // reflection.cpp:193-225
            if (fabsf(wo.z) < kEpsilon) return v3s(0.f);
            bool entering = wo.z > 0.0f;
            float etaI = entering ? 1.0f : l.eta;
            float etaT = entering ? l.eta : 1.0f;
            V3 wh = ggxSampleWh(l.ggx, wo, u);
            float dotO = dot(wo, wh);
            if (dotO <= 0.0f) { pdf = 0.0f; return v3s(0.f); }
            float F = frDielectric(dotO, etaI, etaT);
            if (uc < F) {
                wi = -wo + (wh * 2.0f) * dotO;
                if (wo.z * wi.z <= 0.0f) { pdf = 0.0f; return v3s(0.f); }
                type = kRefl | kGlossy;
            } else {
                if (!refract(wo, wh, etaI / etaT, wi)) { pdf = 0.0f; return v3s(0.f); }
                if (wo.z * wi.z > 0.0f) { pdf = 0.0f; return v3s(0.f); }
                type = kTrans | kGlossy;
            }
            pdf = mfFresPdf(l, wo, wi);
            return mfFresF(l, wo, wi);
        }
        if ((M & (1u << 5)) && kind == 5) {   // reflection.cpp:266-284
            if (wo.z < kEpsilon) { pdf = 0.0f; return v3s(0.f); }
            float ps = frDielectric(wo.z, 1.0f, l.eta);
            if (uc < ps) {
                wi = v3(-wo.x, -wo.y, wo.z);
                pdf = ps;
                type = kRefl | kSpecular;
                return l.b;
            }
            wi = squareToCosineHemisphere(u);
            if (wi.z < kEpsilon) { pdf = 0.0f; return v3s(0.f); }
            pdf = (1.0f - ps) * cosineHemispherePdf(wi);
            type = kRefl | kDiffuse;
            return smoothPlasticF(l, wo, wi);
        }
        if ((M & (1u << 6)) && kind == 6) {  // reflection.cpp:315-335
            if (wo.z < kEpsilon) { pdf = 0.0f; return v3s(0.f); }
            float ps = frDielectric(wo.z, 1.0f, l.eta);
            if (uc < ps) {
                V3 wh = ggxSampleWh(l.ggx, wo, u);
                float dotO = dot(wo, wh);
                if (dotO <= 0.0f) { pdf = 0.0f; return v3s(0.f); }
                wi = -wo + (wh * 2.0f) * dotO;
                if (wi.z < kEpsilon) { pdf = 0.0f; return v3s(0.f); }
                type = kRefl | kGlossy;
            } else {
                wi = squareToCosineHemisphere(u);
                if (wi.z < kEpsilon) { pdf = 0.0f; return v3s(0.f); }
                type = kRefl | kDiffuse;
            }
            pdf = roughPlasticPdf(l, wo, wi);
            return roughPlasticF(l, wo, wi);
        }
    }
    pdf = 0.0f;
    return v3s(0.f);
}

// Material -> lobe at a shading point (matte.cpp:46-53, plastic.cpp:74-91,
// conductor.cpp:101-120, glass.cpp:98-115). Returns false for the index material.
// `tex` evaluates a color slot at the point; with TexF::kTrees it also evaluates the
// roughness / eta / k trees (tex.node(root)), else those fields are the constants.
template <uint32_t M, class TexF>
__device__ __forceinline__ bool makeLobeT(const Material& m, const TexF& tex, Lobe& l) {
    float rough = m.roughness;
    if (TexF::kTrees && m.roughTex) rough = tex.node(m.roughTex - 1).x;
    switch (m.type) {
        case kMatMatte:
            if (!(M & kLobesMatte)) return false;
            l.kind = 0;
            l.a = tex(m.a);
            return true;
        case kMatPlastic:
            if (!(M & kLobesPlastic)) return false;
            l.a = tex(m.a);
            l.b = tex(m.b);
            l.eta = (TexF::kTrees && m.etaTex) ? tex.node(m.etaTex - 1).x : m.eta;
            if (rough == 0.0f) l.kind = 5;
            else { l.kind = 6; l.ggx = makeGgx(roughnessToAlpha(rough)); }
            return true;
        case kMatConductor:
            if (!(M & kLobesConductor)) return false;
            l.a = tex(m.a);
            l.ceta = (TexF::kTrees && m.etaTex) ? tex.node(m.etaTex - 1) : v3(m.condEta[0], m.condEta[1], m.condEta[2]);
            l.ck = (TexF::kTrees && m.kTex) ? tex.node(m.kTex - 1) : v3(m.condK[0], m.condK[1], m.condK[2]);
            if (rough == 0.0f) l.kind = 1;
            else { l.kind = 3; l.ggx = makeGgx(roughnessToAlpha(rough)); }
            return true;
        case kMatGlass:
            if (!(M & kLobesGlass)) return false;
            l.a = tex(m.a);
            l.b = tex(m.b);
            l.eta = (TexF::kTrees && m.etaTex) ? tex.node(m.etaTex - 1).x : m.eta;
            if (rough == 0.0f) l.kind = 2;
            else { l.kind = 4; l.ggx = makeGgx(roughnessToAlpha(rough)); }
            return true;
        default:
            return false;
    }
}
// Color slots by uv only (constant and checkerboard), constant roughness / eta / k.
struct SlotTexUV {
    static constexpr bool kTrees = false;
    V2 uv;
    __device__ __forceinline__ V3 operator()(const ColorTex& t) const { return evalTex(t, uv); }
    __device__ __forceinline__ V3 node(uint32_t) const { return v3s(0.0f); }
};
template <uint32_t M = kLobesAll>
__device__ __forceinline__ bool makeLobe(const Material& m, V2 uv, Lobe& l) {
    return makeLobeT<M>(m, SlotTexUV{uv}, l);
}

// BSDF with one lobe of weight 1 (bsdf.cpp:6-136): world-space evaluation.
struct Bsdf {
    Frame fr;
    Lobe lobe;
};
__device__ __forceinline__ Frame shadingFrame(V3 n, V3 dpdu) {
    Frame f;
    f.x = dpdu;
    f.y = normalize(cross(n, dpdu));
    f.z = n;
    return f;
}
// bsdf.cpp:19-31
template <uint32_t M = kLobesAll>
__device__ __forceinline__ V3 bsdfF(const Bsdf& b, V3 woW, V3 wiW) {
    V3 wo = toLocal(b.fr, woW), wi = toLocal(b.fr, wiW);
    if (wo.z == 0.0f) return v3s(0.f);
    return v3s(0.f) + lobeF<M>(b.lobe, wo, wi);
}
// bsdf.cpp:109-136 (one lobe: probability weight 1/1)
template <uint32_t M = kLobesAll>
__device__ __forceinline__ float bsdfPdf(const Bsdf& b, V3 woW, V3 wiW) {
    V3 wo = toLocal(b.fr, woW), wi = toLocal(b.fr, wiW);
    if (wo.z == 0.0f) return 0.0f;
    return 0.0f + (1.0f / 1.0f) * lobePdf<M>(b.lobe, wo, wi);
}
// bsdf.cpp:33-107 (one lobe; selectedProb = 1). Returns f*|cos|/pdf. When the reference
// returns early without writing *pdf the value passed in is kept.
template <uint32_t M = kLobesAll>
__device__ __forceinline__ V3 bsdfSample(const Bsdf& b, V3 woW, V3& wiW, V2 u, float uc, float& pdfOut, uint32_t& type) {
    V3 wo = toLocal(b.fr, woW);
    if (wo.z == 0.0f) return v3s(0.f);
    V3 wi = v3s(0.f);
    float lp = 0.0f;
    type = 0;
    V3 f = lobeSample<M>(b.lobe, wo, wi, u, uc, lp, type);
    wiW = toWorld(b.fr, wi);
    if (lp == 0.0f || isBlack(f)) { pdfOut = 0.0f; return v3s(0.f); }
    if (type & kSpecular) {
        pdfOut = lp * 1.0f;
        return cdiv(f, pdfOut);
    }
    float tp = lp * 1.0f;
    pdfOut = tp;
    if (tp < kEpsilon) return v3s(0.f);
    return cdiv(f * fabsf(wi.z), tp);
}

// ---------------------------------------------------------------- phase function
// phase.h:40-93 (sampling inverts with 1-g+2g*u while p() evaluates with +2g*cos)
__device__ __forceinline__ float hgClampG(float g) { return clampf(g, -0.999f, 0.999f); }
__device__ __forceinline__ float phaseHG(float cosTheta, float g) {
    float denom = 1.0f + g * g + 2.0f * g * cosTheta;
    return kInv4Pi * (1.0f - g * g) / (denom * sqrtf(denom));
}
__device__ __forceinline__ float hgSample(float g, V3 wo, V3& wi, V2 u) {
    float cosT;
    if (fabsf(g) < 1e-3f) {
        cosT = 1.0f - 2.0f * u.x;
    } else {
        float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u.x);
        cosT = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    float sinT = sqrtf(fmaxf_(0.0f, 1.0f - cosT * cosT));
    float phi = (float)(2.0 * kPiD * (double)u.y);
    V3 v2;
    if (fabsf(wo.x) > fabsf(wo.y)) {
        float il = 1.0f / sqrtf(wo.x * wo.x + wo.z * wo.z);
        v2 = v3(-wo.z * il, 0.0f, wo.x * il);
    } else {
        float il = 1.0f / sqrtf(wo.y * wo.y + wo.z * wo.z);
        v2 = v3(0.0f, wo.z * il, -wo.y * il);
    }
    V3 v3_ = cross(wo, v2);
    wi = (v2 * (sinT * cosf(phi)) + v3_ * (sinT * sinf(phi))) + wo * cosT;
    return phaseHG(cosT, g);
}

// ---------------------------------------------------------------- media
// homogeneous.cpp:22-30
__device__ __forceinline__ V3 mediumTr(const Medium& m, float tmax) {
    if (isinf(tmax)) return v3s(0.0f);
    return v3(expf(-m.sigT[0] * tmax), expf(-m.sigT[1] * tmax), expf(-m.sigT[2] * tmax));
}

// ---------------------------------------------------------------- power heuristic
__device__ __forceinline__ float powerHeuristic(float fPdf, float gPdf) {
    float f = 1 * fPdf, g = 1 * gPdf;
    float denom = (f * f) + (g * g);
    return denom > 0.0f ? (f * f) / denom : 0.0f;
}

}  // namespace gnd
