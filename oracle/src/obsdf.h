// Oracle (test infrastructure only): Fresnel terms, GGX microfacet distribution,
// BxDF lobes and the BSDF container of the reference, restated on the CPU.
#pragma once
#include "omath.h"
#include "osampling.h"
#include <cstddef>
#include <new>
#include <vector>

namespace orc {

// arena.h:10-118 (bump allocator reset once per camera sample)
class Arena {
public:
    explicit Arena(size_t bytes = 1 << 16) : m_buf(bytes) {}
    template <typename T, typename... A>
    T* create(A&&... a) {
        size_t align = alignof(T);
        size_t off = (m_off + align - 1) & ~(align - 1);
        if (off + sizeof(T) > m_buf.size()) { m_extra.emplace_back(sizeof(T) + align); return new (align_ptr(m_extra.back().data(), align)) T(static_cast<A&&>(a)...); }
        m_off = off + sizeof(T);
        return new (m_buf.data() + off) T(static_cast<A&&>(a)...);
    }
    void reset() { m_off = 0; m_extra.clear(); }
private:
    static void* align_ptr(unsigned char* p, size_t a) { return (void*)(((uintptr_t)p + a - 1) & ~(uintptr_t)(a - 1)); }
    std::vector<unsigned char> m_buf;
    std::vector<std::vector<unsigned char>> m_extra;
    size_t m_off = 0;
};

// bxdf.h:7-15
enum BxDFType {
    BSDF_REFLECTION = 1 << 0,
    BSDF_TRANSMISSION = 1 << 1,
    BSDF_DIFFUSE = 1 << 2,
    BSDF_GLOSSY = 1 << 3,
    BSDF_SPECULAR = 1 << 4,
    BSDF_ALL = 31
};

// fresnel.h:13-40
float FrDielectric(float cosThetaI, float etaExt, float etaInt);
// fresnel.h:47-58
bool Refract(const Vec3& wi, const Vec3& n, float eta, Vec3* wt);
// fresnel.h:111-140 (one channel)
float FrConductorChannel(float cosThetaI, float etaI, float etaT, float k);

struct Fresnel {
    virtual ~Fresnel() = default;
    virtual Color evaluate(float cosThetaI) const = 0;
};
struct FresnelNoOp : Fresnel {
    Color evaluate(float) const override { return Color(1.f); }
};
struct FresnelConductor : Fresnel {
    Color etaI, etaT, k;
    FresnelConductor(const Color& a, const Color& b, const Color& c) : etaI(a), etaT(b), k(c) {}
    Color evaluate(float c) const override {
        return Color(FrConductorChannel(c, etaI.r, etaT.r, k.r), FrConductorChannel(c, etaI.g, etaT.g, k.g),
                     FrConductorChannel(c, etaI.b, etaT.b, k.b));
    }
};

// microfacet.h:26-29
inline float roughnessToAlpha(float r) { r = std::max(r, 1e-3f); return r * r; }

// microfacet.cpp:7-66 (isotropic Trowbridge-Reitz; alpha clamped to 1e-4)
struct TrowbridgeReitz {
    float ax, ay;
    explicit TrowbridgeReitz(float a) : ax(std::max(1e-4f, a)), ay(std::max(1e-4f, a)) {}
    float D(const Vec3& wh) const;
    float G1(const Vec3& w) const;
    float G(const Vec3& wo, const Vec3& wi) const { return G1(wo) * G1(wi); }
    Vec3 sample_wh(const Vec3& wo, const Vec2& u) const;
    float pdf(const Vec3& wo, const Vec3& wh) const;
};

struct BxDF {
    const BxDFType type;
    explicit BxDF(BxDFType t) : type(t) {}
    virtual ~BxDF() = default;
    bool matchesFlags(BxDFType t) const { return (type & t) == type; }
    virtual Color f(const Vec3& wo, const Vec3& wi) const = 0;
    virtual Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const = 0;
    virtual float pdf(const Vec3& wo, const Vec3& wi) const = 0;
};

// reflection.cpp:8-31
struct Lambertian : BxDF {
    Color R;
    explicit Lambertian(const Color& r) : BxDF(BxDFType(BSDF_REFLECTION | BSDF_DIFFUSE)), R(r) {}
    Color f(const Vec3&, const Vec3&) const override { return R * InvPi; }
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3&, const Vec3& wi) const override { return warp::squareToCosineHemispherePdf(wi); }
};
// reflection.cpp:36-52
struct SpecularReflection : BxDF {
    Color R; const Fresnel* fr;
    SpecularReflection(const Color& r, const Fresnel* f) : BxDF(BxDFType(BSDF_REFLECTION | BSDF_SPECULAR)), R(r), fr(f) {}
    Color f(const Vec3&, const Vec3&) const override { return Color(0.f); }
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3&, const Vec3&) const override { return 0.f; }
};
// transmission.cpp:10-39
struct SpecularTransmission : BxDF {
    Color T; float etaExt, etaInt;
    SpecularTransmission(const Color& t, float a, float b) : BxDF(BxDFType(BSDF_TRANSMISSION | BSDF_SPECULAR)), T(t), etaExt(a), etaInt(b) {}
    Color f(const Vec3&, const Vec3&) const override { return Color(0.f); }
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3&, const Vec3&) const override { return 0.f; }
};
// reflection.cpp:57-98
struct FresnelSpecular : BxDF {
    Color R, T; float etaExt, etaInt;
    FresnelSpecular(const Color& r, const Color& t, float a, float b)
        : BxDF(BxDFType(BSDF_REFLECTION | BSDF_TRANSMISSION | BSDF_SPECULAR)), R(r), T(t), etaExt(a), etaInt(b) {}
    Color f(const Vec3&, const Vec3&) const override { return Color(0.f); }
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3&, const Vec3&) const override { return 0.f; }
};
// reflection.cpp:103-146
struct MicrofacetReflection : BxDF {
    Color R; const TrowbridgeReitz* dist; const Fresnel* fr;
    MicrofacetReflection(const Color& r, const TrowbridgeReitz* d, const Fresnel* f)
        : BxDF(BxDFType(BSDF_REFLECTION | BSDF_GLOSSY)), R(r), dist(d), fr(f) {}
    Color f(const Vec3& wo, const Vec3& wi) const override;
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3& wo, const Vec3& wi) const override;
};
// reflection.cpp:151-253
struct MicrofacetFresnel : BxDF {
    Color R, T; float etaExt, etaInt; const TrowbridgeReitz* dist;
    MicrofacetFresnel(const Color& r, const Color& t, float a, float b, const TrowbridgeReitz* d)
        : BxDF(BxDFType(BSDF_REFLECTION | BSDF_TRANSMISSION | BSDF_GLOSSY)), R(r), T(t), etaExt(a), etaInt(b), dist(d) {}
    Color f(const Vec3& wo, const Vec3& wi) const override;
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3& wo, const Vec3& wi) const override;
};
// reflection.cpp:258-290
struct SmoothPlastic : BxDF {
    Color Kd, Ks; float eta;
    SmoothPlastic(const Color& kd, const Color& ks, float e) : BxDF(BxDFType(BSDF_REFLECTION | BSDF_DIFFUSE | BSDF_SPECULAR)), Kd(kd), Ks(ks), eta(e) {}
    Color f(const Vec3& wo, const Vec3& wi) const override;
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3& wo, const Vec3& wi) const override;
};
// reflection.cpp:295-348
struct RoughPlastic : BxDF {
    Color Kd, Ks; float eta; const TrowbridgeReitz* dist;
    RoughPlastic(const Color& kd, const Color& ks, float e, const TrowbridgeReitz* d)
        : BxDF(BxDFType(BSDF_REFLECTION | BSDF_DIFFUSE | BSDF_GLOSSY)), Kd(kd), Ks(ks), eta(e), dist(d) {}
    Color f(const Vec3& wo, const Vec3& wi) const override;
    Color sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const override;
    float pdf(const Vec3& wo, const Vec3& wi) const override;
};

// bsdf.cpp:6-136; bsdf.h:58-111
class BSDF {
public:
    BSDF(const Vec3& n, const Vec3& dpdu, float eta = 1.0f);
    void add(BxDF* b, float w = 1.0f) { if (m_n < 8) { m_b[m_n] = b; m_w[m_n] = w; ++m_n; } }
    int numComponents(BxDFType flags = BSDF_ALL) const;
    Color f(const Vec3& woW, const Vec3& wiW, BxDFType flags = BSDF_ALL) const;
    Color sample(const Vec3& woW, Vec3* wiW, const Vec2& u, float uc, float* pdf, BxDFType* st, BxDFType type = BSDF_ALL) const;
    float pdf(const Vec3& woW, const Vec3& wiW, BxDFType flags = BSDF_ALL) const;
    const float eta;
    Frame frame;
private:
    int m_n = 0;
    BxDF* m_b[8];
    float m_w[8];
};

// phase.h:40-93 (Henyey-Greenstein, g clamped to (-0.999, 0.999))
struct HGPhase {
    float g;
    explicit HGPhase(float g_) : g(std::clamp(g_, -0.999f, 0.999f)) {}
    static float phaseHG(float cosTheta, float g) {
        float denom = 1.0f + g * g + 2.0f * g * cosTheta;
        return Inv4Pi * (1.0f - g * g) / (denom * std::sqrt(denom));
    }
    float p(const Vec3& wo, const Vec3& wi) const { return phaseHG(Dot(wo, wi), g); }
    float sample(const Vec3& wo, Vec3* wi, const Vec2& u) const;
};

}  // namespace orc
