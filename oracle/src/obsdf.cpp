// Oracle (test infrastructure only): BxDF lobes, Fresnel, GGX and the BSDF container.
// Each function restates the reference function cited beside it, in the same
// operation order.
#include "obsdf.h"

namespace orc {

// fresnel.h:13-40
float FrDielectric(float cosThetaI, float etaExt, float etaInt) {
    if (etaExt == etaInt) return 0.0f;
    cosThetaI = std::clamp(cosThetaI, -1.f, 1.f);
    if (cosThetaI < 0.f) {
        std::swap(etaExt, etaInt);
        cosThetaI = -cosThetaI;
    }
    float sinThetaI = std::sqrt(std::max(0.f, 1.f - cosThetaI * cosThetaI));
    float sinThetaT = etaExt / etaInt * sinThetaI;
    if (sinThetaT >= 1.f) return 1.f;
    float cosThetaT = std::sqrt(std::max(0.f, 1.f - sinThetaT * sinThetaT));
    float rParl = ((etaInt * cosThetaI) - (etaExt * cosThetaT)) / ((etaInt * cosThetaI) + (etaExt * cosThetaT));
    float rPerp = ((etaExt * cosThetaI) - (etaInt * cosThetaT)) / ((etaExt * cosThetaI) + (etaInt * cosThetaT));
    return (rParl * rParl + rPerp * rPerp) / 2.f;
}

// fresnel.h:47-58
bool Refract(const Vec3& wi, const Vec3& n, float eta, Vec3* wt) {
    float cosThetaI = Dot(n, wi);
    float sin2ThetaI = std::max(0.f, 1.f - cosThetaI * cosThetaI);
    float sin2ThetaT = eta * eta * sin2ThetaI;
    if (sin2ThetaT >= 1.f) return false;
    float cosThetaT = std::sqrt(1.f - sin2ThetaT);
    *wt = -wi * eta + n * (eta * cosThetaI - cosThetaT);
    return true;
}

// fresnel.h:111-133
float FrConductorChannel(float cosThetaI, float eta_i, float eta_t, float k_c) {
    float cosThetaI2 = cosThetaI * cosThetaI;
    float sinThetaI2 = std::max(0.0f, 1.f - cosThetaI2);
    float eta = eta_t / eta_i;
    float etak = k_c / eta_i;
    float eta2 = eta * eta;
    float etak2 = etak * etak;
    float t0 = eta2 - etak2 - sinThetaI2;
    float a2plusb2 = std::sqrt(t0 * t0 + 4.f * eta2 * etak2);
    float t1 = a2plusb2 + cosThetaI2;
    float a = std::sqrt(std::max(0.0f, 0.5f * (a2plusb2 + t0)));
    float t2 = 2.f * std::abs(cosThetaI) * a;
    float Rs = (t1 - t2) / (t1 + t2);
    float t3 = cosThetaI2 * a2plusb2 + sinThetaI2 * sinThetaI2;
    float t4 = t2 * sinThetaI2;
    float Rp = Rs * (t3 - t4) / (t3 + t4);
    return 0.5f * (Rp + Rs);
}

// microfacet.cpp:7-15
float TrowbridgeReitz::D(const Vec3& wh) const {
    if (std::abs(wh.z) < Epsilon) return 0.0f;
    float d = (wh.x * wh.x) / (ax * ax) + (wh.y * wh.y) / (ay * ay) + (wh.z * wh.z);
    return 1.0f / (Pi * ax * ay * d * d);
}
// microfacet.cpp:17-24
float TrowbridgeReitz::G1(const Vec3& w) const {
    if (std::abs(w.z) < Epsilon) return 0.0f;
    float a2tan2 = (w.x * w.x * ax * ax + w.y * w.y * ay * ay) / (w.z * w.z);
    float lambda = 0.5f * (-1.0f + std::sqrt(1.0f + a2tan2));
    return 1.0f / (1.0f + lambda);
}
// microfacet.cpp:30-56 (visible-normal sampling)
Vec3 TrowbridgeReitz::sample_wh(const Vec3& wo, const Vec2& u) const {
    bool flip = wo.z < 0.0f;
    Vec3 wo_h = flip ? -wo : wo;
    Vec3 Vh = Normalize(Vec3(ax * wo_h.x, ay * wo_h.y, wo_h.z));
    float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    Vec3 T1 = lensq > 0.0f ? Vec3(-Vh.y, Vh.x, 0.0f) / std::sqrt(lensq) : Vec3(1.0f, 0.0f, 0.0f);
    Vec3 T2 = Cross(Vh, T1);
    float r = std::sqrt(u.x);
    float phi = 2.0f * Pi * u.y;
    float t1 = r * std::cos(phi);
    float t2 = r * std::sin(phi);
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * std::sqrt(std::max(0.0f, 1.0f - t1 * t1)) + s * t2;
    Vec3 Nh = (T1 * t1 + T2 * t2) + Vh * std::sqrt(std::max(0.0f, 1.0f - t1 * t1 - t2 * t2));
    Vec3 wh = Normalize(Vec3(ax * Nh.x, ay * Nh.y, std::max(0.0f, Nh.z)));
    if (flip) wh = -wh;
    return wh;
}
// microfacet.cpp:58-66
float TrowbridgeReitz::pdf(const Vec3& wo, const Vec3& wh) const {
    if (wo.z * wh.z < 0.0f) return 0.0f;
    float cosThetaO = std::abs(wo.z);
    if (cosThetaO == 0.0f) return 0.0f;
    float dotOH = std::abs(Dot(wo, wh));
    return D(wh) * G1(wo) * dotOH / cosThetaO;
}

// reflection.cpp:12-27
Color Lambertian::sample(const Vec3& wo, Vec3& wi, const Vec2& u, float, float& pdf, BxDFType* st) const {
    if (wo.z <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
    wi = warp::squareToCosineHemisphere(u);
    pdf = warp::squareToCosineHemispherePdf(wi);
    if (st) *st = type;
    return R * InvPi;
}

// reflection.cpp:40-47
Color SpecularReflection::sample(const Vec3& wo, Vec3& wi, const Vec2&, float, float& pdf, BxDFType* st) const {
    wi = Vec3(-wo.x, -wo.y, wo.z);
    pdf = 1.0f;
    if (st) *st = type;
    return R * fr->evaluate(wo.z);
}

// transmission.cpp:10-34
Color SpecularTransmission::sample(const Vec3& wo, Vec3& wi, const Vec2&, float, float& pdf, BxDFType* st) const {
    bool entering = wo.z > 0;
    float etaI = entering ? etaExt : etaInt;
    float etaT = entering ? etaInt : etaExt;
    Vec3 n(0, 0, entering ? 1.f : -1.f);
    float etaRatio = etaI / etaT;
    Vec3 wr;
    if (!Refract(wo, n, etaRatio, &wr)) return Color(0.f);
    wi = wr;
    pdf = 1.f;
    Color ft = T * (1.f - FrDielectric(wo.z, etaExt, etaInt));
    if (st) *st = type;
    ft *= (etaRatio * etaRatio);
    return ft;
}

// reflection.cpp:61-93
Color FresnelSpecular::sample(const Vec3& wo, Vec3& wi, const Vec2& u, float, float& pdf, BxDFType* st) const {
    float F = FrDielectric(wo.z, etaExt, etaInt);
    if (u.x < F) {
        wi = Vec3(-wo.x, -wo.y, wo.z);
        if (st) *st = BxDFType(BSDF_SPECULAR | BSDF_REFLECTION);
        pdf = F;
        return R * F;
    }
    bool entering = wo.z > 0;
    float etaI = entering ? etaExt : etaInt;
    float etaT = entering ? etaInt : etaExt;
    Vec3 n(0, 0, entering ? 1.f : -1.f);
    Vec3 wr;
    if (!Refract(wo, n, etaI / etaT, &wr)) return Color(0.f);
    wi = wr;
    if (st) *st = BxDFType(BSDF_SPECULAR | BSDF_TRANSMISSION);
    pdf = 1.f - F;
    float etaRatio = etaI / etaT;
    return T * etaRatio * etaRatio * (1.0f - F);
}

// reflection.cpp:103-121
Color MicrofacetReflection::f(const Vec3& wo, const Vec3& wi) const {
    if (wo.z * wi.z <= 0.0f) return Color(0.0f);
    float cosThetaO = std::abs(wo.z), cosThetaI = std::abs(wi.z);
    if (cosThetaO == 0.0f || cosThetaI == 0.0f) return Color(0.0f);
    Vec3 wh = wo + wi;
    if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return Color(0.0f);
    wh = Normalize(wh);
    if (wh.z < 0.0f) wh = -wh;
    if (Dot(wo, wh) * wo.z < 0.0f || Dot(wi, wh) * wi.z < 0.0f) return Color(0.0f);
    Color F = fr->evaluate(Dot(wi, wh));
    float D = dist->D(wh);
    float G = dist->G(wo, wi);
    return R * D * G * F / (4.0f * cosThetaI * cosThetaO);
}
// reflection.cpp:123-138
Color MicrofacetReflection::sample(const Vec3& wo, Vec3& wi, const Vec2& u, float, float& pdf, BxDFType* st) const {
    if (std::abs(wo.z) < Epsilon) { pdf = 0.0f; return Color(0.0f); }
    Vec3 wh = dist->sample_wh(wo, u);
    float dotO = Dot(wo, wh);
    if (dotO <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
    wi = -wo + wh * 2.0f * dotO;
    if (wo.z * wi.z <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
    pdf = this->pdf(wo, wi);
    if (st) *st = type;
    return f(wo, wi);
}
// reflection.cpp:140-146
float MicrofacetReflection::pdf(const Vec3& wo, const Vec3& wi) const {
    if (wo.z * wi.z <= 0.0f) return 0.0f;
    Vec3 wh = Normalize(wo + wi);
    if (wh.z < 0.0f) wh = -wh;
    return dist->pdf(wo, wh) / (4.0f * Dot(wo, wh));
}

// reflection.cpp:151-191
Color MicrofacetFresnel::f(const Vec3& wo, const Vec3& wi) const {
    bool reflect = (wo.z * wi.z > 0.0f);
    bool entering = wo.z > 0.0f;
    float etaI = entering ? etaExt : etaInt;
    float etaT = entering ? etaInt : etaExt;
    Vec3 wh = reflect ? Normalize(wo + wi) : Normalize(wo * etaI + wi * etaT);
    if (wh.z * wo.z < 0.0f) wh = -wh;
    float dotO = Dot(wo, wh);
    float dotI = Dot(wi, wh);
    if (reflect) {
        if (dotO <= 0.0f || dotI <= 0.0f) return Color(0.0f);
    } else {
        if (dotO <= 0.0f || dotI >= 0.0f) return Color(0.0f);
    }
    float F = FrDielectric(dotO, etaI, etaT);
    float D = dist->D(wh);
    float G = dist->G(wo, wi);
    if (reflect) return R * D * G * F / (4.0f * std::abs(wo.z * wi.z));
    if (dotO * dotI > 0.0f) return Color(0.0f);
    float denom = (etaI * dotO + etaT * dotI);
    denom *= denom;
    float factor = std::abs(dotO * dotI) / std::abs(wo.z * wi.z);
    return T * factor * (etaI * etaI) * D * G * (1.0f - F) / denom;
}
// reflection.cpp:193-225
Color MicrofacetFresnel::sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const {
    if (std::abs(wo.z) < Epsilon) return Color(0.0f);
    bool entering = wo.z > 0.0f;
    float etaI = entering ? etaExt : etaInt;
    float etaT = entering ? etaInt : etaExt;
    Vec3 wh = dist->sample_wh(wo, u);
    float dotO = Dot(wo, wh);
    if (dotO <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
    float F = FrDielectric(dotO, etaI, etaT);
    if (uc < F) {
        wi = -wo + wh * 2.0f * dotO;
        if (wo.z * wi.z <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
        if (st) *st = BxDFType(BSDF_REFLECTION | BSDF_GLOSSY);
    } else {
        if (!Refract(wo, wh, etaI / etaT, &wi)) { pdf = 0.0f; return Color(0.0f); }
        if (wo.z * wi.z > 0.0f) { pdf = 0.0f; return Color(0.0f); }
        if (st) *st = BxDFType(BSDF_TRANSMISSION | BSDF_GLOSSY);
    }
    pdf = this->pdf(wo, wi);
    return f(wo, wi);
}
// reflection.cpp:227-253
float MicrofacetFresnel::pdf(const Vec3& wo, const Vec3& wi) const {
    bool reflect = (wo.z * wi.z > 0.0f);
    bool entering = wo.z > 0.0f;
    float etaI = entering ? etaExt : etaInt;
    float etaT = entering ? etaInt : etaExt;
    Vec3 wh = reflect ? Normalize(wo + wi) : Normalize(wo * etaI + wi * etaT);
    if (wh.z * wo.z < 0.0f) wh = -wh;
    float dotO = Dot(wo, wh);
    float dotI = Dot(wi, wh);
    float F = FrDielectric(dotO, etaI, etaT);
    float pdf_wh = dist->pdf(wo, wh);
    if (reflect) return F * pdf_wh / (4.0f * std::abs(dotO));
    if (dotO * dotI > 0.0f) return 0.0f;
    float denom = (etaI * dotO + etaT * dotI);
    float dwh_dwi = (etaT * etaT * std::abs(dotI)) / (denom * denom);
    return (1.0f - F) * pdf_wh * dwh_dwi;
}

static const float kInvPiF = (float)M_1_PI;

// reflection.cpp:258-264
Color SmoothPlastic::f(const Vec3& wo, const Vec3& wi) const {
    if (wo.z < Epsilon || wi.z < Epsilon) return Color(0.0f);
    float Fo = FrDielectric(wo.z, 1.0f, eta);
    float Fi = FrDielectric(wi.z, 1.0f, eta);
    return Kd * kInvPiF * (1.0f - Fo) * (1.0f - Fi);
}
// reflection.cpp:266-284
Color SmoothPlastic::sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const {
    if (wo.z < Epsilon) { pdf = 0.0f; return Color(0.0f); }
    float probSpec = FrDielectric(wo.z, 1.0f, eta);
    if (uc < probSpec) {
        wi = Vec3(-wo.x, -wo.y, wo.z);
        pdf = probSpec;
        if (st) *st = BxDFType(BSDF_REFLECTION | BSDF_SPECULAR);
        return Ks;
    }
    wi = warp::squareToCosineHemisphere(u);
    if (wi.z < Epsilon) { pdf = 0.0f; return Color(0.0f); }
    pdf = (1.0f - probSpec) * warp::squareToCosineHemispherePdf(wi);
    if (st) *st = BxDFType(BSDF_REFLECTION | BSDF_DIFFUSE);
    return f(wo, wi);
}
// reflection.cpp:286-290
float SmoothPlastic::pdf(const Vec3& wo, const Vec3& wi) const {
    if (wo.z < Epsilon || wi.z < Epsilon) return 0.0f;
    float Fo = FrDielectric(wo.z, 1.0f, eta);
    return (1.0f - Fo) * warp::squareToCosineHemispherePdf(wi);
}

// reflection.cpp:295-313
Color RoughPlastic::f(const Vec3& wo, const Vec3& wi) const {
    if (wo.z < Epsilon || wi.z < Epsilon) return Color(0.0f);
    float Fo = FrDielectric(wo.z, 1.0f, eta);
    float Fi = FrDielectric(wi.z, 1.0f, eta);
    Color diffuse = Kd * kInvPiF * (1.0f - Fo) * (1.0f - Fi);
    Vec3 wh = Normalize(wo + wi);
    if (wh.z < 0.0f) wh = -wh;
    if (Dot(wo, wh) * wo.z < 0.0f || Dot(wi, wh) * wi.z < 0.0f) return Color(0.0f);
    float Fh = FrDielectric(Dot(wo, wh), 1.0f, eta);
    float D = dist->D(wh);
    float G = dist->G(wo, wi);
    Color specular = Ks * D * G * Fh / (4.0f * wo.z * wi.z);
    return diffuse + specular;
}
// reflection.cpp:315-335
Color RoughPlastic::sample(const Vec3& wo, Vec3& wi, const Vec2& u, float uc, float& pdf, BxDFType* st) const {
    if (wo.z < Epsilon) { pdf = 0.0f; return Color(0.0f); }
    float probSpec = FrDielectric(wo.z, 1.0f, eta);
    if (uc < probSpec) {
        Vec3 wh = dist->sample_wh(wo, u);
        float dotO = Dot(wo, wh);
        if (dotO <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
        wi = -wo + wh * 2.0f * dotO;
        if (wi.z < Epsilon) { pdf = 0.0f; return Color(0.0f); }
        if (st) *st = BxDFType(BSDF_REFLECTION | BSDF_GLOSSY);
    } else {
        wi = warp::squareToCosineHemisphere(u);
        if (wi.z < Epsilon) { pdf = 0.0f; return Color(0.0f); }
        if (st) *st = BxDFType(BSDF_REFLECTION | BSDF_DIFFUSE);
    }
    pdf = this->pdf(wo, wi);
    return f(wo, wi);
}
// reflection.cpp:337-348
float RoughPlastic::pdf(const Vec3& wo, const Vec3& wi) const {
    if (wo.z < Epsilon || wi.z < Epsilon) return 0.0f;
    Vec3 wh = Normalize(wo + wi);
    if (wh.z < 0.0f) wh = -wh;
    float probSpec = FrDielectric(wo.z, 1.0f, eta);
    float pdfSpec = dist->pdf(wo, wh) / (4.0f * Dot(wo, wh));
    float pdfDiff = warp::squareToCosineHemispherePdf(wi);
    return probSpec * pdfSpec + (1.0f - probSpec) * pdfDiff;
}

// bsdf.cpp:6-10
BSDF::BSDF(const Vec3& n, const Vec3& dpdu, float e) : eta(e) {
    Vec3 bitangent = Normalize(Cross(n, dpdu));
    frame = Frame(dpdu, bitangent, n);
}
// bsdf.cpp:12-17
int BSDF::numComponents(BxDFType flags) const {
    int num = 0;
    for (int i = 0; i < m_n; ++i) if (m_b[i]->matchesFlags(flags)) num++;
    return num;
}
// bsdf.cpp:19-31
Color BSDF::f(const Vec3& woW, const Vec3& wiW, BxDFType flags) const {
    Vec3 wo = frame.toLocal(woW), wi = frame.toLocal(wiW);
    if (wo.z == 0.0f) return Color(0.0f);
    Color result(0.0f);
    for (int i = 0; i < m_n; ++i) if (m_b[i]->matchesFlags(flags)) result += m_b[i]->f(wo, wi);
    return result;
}
// bsdf.cpp:33-107 (a zero wo.z returns black without writing *pdf, as the reference does)
Color BSDF::sample(const Vec3& woW, Vec3* wiW, const Vec2& u, float uc, float* pdf, BxDFType* st, BxDFType type) const {
    int matching = numComponents(type);
    if (matching == 0) { *pdf = 0.0f; return Color(0.0f); }
    float wsum = 0.0f;
    for (int i = 0; i < m_n; ++i) if (m_b[i]->matchesFlags(type)) wsum += m_w[i];
    if (wsum == 0.0f) { *pdf = 0.0f; return Color(0.0f); }
    BxDF* bxdf = nullptr;
    float cdf = 0.0f, selectedProb = 0.0f;
    for (int i = 0; i < m_n; ++i) {
        if (m_b[i]->matchesFlags(type)) {
            float prob = m_w[i] / wsum;
            cdf += prob;
            if (uc <= cdf || i == m_n - 1) { bxdf = m_b[i]; selectedProb = prob; break; }
        }
    }
    Vec3 wo = frame.toLocal(woW);
    if (wo.z == 0.0f) return Color(0.0f);
    Vec3 wi;
    float lobePdf = 0.0f;
    BxDFType lobeType = BxDFType(0);
    Color fv = bxdf->sample(wo, wi, u, uc, lobePdf, &lobeType);
    *wiW = frame.toWorld(wi);
    if (st) *st = lobeType;
    if (lobePdf == 0.0f || fv.isBlack()) { *pdf = 0.0f; return Color(0.0f); }
    if (lobeType & BSDF_SPECULAR) {
        *pdf = lobePdf * selectedProb;
        return fv / *pdf;
    }
    Color total_f = fv;
    float total_pdf = lobePdf * selectedProb;
    if (matching > 1) {
        total_f = this->f(woW, *wiW, type);
        total_pdf = this->pdf(woW, *wiW, type);
    }
    *pdf = total_pdf;
    if (total_pdf < Epsilon) return Color(0.0f);
    return total_f * std::abs(wi.z) / total_pdf;
}
// bsdf.cpp:109-136
float BSDF::pdf(const Vec3& woW, const Vec3& wiW, BxDFType flags) const {
    int matching = numComponents(flags);
    if (matching == 0) return 0.0f;
    Vec3 wo = frame.toLocal(woW), wi = frame.toLocal(wiW);
    if (wo.z == 0.0f) return 0.0f;
    float wsum = 0.0f;
    for (int i = 0; i < m_n; ++i) if (m_b[i]->matchesFlags(flags)) wsum += m_w[i];
    if (wsum == 0.0f) return 0.0f;
    float s = 0.0f;
    for (int i = 0; i < m_n; ++i)
        if (m_b[i]->matchesFlags(flags)) s += (m_w[i] / wsum) * m_b[i]->pdf(wo, wi);
    return s;
}

// phase.h:84-107 (sampling uses the 1-g+2g*u inversion while p() evaluates with +2g*cos;
// the restatement keeps both as written)
float HGPhase::sample(const Vec3& wo, Vec3* wi, const Vec2& u) const {
    float cosTheta;
    if (std::abs(g) < 1e-3f) {
        cosTheta = 1.0f - 2.0f * u.x;
    } else {
        float sqrTerm = (1.0f - g * g) / (1.0f - g + 2.0f * g * u.x);
        cosTheta = (1.0f + g * g - sqrTerm * sqrTerm) / (2.0f * g);
    }
    float sinTheta = std::sqrt(std::max(0.0f, 1.0f - cosTheta * cosTheta));
    float phi = (float)(2.0f * M_PI * u.y);
    Vec3 v2, v3;
    if (std::abs(wo.x) > std::abs(wo.y)) {
        float invLen = 1.0f / std::sqrt(wo.x * wo.x + wo.z * wo.z);
        v2 = Vec3(-wo.z * invLen, 0.0f, wo.x * invLen);
    } else {
        float invLen = 1.0f / std::sqrt(wo.y * wo.y + wo.z * wo.z);
        v2 = Vec3(0.0f, wo.z * invLen, -wo.y * invLen);
    }
    v3 = Cross(wo, v2);
    *wi = (v2 * (sinTheta * std::cos(phi)) + v3 * (sinTheta * std::sin(phi))) + wo * cosTheta;
    return phaseHG(cosTheta, g);
}

}  // namespace orc
