// Oracle (test infrastructure only): plugin objects of the reference (materials,
// textures, media, emitters, camera, film, filters, scene) and the name registry,
// restated on the CPU.
#include "oscene.h"
#include "otextures.h"
#include <algorithm>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <iterator>
#include <limits>

namespace orc {

const char* classTypeName(ClassType t) {
    switch (t) {
        case EScene: return "scene"; case EPrimitive: return "primitive"; case EShape: return "shape";
        case ECamera: return "camera"; case EIntegrator: return "integrator"; case ESampler: return "sampler";
        case ETexture: return "texture"; case EMaterial: return "material"; case EEmitter: return "emitter";
        case EFilter: return "filter"; case EMedium: return "medium";
    }
    return "unknown";
}

// ---------------------------------------------------------------- textures
// constant.h:9-32
template <typename T>
struct ConstantTexture : Texture<T> {
    T value;
    explicit ConstantTexture(const PropertyList& p) {
        if constexpr (std::is_same_v<T, float>) value = p.getFloat("value", 1.0f);
        else value = p.getColor("value", Color(1.0f));
    }
    T evaluate(const SurfaceInteraction&) const override { return value; }
};
// checkerboard.h:20-48
template <typename T>
struct CheckerTexture : Texture<T> {
    T v1, v2;
    Vec2 scale, delta;
    explicit CheckerTexture(const PropertyList& p) {
        if constexpr (std::is_same_v<T, float>) { v1 = p.getFloat("value1", 1.0f); v2 = p.getFloat("value2", 0.0f); }
        else { v1 = p.getColor("value1", Color(1.0f)); v2 = p.getColor("value2", Color(0.0f)); }
        scale = p.getVector2("scale", Vec2(1.0f, 1.0f));
        delta = p.getPoint2("delta", Vec2(0.0f, 0.0f));
    }
    T evaluate(const SurfaceInteraction& si) const override {
        Vec2 uv = si.uv;
        uv.x /= scale.x; uv.y /= scale.y;
        uv.x -= delta.x; uv.y -= delta.y;
        int s = (int)std::floor(uv.x), t = (int)std::floor(uv.y);
        return ((s + t) % 2 == 0) ? v1 : v2;
    }
};

template <typename T>
static std::shared_ptr<Texture<T>> constTex(const T& v) {
    PropertyList p;
    if constexpr (std::is_same_v<T, float>) p.f["value"] = v; else p.c["value"] = v;
    return std::make_shared<ConstantTexture<T>>(p);
}
// matte.cpp:33-43, area.cpp:31-43: the "missing texture" magenta checkerboard
static std::shared_ptr<ColorTexture> missingTex() {
    PropertyList p;
    p.c["value1"] = Color(0.0f);
    p.c["value2"] = Color(1.0f, 0.0f, 1.0f);
    p.v2["scale"] = Vec2(0.1f, 0.1f);
    return std::make_shared<CheckerTexture<Color>>(p);
}

// ---------------------------------------------------------------- materials
// material.h:36-59
void Material::addChild(ObjectPtr child) {
    if (child->classType() == ETexture && child->name == "normal") {
        if (normalMap) throw std::runtime_error("Material: normal map already defined!");
        normalMap = std::static_pointer_cast<Texture<Color>>(child);
    } else if (child->classType() == ETexture && child->name == "bump") {
        if (bumpMap) throw std::runtime_error("Material: bump map already defined!");
        bumpMap = std::static_pointer_cast<Texture<float>>(child);
    } else if (child->classType() == EMedium && child->name == "inside") {
        if (inside) throw std::runtime_error("Material: inside medium already defined!");
        inside = std::static_pointer_cast<Medium>(child);
    } else if (child->classType() == EMedium && child->name == "outside") {
        if (outside) throw std::runtime_error("Material: outside medium already defined!");
        outside = std::static_pointer_cast<Medium>(child);
    } else {
        throw std::runtime_error("Material: cannot add specified child (" + child->name + ")!");
    }
}

// material.h:71-117: the normal map replaces n by its (x, y, z) in the (dpdu, n x dpdu, n)
// frame; the bump map tilts dpdu and dpdv by the height's forward differences (steps of
// 0.001 along dpdu / dpdv in p and along u / v); dpdu is re-orthogonalised either way.
void Material::applyNormalOrBump(SurfaceInteraction& si) const {
    if (normalMap) {
        Color nm = normalMap->evaluate(si);
        Vec3 dpdv = Normalize(Cross(si.n, si.dpdu));
        Vec3 pn = si.dpdu * nm.r + dpdv * nm.g + si.n * nm.b;
        si.n = Normalize(pn);
        Vec3 nd = si.dpdu - si.n * Dot(si.n, si.dpdu);
        si.dpdu = Normalize(nd);
    } else if (bumpMap) {
        Vec3 dpdu = si.dpdu;
        Vec3 dpdv = Normalize(Cross(si.n, dpdu));
        const float du = 0.001f, dv = 0.001f;
        float hBase = bumpMap->evaluate(si);
        SurfaceInteraction sDu = si;
        sDu.p = si.p + dpdu * du;
        sDu.uv.x += du;
        float hDu = bumpMap->evaluate(sDu);
        SurfaceInteraction sDv = si;
        sDv.p = si.p + dpdv * dv;
        sDv.uv.y += dv;
        float hDv = bumpMap->evaluate(sDv);
        float dhdu = (hDu - hBase) / du;
        float dhdv = (hDv - hBase) / dv;
        dhdu *= bumpScale;
        dhdv *= bumpScale;
        Vec3 ndu = dpdu + si.n * dhdu;
        Vec3 ndv = dpdv + si.n * dhdv;
        si.n = Normalize(Cross(ndu, ndv));
        Vec3 proj = ndu - si.n * Dot(si.n, ndu);
        si.dpdu = Normalize(proj);
    }
}

template <typename T>
static void setTex(std::shared_ptr<Texture<T>>& slot, ObjectPtr child) {
    slot = std::static_pointer_cast<Texture<T>>(child);
}

// matte.cpp:7-53
struct Matte : Material {
    std::shared_ptr<ColorTexture> albedo;
    explicit Matte(const PropertyList& p) {
        bumpScale = p.getFloat("bump_scale", 1.0f);
        if (p.hasColor("albedo")) albedo = constTex(p.getColor("albedo"));
    }
    void addChild(ObjectPtr c) override {
        if (c->classType() != ETexture) throw std::runtime_error("Matte: cannot add specified child!");
        if (c->name == "albedo") { if (albedo) throw std::runtime_error("Matte: there's already an albedo defined!"); setTex(albedo, c); }
        else Material::addChild(c);
    }
    void activate() override { if (!albedo) albedo = missingTex(); }
    void computeScatteringFunctions(SurfaceInteraction& si, Arena& a) const override {
        applyNormalOrBump(si);
        si.bsdf = a.create<BSDF>(si.n, si.dpdu);
        si.bsdf->add(a.create<Lambertian>(albedo->evaluate(si)));
    }
};
// plastic.cpp:8-91
struct Plastic : Material {
    std::shared_ptr<ColorTexture> Kd, Ks;
    std::shared_ptr<FloatTexture> rough, eta;
    explicit Plastic(const PropertyList& p) {
        bumpScale = p.getFloat("bump_scale", 1.0f);
        if (p.hasColor("Kd")) Kd = constTex(p.getColor("Kd"));
        if (p.hasColor("Ks")) Ks = constTex(p.getColor("Ks"));
        if (p.hasFloat("roughness")) rough = constTex(p.getFloat("roughness"));
        if (p.hasFloat("eta")) eta = constTex(p.getFloat("eta"));
    }
    void addChild(ObjectPtr c) override {
        if (c->classType() != ETexture) return;
        if (c->name == "Kd") setTex(Kd, c); else if (c->name == "Ks") setTex(Ks, c);
        else if (c->name == "roughness") setTex(rough, c); else if (c->name == "eta") setTex(eta, c);
        else Material::addChild(c);
    }
    void activate() override {
        if (!Kd) Kd = constTex(Color(0.25f));
        if (!Ks) Ks = constTex(Color(0.25f));
        if (!rough) rough = constTex(0.1f);
        if (!eta) eta = constTex(1.5f);
    }
    void computeScatteringFunctions(SurfaceInteraction& si, Arena& a) const override {
        applyNormalOrBump(si);
        Color kd = Kd->evaluate(si), ks = Ks->evaluate(si);
        float r = rough->evaluate(si), e = eta->evaluate(si);
        si.bsdf = a.create<BSDF>(si.n, si.dpdu);
        if (r == 0.0f) si.bsdf->add(a.create<SmoothPlastic>(kd, ks, e));
        else si.bsdf->add(a.create<RoughPlastic>(kd, ks, e, a.create<TrowbridgeReitz>(roughnessToAlpha(r))));
    }
};
// conductor.cpp:9-120
struct Conductor : Material {
    std::shared_ptr<ColorTexture> R, eta, k;
    std::shared_ptr<FloatTexture> rough;
    explicit Conductor(const PropertyList& p) {
        bumpScale = p.getFloat("bump_scale", 1.0f);
        if (p.hasColor("R")) R = constTex(p.getColor("R"));
        if (p.hasColor("eta")) eta = constTex(p.getColor("eta"));
        if (p.hasColor("k")) k = constTex(p.getColor("k"));
        if (p.hasFloat("roughness")) rough = constTex(p.getFloat("roughness"));
    }
    void addChild(ObjectPtr c) override {
        if (c->classType() != ETexture) throw std::runtime_error("Conductor: cannot add specified child!");
        if (c->name == "R") setTex(R, c); else if (c->name == "eta") setTex(eta, c);
        else if (c->name == "k") setTex(k, c); else if (c->name == "roughness") setTex(rough, c);
        else Material::addChild(c);
    }
    void activate() override {
        if (!R) R = constTex(Color(1.0f));
        if (!eta) eta = constTex(Color(1.0f));
        if (!k) k = constTex(Color(1.0f));
        if (!rough) rough = constTex(0.0f);
    }
    void computeScatteringFunctions(SurfaceInteraction& si, Arena& a) const override {
        applyNormalOrBump(si);
        Color r = R->evaluate(si), e = eta->evaluate(si), kk = k->evaluate(si);
        float ro = rough->evaluate(si);
        si.bsdf = a.create<BSDF>(si.n, si.dpdu);
        Fresnel* fr = a.create<FresnelConductor>(Color(1.0f), e, kk);
        if (ro == 0.0f) si.bsdf->add(a.create<SpecularReflection>(r, fr));
        else si.bsdf->add(a.create<MicrofacetReflection>(r, a.create<TrowbridgeReitz>(roughnessToAlpha(ro)), fr));
    }
};
// glass.cpp:8-115
struct Glass : Material {
    std::shared_ptr<ColorTexture> R, T;
    std::shared_ptr<FloatTexture> rough, eta;
    explicit Glass(const PropertyList& p) {
        bumpScale = p.getFloat("bump_scale", 1.0f);
        if (p.hasColor("R")) R = constTex(p.getColor("R"));
        if (p.hasColor("T")) T = constTex(p.getColor("T"));
        if (p.hasFloat("roughness")) rough = constTex(p.getFloat("roughness"));
        if (p.hasFloat("eta")) eta = constTex(p.getFloat("eta"));
    }
    void addChild(ObjectPtr c) override {
        if (c->name == "R") setTex(R, c); else if (c->name == "T") setTex(T, c);
        else if (c->name == "roughness") setTex(rough, c); else if (c->name == "eta") setTex(eta, c);
        else Material::addChild(c);
    }
    void activate() override {
        if (!R) R = constTex(Color(1.0f));
        if (!T) T = constTex(Color(1.0f));
        if (!rough) rough = constTex(0.0f);
        if (!eta) eta = constTex(1.5f);
    }
    void computeScatteringFunctions(SurfaceInteraction& si, Arena& a) const override {
        applyNormalOrBump(si);
        applyMediums(si);
        Color r = R->evaluate(si), t = T->evaluate(si);
        float e = eta->evaluate(si), ro = rough->evaluate(si);
        si.bsdf = a.create<BSDF>(si.n, si.dpdu);
        if (ro == 0.0f) si.bsdf->add(a.create<FresnelSpecular>(r, t, 1.0f, e));
        else si.bsdf->add(a.create<MicrofacetFresnel>(r, t, 1.0f, e, a.create<TrowbridgeReitz>(roughnessToAlpha(ro))));
    }
};
// index.cpp:6-16 (null BSDF: a pass-through medium boundary)
struct IndexMaterial : Material {
    explicit IndexMaterial(const PropertyList& p) { bumpScale = p.getFloat("bump_scale", 1.0f); }
    void computeScatteringFunctions(SurfaceInteraction& si, Arena&) const override {
        applyNormalOrBump(si);
        applyMediums(si);
        si.bsdf = nullptr;
    }
};

// ---------------------------------------------------------------- media
// homogeneous.cpp:14-20
HomogeneousMedium::HomogeneousMedium(const PropertyList& p) {
    sigma_a = p.getColor("sigma_a", Color(0.1f));
    sigma_s = p.getColor("sigma_s", Color(0.1f));
    g = p.getFloat("g", 0.0f);
    sigma_t = sigma_a + sigma_s;
}
// homogeneous.cpp:22-30
Color HomogeneousMedium::Tr(const Ray& ray) const {
    if (std::isinf(ray.tMax)) return Color(0.0f);
    return Color(std::exp(-sigma_t.r * ray.tMax), std::exp(-sigma_t.g * ray.tMax), std::exp(-sigma_t.b * ray.tMax));
}
// homogeneous.cpp:32-63
Color HomogeneousMedium::sample(const Ray& ray, Sampler& s, Arena& a, MediumInteraction& mi) const {
    float u0 = s.next1D();
    float u1 = s.next1D();
    return sampleU(ray, u0, u1, a, mi);
}
Color HomogeneousMedium::sampleU(const Ray& ray, float u0, float u1, Arena& a, MediumInteraction& mi) const {
    int channel = std::min((int)(u0 * 3.0f), 2);
    float dist = -std::log(1.0f - u1) / sigma_t[channel];
    float t = std::min(dist, ray.tMax);
    bool sampledMedium = t < ray.tMax;
    Color Trv(std::exp(-sigma_t.r * t), std::exp(-sigma_t.g * t), std::exp(-sigma_t.b * t));
    Color pc = sampledMedium ? (sigma_t * Trv) : Trv;
    float pdf = (pc.r + pc.g + pc.b) / 3.0f;
    if (pdf == 0.0f) return Color(0.0f);
    if (sampledMedium) {
        mi.p = ray.o + ray.d * t;
        mi.wo = -ray.d;
        mi.medium = this;
        mi.phase = a.create<HGPhase>(g);
        mi.sigma_a = sigma_a;
        mi.sigma_s = sigma_s;
    }
    return Trv / pdf;
}

// ---------------------------------------------------------------- emitters
// area.cpp:7-119
struct AreaLight : Emitter {
    std::shared_ptr<ColorTexture> radiance;
    explicit AreaLight(const PropertyList& p) { if (p.hasColor("radiance")) radiance = constTex(p.getColor("radiance")); }
    void addChild(ObjectPtr c) override {
        if (c->classType() != ETexture) throw std::runtime_error("AreaLight: cannot add specified child!");
        if (c->name == "radiance") { if (radiance) throw std::runtime_error("AreaLight: radiance already defined!"); setTex(radiance, c); }
    }
    void activate() override { if (!radiance) radiance = missingTex(); }
    // area.cpp:45-49
    Color eval(const SurfaceInteraction& si, const Vec3& w) const override {
        if (Dot(si.n, w) > 0.0f) return radiance->evaluate(si);
        return Color(0.0f);
    }
    // area.cpp:51-88 (pdf is left unwritten on the early return, as in the reference)
    Color sample(const SurfaceInteraction& ref, const Vec2& u, SurfaceInteraction& info, float& pdf, Ray& sr) const override {
        SurfaceInteraction local;
        const Transform tw = prim->getToWorld(ref.time);   // area.cpp:54
        float areaPdf = prim->shape->sampleSurface(ref.p, u, local);
        info.p = tw.point(local.p);
        info.n = Normalize(tw.normal(local.n));
        info.uv = local.uv;
        info.time = ref.time;
        Frame fr = Frame::fromNormal(local.n);
        Vec3 t1 = tw.vector(fr.x), t2 = tw.vector(fr.y);
        float areaScale = Cross(t1, t2).length();
        if (areaScale > 0.0f) areaPdf /= areaScale;
        sr.o = ref.p;
        sr.d = Normalize(info.p - ref.p);
        sr.tMin = Epsilon;
        sr.tMax = (info.p - ref.p).length() - Epsilon;
        sr.time = ref.time;
        float dist = (ref.p - info.p).lengthSquared();
        Vec3 wi = sr.d;
        float cosTheta = Dot(info.n, -wi);
        if (areaPdf <= Epsilon || cosTheta <= Epsilon) return Color(0.0f);
        float anglePdf = areaPdf * dist / cosTheta;
        pdf = anglePdf;
        return eval(info, Normalize(ref.p - info.p)) / pdf;
    }
    // area.cpp:90-119
    float pdf(const SurfaceInteraction& ref, const SurfaceInteraction& info) const override {
        SurfaceInteraction local;
        const Transform tw = prim->getToWorld(ref.time);   // area.cpp:92
        const Transform tl = tw.inverse();
        local.p = tl.point(info.p);
        local.n = tl.normal(info.n);
        local.uv = info.uv;
        float areaPdf = prim->shape->pdfSurface(tl.point(ref.p), local);
        Frame fr = Frame::fromNormal(local.n);
        Vec3 t1 = tw.vector(fr.x), t2 = tw.vector(fr.y);
        float areaScale = Cross(t1, t2).length();
        if (areaScale > 0.0f) areaPdf /= areaScale;
        float dist = (ref.p - info.p).lengthSquared();
        Vec3 wi = Normalize(info.p - ref.p);
        float cosTheta = Dot(info.n, -wi);
        if (areaPdf <= Epsilon || cosTheta <= Epsilon) return 0.0f;
        return areaPdf * dist / cosTheta;
    }
};

// pointlight.cpp:9-35
struct PointLight : Emitter {
    Vec3 position;
    Color power;
    explicit PointLight(const PropertyList& p)
        : position(PropertyList::get(p.p3, std::string("position"), Vec3(0.0f, 0.0f, 0.0f))), power(p.getColor("power", Color(10.0f))) {}
    bool isDelta() const override { return true; }
    Color eval(const SurfaceInteraction&, const Vec3&) const override { return Color(0.0f); }
    Color sample(const SurfaceInteraction& ref, const Vec2&, SurfaceInteraction& info, float& pdf, Ray& sr) const override {
        Color I = power * Inv4Pi;
        float squaredDist = (position - ref.p).lengthSquared();
        info.p = position;
        pdf = 1.0f;
        sr.o = ref.p;
        sr.d = Normalize(info.p - ref.p);
        sr.tMin = Epsilon;
        sr.tMax = (info.p - ref.p).length() - Epsilon;
        sr.time = info.time;
        return I / squaredDist;
    }
    float pdf(const SurfaceInteraction&, const SurfaceInteraction&) const override { return 0.0f; }
};

// spotlight.cpp:9-64
struct SpotLight : Emitter {
    Vec3 position, direction;
    Color power;
    float cosTotalWidth, cosFalloffStart;
    explicit SpotLight(const PropertyList& p) {
        position = PropertyList::get(p.p3, std::string("position"), Vec3(0.0f, 0.0f, 0.0f));
        direction = Normalize(p.getVector3("direction", Vec3(0.0f, 0.0f, -1.0f)));
        power = p.getColor("power", Color(10.0f));
        float spotSize = p.getFloat("spot_size", 45.0f);
        float blend = p.getFloat("blend", 0.15f);
        float halfAngle = spotSize * 0.5f;
        float innerAngle = halfAngle * (1.0f - blend);
        cosTotalWidth = std::cos((Pi / 180.f) * halfAngle);
        cosFalloffStart = std::cos((Pi / 180.f) * innerAngle);
    }
    bool isDelta() const override { return true; }
    Color eval(const SurfaceInteraction&, const Vec3&) const override { return Color(0.0f); }
    Color sample(const SurfaceInteraction& ref, const Vec2&, SurfaceInteraction& info, float& pdf, Ray& sr) const override {
        Vec3 wi = Normalize(position - ref.p);
        float dist = (position - ref.p).length();
        float squaredDist = dist * dist;
        info.p = position;
        pdf = 1.0f;
        sr.o = ref.p;
        sr.d = wi;
        sr.tMin = Epsilon;
        sr.tMax = dist - Epsilon;
        sr.time = ref.time;
        float cosTheta = Dot(-wi, direction);
        if (cosTheta <= cosTotalWidth) return Color(0.0f);
        float falloff = 1.0f;
        if (cosTheta < cosFalloffStart) {
            float t = (cosTheta - cosTotalWidth) / (cosFalloffStart - cosTotalWidth);
            falloff = (t * t) * (3.0f - 2.0f * t);
        }
        Color I = power * Inv4Pi;
        return (I * falloff) / squaredDist;
    }
    float pdf(const SurfaceInteraction&, const SurfaceInteraction&) const override { return 0.0f; }
};

// directional.cpp:9-38
struct DirectionalLight : Emitter {
    Vec3 direction;   // towards the light
    Color irradiance;
    explicit DirectionalLight(const PropertyList& p) {
        direction = -Normalize(p.getVector3("direction", Vec3(0.0f, -1.0f, 0.0f)));
        irradiance = p.getColor("irradiance", Color(1.0f));
    }
    bool isDelta() const override { return true; }
    Color eval(const SurfaceInteraction&, const Vec3&) const override { return Color(0.0f); }
    Color sample(const SurfaceInteraction& ref, const Vec2&, SurfaceInteraction& info, float& pdf, Ray& sr) const override {
        Vec3 wi = direction;
        info.p = ref.p + wi * 1e5f;
        info.time = ref.time;
        pdf = 1.0f;
        sr.o = ref.p;
        sr.d = wi;
        sr.tMin = Epsilon;
        sr.tMax = std::numeric_limits<float>::max();
        sr.time = ref.time;
        return irradiance;
    }
    float pdf(const SurfaceInteraction&, const SurfaceInteraction&) const override { return 0.0f; }
};

// distribution.cpp:6-81
struct Distribution1D {
    std::vector<float> func, cdf;
    float funcInt = 0.0f;
    Distribution1D(const float* f, int n) : func(f, f + n), cdf(n + 1) {
        cdf[0] = 0.0f;
        for (int i = 1; i < n + 1; ++i) cdf[i] = cdf[i - 1] + func[i - 1] / n;
        funcInt = cdf[n];
        if (funcInt == 0.0f) {
            for (int i = 1; i < n + 1; ++i) cdf[i] = float(i) / float(n);
        } else {
            for (int i = 1; i < n + 1; ++i) cdf[i] /= funcInt;
        }
    }
    int count() const { return (int)func.size(); }
    float sampleContinuous(float u, float* pdf, int* off = nullptr) const {
        auto it = std::upper_bound(cdf.begin(), cdf.end(), u);
        int offset = std::clamp<int>((int)std::distance(cdf.begin(), it) - 1, 0, (int)cdf.size() - 2);
        if (off) *off = offset;
        float du = u - cdf[offset];
        if ((cdf[offset + 1] - cdf[offset]) > 0.0f) du /= (cdf[offset + 1] - cdf[offset]);
        if (pdf) *pdf = (funcInt > 0.0f) ? func[offset] / funcInt : 0.0f;
        return (offset + du) / count();
    }
};
struct Distribution2D {
    std::vector<Distribution1D> cond;
    std::unique_ptr<Distribution1D> marginal;
    Distribution2D(const float* data, int nu, int nv) {
        cond.reserve(nv);
        for (int v = 0; v < nv; ++v) cond.emplace_back(&data[v * nu], nu);
        std::vector<float> m;
        for (int v = 0; v < nv; ++v) m.push_back(cond[v].funcInt);
        marginal = std::make_unique<Distribution1D>(m.data(), nv);
    }
    Vec2 sampleContinuous(const Vec2& u, float* pdf) const {
        float pdfs[2];
        int v;
        float d1 = marginal->sampleContinuous(u.y, &pdfs[1], &v);
        float d0 = cond[v].sampleContinuous(u.x, &pdfs[0]);
        *pdf = pdfs[0] * pdfs[1];
        return Vec2(d0, d1);
    }
    float pdf(const Vec2& p) const {
        int iu = std::clamp<int>((int)(p.x * cond[0].count()), 0, cond[0].count() - 1);
        int iv = std::clamp<int>((int)(p.y * marginal->count()), 0, marginal->count() - 1);
        return cond[iv].func[iu] / marginal->funcInt;
    }
};

// constants.h:80-98
static Vec2 sphericalCoordinates(const Vec3& w) {
    Vec2 r(std::acos(std::clamp(w.z, -1.0f, 1.0f)), std::atan2(w.y, w.x));
    if (r.y < 0.0f) r.y += 2.0f * Pi;
    return r;
}
static Vec3 sphericalDirection(const Vec2& p) {
    float cosTheta = std::cos(p.x), sinTheta = std::sin(p.x), cosPhi = std::cos(p.y), sinPhi = std::sin(p.y);
    return Vec3(sinTheta * cosPhi, sinTheta * sinPhi, cosTheta);
}

// Uncompressed scanline OpenEXR (the images the tests write), channels R, G, B as FLOAT
// or HALF; the reference reads any file through OpenEXR (image2d.h:100-135).
static float halfToFloat(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    const uint32_t e = (h >> 10) & 31, m = h & 1023;
    float v;
    if (e == 0) v = std::ldexp((float)m, -24);
    else if (e == 31) v = m ? std::numeric_limits<float>::quiet_NaN() : std::numeric_limits<float>::infinity();
    else v = std::ldexp((float)(m | 1024), (int)e - 25);
    return sign ? -v : v;
}
void loadEXR(const std::string& path, int& w, int& h, std::vector<Color>& px) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("EnvMap: cannot open " + path);
    std::vector<uint8_t> d((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    auto rd32 = [&](size_t at) { int32_t v; std::memcpy(&v, &d.at(at + 3) - 3, 4); return v; };
    if (d.size() < 8 || rd32(0) != 20000630) throw std::runtime_error("EnvMap: not an OpenEXR file");
    size_t pos = 8;
    auto cstr = [&](size_t& at) { std::string s; while (d.at(at)) s += (char)d[at++]; ++at; return s; };
    std::vector<std::pair<std::string, int>> chans;
    int comp = -1, x0 = 0, y0 = 0, x1 = -1, y1 = -1;
    while (d.at(pos)) {
        std::string name = cstr(pos), type = cstr(pos);
        int32_t n = rd32(pos);
        size_t at = pos + 4;
        if (name == "channels") {
            size_t q = at;
            while (d.at(q)) { std::string c = cstr(q); chans.push_back({c, rd32(q)}); q += 16; }
        } else if (name == "compression") {
            comp = d.at(at);
        } else if (name == "dataWindow") {
            x0 = rd32(at); y0 = rd32(at + 4); x1 = rd32(at + 8); y1 = rd32(at + 12);
        }
        pos = at + n;
    }
    ++pos;
    if (comp != 0) throw std::runtime_error("EnvMap: only uncompressed OpenEXR files are read here");
    w = x1 - x0 + 1;
    h = y1 - y0 + 1;
    if (w <= 0 || h <= 0) throw std::runtime_error("EnvMap: empty image");
    px.assign((size_t)w * h, Color(0.0f));
    size_t lineBytes = 0;
    for (auto& c : chans) lineBytes += (size_t)w * (c.second == 1 ? 2 : 4);
    for (int line = 0; line < h; ++line) {
        uint64_t off;
        std::memcpy(&off, &d.at(pos + 8 * (size_t)line), 8);
        const int y = rd32(off) - y0;
        size_t at = off + 8;
        for (auto& c : chans) {
            const int k = c.first == "R" ? 0 : c.first == "G" ? 1 : c.first == "B" ? 2 : -1;
            const size_t sz = c.second == 1 ? 2 : 4;
            for (int x = 0; x < w; ++x, at += sz) {
                if (k < 0 || y < 0 || y >= h) continue;
                float v;
                if (sz == 4) std::memcpy(&v, &d.at(at), 4);
                else { uint16_t hv; std::memcpy(&hv, &d.at(at), 2); v = halfToFloat(hv); }
                (k == 0 ? px[(size_t)y * w + x].r : k == 1 ? px[(size_t)y * w + x].g : px[(size_t)y * w + x].b) = v;
            }
        }
        (void)lineBytes;
    }
}

// environment.cpp:13-129
struct EnvironmentMap : Emitter {
    std::string relPath, baseDir;
    float strength;
    int width = 0, height = 0;
    std::vector<Color> bitmap;
    std::unique_ptr<Distribution2D> distribution;
    explicit EnvironmentMap(const PropertyList& p) : relPath(p.getString("filename")), strength(p.getFloat("strength", 1.0f)) {}
    void setBaseDir(const std::string& d) override { baseDir = d; }
    void activate() override {
        std::filesystem::path abs = std::filesystem::path(relPath).is_relative() ? std::filesystem::path(baseDir) / relPath : std::filesystem::path(relPath);
        if (!std::filesystem::is_regular_file(abs)) throw std::runtime_error("EnvMap: Invalid environment map path.");
        if (abs.extension() != ".exr") throw std::runtime_error("EnvMap: Invalid environment map extension.");
        loadEXR(abs.string(), width, height, bitmap);
        // buildPDFs (environment.cpp:111-124)
        std::vector<float> img((size_t)width * height);
        for (int i = 0; i < height; i++) {
            float sinTheta = (float)std::sin(M_PI * (i + 0.5f) / height);
            for (int j = 0; j < width; j++) img[(size_t)i * width + j] = bitmap[(size_t)i * width + j].luminance() * sinTheta;
        }
        distribution = std::make_unique<Distribution2D>(img.data(), width, height);
    }
    bool isInfiniteAreaLight() const override { return true; }
    // film.cpp:126-151
    Color pixelBilinear(float u, float v) const {
        float x = u * width - 0.5f, y = v * height - 0.5f;
        int x0 = (int)std::floor(x), y0 = (int)std::floor(y);
        float dx = x - x0, dy = y - y0;
        int px0 = (x0 % width + width) % width;
        int px1 = (px0 + 1) % width;
        int py0 = std::clamp(y0, 0, height - 1), py1 = std::clamp(y0 + 1, 0, height - 1);
        Color c00 = bitmap[(size_t)py0 * width + px0], c10 = bitmap[(size_t)py0 * width + px1];
        Color c01 = bitmap[(size_t)py1 * width + px0], c11 = bitmap[(size_t)py1 * width + px1];
        Color c0 = c00 * (1.0f - dx) + c10 * dx;
        Color c1 = c01 * (1.0f - dx) + c11 * dx;
        return c0 * (1.0f - dy) + c1 * dy;
    }
    Color eval(const SurfaceInteraction&, const Vec3& w) const override {
        Vec2 sph = sphericalCoordinates(w);
        float u = (float)(sph.y * M_1_PI * 0.5f);
        float v = (float)(sph.x * M_1_PI);
        return strength * pixelBilinear(u, v);
    }
    Color sample(const SurfaceInteraction& ref, const Vec2& u, SurfaceInteraction& info, float& pdf, Ray& sr) const override {
        float mapPdf;
        Vec2 uv = distribution->sampleContinuous(u, &mapPdf);
        if (mapPdf == 0.0f) { pdf = 0.0f; return Color(0.0f); }
        float theta = (float)(uv.y * M_PI);
        float phi = (float)(uv.x * 2.0f * M_PI);
        Vec3 wi = sphericalDirection(Vec2(theta, phi));
        info.p = ref.p + wi * 1e5f;
        info.n = -wi;
        info.time = ref.time;
        sr = Ray(ref.p, wi);
        sr.time = ref.time;
        float sinTheta = std::sin(theta);
        if (sinTheta <= 0.0f) { pdf = 0.0f; return Color(0.0f); }
        pdf = (float)(mapPdf / (2.0f * M_PI * M_PI * sinTheta));
        return eval(info, wi) / pdf;
    }
    float pdf(const SurfaceInteraction& ref, const SurfaceInteraction& info) const override {
        Vec3 wi = Normalize(info.p - ref.p);
        Vec2 sph = sphericalCoordinates(wi);
        float sinTheta = std::sin(sph.x);
        if (sinTheta <= 0.0f) return 0.0f;
        float u = (float)(sph.y * M_1_PI * 0.5f);
        float v = (float)(sph.x * M_1_PI);
        float mapPdf = distribution->pdf(Vec2(u, v));
        return (float)(mapPdf / (2.0f * M_PI * M_PI * sinTheta));
    }
};

// ---------------------------------------------------------------- filters, film, camera
// filter.h:20-32
struct BoxFilter : Filter {
    explicit BoxFilter(const PropertyList&) { radius = Vec2(0.5f, 0.5f); }
    float evaluate(const Vec2& p) const override {
        return (std::abs(p.x) <= radius.x && std::abs(p.y) <= radius.y) ? 1.0f : 0.0f;
    }
};
// filter.h:34-54
struct GaussianFilter : Filter {
    float alpha, expX, expY;
    explicit GaussianFilter(const PropertyList& p) {
        radius = p.getVector2("radius", Vec2(2.0f, 2.0f));
        alpha = p.getFloat("alpha", 2.0f);
        expX = std::exp(-alpha * radius.x * radius.x);
        expY = std::exp(-alpha * radius.y * radius.y);
    }
    float evaluate(const Vec2& p) const override {
        float gx = std::max(0.0f, std::exp(-alpha * p.x * p.x) - expX);
        float gy = std::max(0.0f, std::exp(-alpha * p.y * p.y) - expY);
        return gx * gy;
    }
};

Film::Film(int w, int h, std::shared_ptr<Filter> f) : width(w), height(h), filter(f), sum((size_t)w * h * 7) {
    if (!filter) filter = std::make_shared<GaussianFilter>(PropertyList());   // film.cpp:29
    clear();
}
void Film::clear() {
    for (auto& a : sum) a.store(0.0f, std::memory_order_relaxed);
    for (auto& a : fixedSum) a.store(0, std::memory_order_relaxed);
}
void Film::enableFixed() {
    fixedMode = true;
    fixedSum = std::vector<std::atomic<uint64_t>>((size_t)width * height * 4);
    for (auto& a : fixedSum) a.store(0, std::memory_order_relaxed);
}
uint64_t toFixed(float x) {
    x = x > 0.0f ? x : 0.0f;          // NaN -> 0
    x = x < 1e11f ? x : 1e11f;
    return (uint64_t)(int64_t)std::nearbyint(x * 16777216.0f);   // default rounding: nearest even
}
static inline void atomicAddF(std::atomic<float>& t, float v) {
    float cur = t.load(std::memory_order_relaxed);
    while (!t.compare_exchange_weak(cur, cur + v, std::memory_order_release, std::memory_order_relaxed)) {}
}
// film.h:26-69 (radiance channel only)
void Film::addSample(const Vec2& pFilm, const Color& L) {
    if (L.hasNaNs()) return;
    Vec2 r = filter->radius;
    int x0 = std::max(0, (int)std::ceil(pFilm.x - r.x - 0.5f));
    int x1 = std::min(width - 1, (int)std::floor(pFilm.x + r.x - 0.5f));
    int y0 = std::max(0, (int)std::ceil(pFilm.y - r.y - 0.5f));
    int y1 = std::min(height - 1, (int)std::floor(pFilm.y + r.y - 0.5f));
    for (int py = y0; py <= y1; ++py) {
        for (int px = x0; px <= x1; ++px) {
            Vec2 off(pFilm.x - (px + 0.5f), pFilm.y - (py + 0.5f));
            float w = filter->evaluate(off);
            if (w > 0.0f) {
                std::atomic<float>* a = &sum[((size_t)py * width + px) * 7];
                if (fixedMode) {
                    std::atomic<uint64_t>* q = &fixedSum[((size_t)py * width + px) * 4];
                    q[0].fetch_add(toFixed(L.r * w), std::memory_order_relaxed);
                    q[1].fetch_add(toFixed(L.g * w), std::memory_order_relaxed);
                    q[2].fetch_add(toFixed(L.b * w), std::memory_order_relaxed);
                    q[3].fetch_add(toFixed(w), std::memory_order_relaxed);
                } else {
                    atomicAddF(a[0], L.r * w);
                    atomicAddF(a[1], L.g * w);
                    atomicAddF(a[2], L.b * w);
                    atomicAddF(a[3], w);
                }
                atomicAddF(a[4], L.r * L.r * w);
                atomicAddF(a[5], L.g * L.g * w);
                atomicAddF(a[6], L.b * L.b * w);
            }
        }
    }
}

// camera.h:30-52, perspective.cpp:9-12
Camera::Camera(const PropertyList& p, int k) {
    toWorld = p.getTransform("toWorld", Transform());
    anim.set(toWorld, p.getTransform("toWorldEnd", toWorld));   // camera.h:20-25
    width = p.getInteger("width", 1280);
    height = p.getInteger("height", 720);
    fov = p.getFloat("fov", 45.0f);
    scale = std::tan((Pi / 180.f) * (fov * 0.5f));
    kind = k;
    if (kind == 1) {   // thinLens.cpp:13-31
        lensRadius = p.getFloat("lens_radius", 0.0f);
        focalDistance = p.getFloat("focal_distance", 10.0f);
        k1 = p.getFloat("k1", 0.0f);
        caAxial = p.getFloat("ca_axial", 0.0f);
        caLateral = p.getFloat("ca_lateral", 0.0f);
        vignetting = p.getBoolean("vignetting", false);
        blades = p.getInteger("blades", 0);
        rollingShutter = p.getBoolean("rolling_shutter", false);
        scanDuration = p.getFloat("scan_duration", 0.9f);
        exposureDuration = p.getFloat("exposure_duration", 0.1f);
    }
}
void Camera::addChild(ObjectPtr c) {
    if (c->classType() == EFilter) {
        if (filterObj) throw std::runtime_error("Camera: cannot define multiple films!");
        filterObj = std::static_pointer_cast<Filter>(c);
    }
}
// perspective.cpp:15-32
float Camera::shootRay(const CameraSample& s, Ray* ray) const {
    if (kind == 0) {   // perspective.cpp:15-32
        float x = (2.0f * s.pFilm.x - 1.0f) * aspect() * scale;
        float y = (2.0f * s.pFilm.y - 1.0f) * scale;
        Vec3 dir = Normalize(Vec3(x, y, -1.0f));
        Ray rc(Vec3(0, 0, 0), dir);
        *ray = anim.interpolate(s.time).ray(rc);
        ray->time = s.time;
        return 1.0f;
    }
    // thinLens.cpp:33-91: barrel distortion, lateral / axial chromatic aberration, depth
    // of field through a disk or polygon aperture, vignetting, rolling shutter
    float ndcX = 2.0f * s.pFilm.x - 1.0f;
    float ndcY = 2.0f * s.pFilm.y - 1.0f;
    float r2 = ndcX * ndcX + ndcY * ndcY;
    float distortion = 1.0f + k1 * r2;
    float distX = ndcX * distortion;
    float distY = ndcY * distortion;
    float scaleMod = scale * (1.0f + caLateral * s.lambdaOffset);
    float x = distX * aspect() * scaleMod;
    float y = distY * scaleMod;
    Vec3 dir(x, y, -1.0f);
    Vec3 rayOrigin(0.0f, 0.0f, 0.0f);
    if (lensRadius > 0.0f) {
        Vec2 pl = blades >= 3 ? warp::squareToUniformPolygon(s.pLens, blades) : warp::squareToUniformDisk(s.pLens);
        Vec2 pLens(pl.x * lensRadius, pl.y * lensRadius);
        float focalDistMod = focalDistance * (1.0f + caAxial * s.lambdaOffset);
        float ft = focalDistMod / std::abs(dir.z);
        Vec3 pFocus = rayOrigin + dir * ft;
        rayOrigin = Vec3(pLens.x, pLens.y, 0.0f);
        dir = pFocus - rayOrigin;
    }
    dir = Normalize(dir);
    float weight = 1.0f;
    if (vignetting) {
        float cosTheta = std::abs(dir.z);
        float cos2 = cosTheta * cosTheta;
        weight = cos2 * cos2;
    }
    float finalTime = s.time;
    if (rollingShutter) {
        float scanline = 1.0f - s.pFilm.y;
        finalTime = scanline * scanDuration + (s.time * exposureDuration);
    }
    Ray rc(rayOrigin, dir);
    *ray = anim.interpolate(finalTime).ray(rc);
    ray->time = finalTime;
    return weight;
}

// ---------------------------------------------------------------- primitive, scene
// primitive.cpp:7-46
// primitive.cpp:6-11
Primitive::Primitive(const PropertyList& p) {
    toWorld = p.getTransform("toWorld", Transform());
    anim.set(toWorld, p.getTransform("toWorldEnd", toWorld));
}
void Primitive::addChild(ObjectPtr c) {
    if (c->classType() == EShape) {
        if (shape) throw std::runtime_error("Primitive: shape already registered!");
        shape = std::static_pointer_cast<Shape>(c);
    } else if (c->classType() == EMaterial) {
        if (material) throw std::runtime_error("Primitive: material already registered!");
        material = std::static_pointer_cast<Material>(c);
    } else if (c->classType() == EEmitter) {
        if (emitter) throw std::runtime_error("Primitive: emitter already registered!");
        emitter = std::static_pointer_cast<Emitter>(c);
        emitter->prim = this;
    } else {
        throw std::runtime_error("Primitive: invalid child class! Expected Shape.");
    }
}
void Primitive::activate() {
    if (!shape) throw std::runtime_error("Primitive: defined without a Shape!");
    if (!material) {
        auto m = std::make_shared<Matte>(PropertyList());
        m->activate();
        material = m;
    }
}

// scene.cpp:9-44
void Scene::addChild(ObjectPtr c) {
    switch (c->classType()) {
        case EPrimitive: {
            auto p = std::static_pointer_cast<Primitive>(c);
            p->originalIndex = (int)prims.size();
            prims.push_back(p);
            if (p->emitter) emitters.push_back(p->emitter);
            break;
        }
        case ECamera:
            if (camera) throw std::runtime_error("Scene: cannot add multiple cameras!");
            camera = std::static_pointer_cast<Camera>(c);
            break;
        case EIntegrator:
            if (integrator) throw std::runtime_error("Scene: cannot add multiple integrators!");
            integrator = std::static_pointer_cast<IntegratorObj>(c);
            break;
        case ESampler:
            if (sampler) throw std::runtime_error("Scene: cannot add multiple samplers!");
            sampler = std::static_pointer_cast<SamplerObj>(c);
            break;
        case EEmitter:   // scene.cpp:33-40
            emitters.push_back(std::static_pointer_cast<Emitter>(c));
            if (emitters.back()->isInfiniteAreaLight()) {
                if (envMap) throw std::runtime_error("Scene: cannot add multiple infinite area lights!");
                envMap = emitters.back();
            }
            break;
        default:
            throw std::runtime_error("Scene: cannot add specified child!");
    }
}
// scene.cpp:46-62
void Scene::activate() {
    if (!camera) throw std::runtime_error("Scene: no camera specified!");
    if (!integrator) throw std::runtime_error("Scene: no integrator specified!");
    if (!sampler) throw std::runtime_error("Scene: no sampler specified!");
    buildTLAS();
}

// ---------------------------------------------------------------- registry
// factory.cpp:17-22 with the class names registered across the reference's plugins
std::unique_ptr<Object> createInstance(const std::string& t, const PropertyList& p) {
    if (t == "scene") return std::make_unique<Scene>(p);
    if (t == "primitive") return std::make_unique<Primitive>(p);
    if (t == "mesh") return std::make_unique<Mesh>(p);
    if (t == "sphere") return std::make_unique<Sphere>(p);
    if (t == "cube") return std::make_unique<Cube>(p);
    if (t == "matte") return std::make_unique<Matte>(p);
    if (t == "plastic") return std::make_unique<Plastic>(p);
    if (t == "conductor") return std::make_unique<Conductor>(p);
    if (t == "glass") return std::make_unique<Glass>(p);
    if (t == "index") return std::make_unique<IndexMaterial>(p);
    if (t == "homogeneous") return std::make_unique<HomogeneousMedium>(p);
    if (t == "area") return std::make_unique<AreaLight>(p);
    if (t == "point") return std::make_unique<PointLight>(p);
    if (t == "spot") return std::make_unique<SpotLight>(p);
    if (t == "directional") return std::make_unique<DirectionalLight>(p);
    if (t == "environment") return std::make_unique<EnvironmentMap>(p);
    if (t == "perspective") return std::make_unique<Camera>(p, 0);
    if (t == "thinlens") return std::make_unique<Camera>(p, 1);
    if (t == "box") return std::make_unique<BoxFilter>(p);
    if (t == "gaussian") return std::make_unique<GaussianFilter>(p);
    if (t == "independent") return std::make_unique<SamplerObj>(p);
    // the GPU drop-ins share the CPU integrators' algorithm
    if (t == "path" || t == "path_gpu") return std::make_unique<IntegratorObj>(0, p);
    if (t == "volpath" || t == "volpath_gpu") return std::make_unique<IntegratorObj>(1, p);
    if (t == "constant_color") return std::make_unique<ConstantTexture<Color>>(p);
    if (t == "constant_float") return std::make_unique<ConstantTexture<float>>(p);
    if (t == "checkerboard_color") return std::make_unique<CheckerTexture<Color>>(p);
    if (t == "checkerboard_float") return std::make_unique<CheckerTexture<float>>(p);
    if (t == "perlin_color") return std::make_unique<PerlinTexture<Color>>(p);
    if (t == "perlin_float") return std::make_unique<PerlinTexture<float>>(p);
    if (t == "marble_color") return std::make_unique<MarbleTexture<Color>>(p);
    if (t == "marble_float") return std::make_unique<MarbleTexture<float>>(p);
    if (t == "wood_color") return std::make_unique<WoodTexture<Color>>(p);
    if (t == "wood_float") return std::make_unique<WoodTexture<float>>(p);
    if (t == "cellular_color") return std::make_unique<CellularTexture<Color>>(p);
    if (t == "cellular_float") return std::make_unique<CellularTexture<float>>(p);
    if (t == "domainWarp_color") return std::make_unique<DomainWarpTexture<Color>>(p);
    if (t == "domainWarp_float") return std::make_unique<DomainWarpTexture<float>>(p);
    if (t == "image_color") return std::make_unique<ImageTexture<Color>>(p);
    if (t == "image_float") return std::make_unique<ImageTexture<float>>(p);
    if (t == "image_normal") {   // ImageTexture<Normal3f>: 2 c - 1 of the rgb, (0, 0, 1) for 1-2 channels
        auto n = std::make_unique<ImageTexture<Color>>(p);
        n->normal = true;
        return n;
    }
    throw std::runtime_error("Cannot instantiate object: class '" + t + "' is not registered!");
}

}  // namespace orc

// ---------------------------------------------------------------- environment-map probes
// Direct calls into the environment emitter for the sampling tests (the reference's
// environment_test.cpp design): load, sample, pdf, eval; the reference point is the
// origin and the light point lies 1e5 along the direction, as in its integrators.
extern "C" {
void* orc_env_load(const char* path, float strength) {
    orc::PropertyList p;
    p.s["filename"] = path;
    p.f["strength"] = strength;
    auto* e = new orc::EnvironmentMap(p);
    try {
        e->activate();
    } catch (...) {
        delete e;
        return nullptr;
    }
    return e;
}
void orc_env_free(void* e) { delete static_cast<orc::EnvironmentMap*>(e); }
void orc_env_sample(void* h, int n, const float* u, float* dir, float* pdf, float* L) {
    auto* e = static_cast<orc::EnvironmentMap*>(h);
    for (int i = 0; i < n; ++i) {
        orc::SurfaceInteraction ref, info;
        orc::Ray sr;
        float p = 0.0f;
        orc::Color c = e->sample(ref, orc::Vec2(u[2 * i], u[2 * i + 1]), info, p, sr);
        orc::Vec3 w = orc::Normalize(info.p - ref.p);
        dir[3 * i] = w.x; dir[3 * i + 1] = w.y; dir[3 * i + 2] = w.z;
        pdf[i] = p;
        L[3 * i] = c.r; L[3 * i + 1] = c.g; L[3 * i + 2] = c.b;
    }
}
void orc_env_pdf(void* h, int n, const float* dir, float* pdf) {
    auto* e = static_cast<orc::EnvironmentMap*>(h);
    for (int i = 0; i < n; ++i) {
        orc::SurfaceInteraction ref, info;
        orc::Vec3 w(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        info.p = ref.p + w * 1e5f;
        pdf[i] = e->pdf(ref, info);
    }
}
void orc_env_eval(void* h, int n, const float* dir, float* L) {
    auto* e = static_cast<orc::EnvironmentMap*>(h);
    for (int i = 0; i < n; ++i) {
        orc::Color c = e->eval(orc::SurfaceInteraction(), orc::Vec3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]));
        L[3 * i] = c.r; L[3 * i + 1] = c.g; L[3 * i + 2] = c.b;
    }
}
}
