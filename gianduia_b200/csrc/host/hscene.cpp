// Host scene framework: matrices, the plugin registry and the scene objects, and the
// flattening of a scene into the device layout (BLAS per unique mesh, TLAS over the
// primitives, material / emitter / medium tables, area CDFs, camera).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <limits>
#include <thread>
#include <unordered_map>

#include "hscene.h"

namespace gndh {

// ---------------------------------------------------------------- matrices
Mat4 Mat4::identity() {
    Mat4 m;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m.c[i][j] = (i == j) ? 1.f : 0.f;
    return m;
}
void Mat4::mulVec(const float v[4], float out[4]) const {
    for (int r = 0; r < 4; ++r) {
        float add0 = c[0][r] * v[0] + c[1][r] * v[1];
        float add1 = c[2][r] * v[2] + c[3][r] * v[3];
        out[r] = add0 + add1;
    }
}
Mat4 Mat4::operator*(const Mat4& b) const {
    Mat4 m;
    for (int col = 0; col < 4; ++col) mulVec(b.c[col], m.c[col]);
    return m;
}
Mat4 Mat4::transpose() const {
    Mat4 m;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m.c[i][j] = c[j][i];
    return m;
}
bool Mat4::operator==(const Mat4& o) const { return std::memcmp(c, o.c, sizeof(c)) == 0; }
gnd::Xf34 Mat4::toXf34() const {
    gnd::Xf34 x;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 4; ++k) x.r[r][k] = c[k][r];
    return x;
}
Mat4 inverse(const Mat4& mm) {
    float a[4][4], inv[4][4];
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) a[r][k] = mm.c[k][r];
    for (int r = 0; r < 4; ++r) {
        for (int k = 0; k < 4; ++k) {
            float s[3][3];
            int si = 0;
            for (int i = 0; i < 4; ++i) {
                if (i == k) continue;
                int sj = 0;
                for (int j = 0; j < 4; ++j) {
                    if (j == r) continue;
                    s[si][sj++] = a[i][j];
                }
                ++si;
            }
            float d3 = s[0][0] * (s[1][1] * s[2][2] - s[1][2] * s[2][1]) - s[0][1] * (s[1][0] * s[2][2] - s[1][2] * s[2][0]) +
                       s[0][2] * (s[1][0] * s[2][1] - s[1][1] * s[2][0]);
            inv[r][k] = ((r + k) & 1) ? -d3 : d3;
        }
    }
    float det = a[0][0] * inv[0][0] + a[0][1] * inv[1][0] + a[0][2] * inv[2][0] + a[0][3] * inv[3][0];
    float invDet = 1.0f / det;
    Mat4 out;
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) out.c[k][r] = inv[r][k] * invDet;
    return out;
}
V3 Transform::point(V3 p) const {
    float in[4] = {p.x, p.y, p.z, 1.f}, o[4];
    m.mulVec(in, o);
    if (o[3] == 1.0f) return gnd::v3(o[0], o[1], o[2]);
    return gnd::v3(o[0] / o[3], o[1] / o[3], o[2] / o[3]);
}
V3 Transform::vector(V3 v) const {
    float in[4] = {v.x, v.y, v.z, 0.f}, o[4];
    m.mulVec(in, o);
    return gnd::v3(o[0], o[1], o[2]);
}
Transform Transform::translate(V3 d) {
    Mat4 a = Mat4::identity(), b = Mat4::identity();
    a.c[3][0] = d.x; a.c[3][1] = d.y; a.c[3][2] = d.z;
    b.c[3][0] = -d.x; b.c[3][1] = -d.y; b.c[3][2] = -d.z;
    return Transform(a, b);
}
Transform Transform::scale(float x, float y, float z) {
    Mat4 a = Mat4::identity(), b = Mat4::identity();
    a.c[0][0] = x; a.c[1][1] = y; a.c[2][2] = z;
    b.c[0][0] = 1.f / x; b.c[1][1] = 1.f / y; b.c[2][2] = 1.f / z;
    return Transform(a, b);
}
// Rodrigues rotation about the normalised axis; inverse = transpose (transform.h:421-426)
Transform Transform::rotate(float degrees, V3 axis) {
    float rad = degrees * 0.01745329251994329576923690768489f;
    float c = std::cos(rad), s = std::sin(rad);
    V3 ax = gnd::normalize(axis);
    V3 tp = ax * (1.0f - c);
    Mat4 m = Mat4::identity();
    m.c[0][0] = c + tp.x * ax.x;
    m.c[0][1] = tp.x * ax.y + s * ax.z;
    m.c[0][2] = tp.x * ax.z - s * ax.y;
    m.c[1][0] = tp.y * ax.x - s * ax.z;
    m.c[1][1] = c + tp.y * ax.y;
    m.c[1][2] = tp.y * ax.z + s * ax.x;
    m.c[2][0] = tp.z * ax.x + s * ax.y;
    m.c[2][1] = tp.z * ax.y - s * ax.x;
    m.c[2][2] = c + tp.z * ax.z;
    return Transform(m, m.transpose());
}
// Right-handed view matrix; camera-to-world is its inverse (transform.h:428-431)
Transform Transform::lookAt(V3 pos, V3 target, V3 up) {
    V3 f = gnd::normalize(target - pos);
    V3 s = gnd::normalize(gnd::cross(f, up));
    V3 u = gnd::cross(s, f);
    Mat4 v = Mat4::identity();
    v.c[0][0] = s.x; v.c[1][0] = s.y; v.c[2][0] = s.z;
    v.c[0][1] = u.x; v.c[1][1] = u.y; v.c[2][1] = u.z;
    v.c[0][2] = -f.x; v.c[1][2] = -f.y; v.c[2][2] = -f.z;
    v.c[3][0] = -gnd::dot(s, pos); v.c[3][1] = -gnd::dot(u, pos); v.c[3][2] = gnd::dot(f, pos);
    return Transform(gndh::inverse(v), v);
}

// ---------------------------------------------------------------- registry
const char* classTypeToString(EClassType t) {
    switch (t) {
        case EScene: return "scene";
        case EPrimitive: return "primitive";
        case EShape: return "shape";
        case ECamera: return "camera";
        case EIntegrator: return "integrator";
        case ESampler: return "sampler";
        case ETexture: return "texture";
        case EMaterial: return "material";
        case EEmitter: return "emitter";
        case EFilter: return "filter";
        case EMedium: return "medium";
    }
    return "unknown";
}
GndFactory* GndFactory::getInstance() {
    static GndFactory f;
    return &f;
}
void GndFactory::registerClass(const std::string& name, const ObjectFactory& f) { m_ctors[name] = f; }
std::unique_ptr<GndObject> GndFactory::createInstance(const std::string& name, const PropertyList& props) {
    auto it = m_ctors.find(name);
    if (it == m_ctors.end()) throw std::runtime_error("Cannot instantiate object: class '" + name + "' is not registered!");
    return it->second(props);
}

// ---------------------------------------------------------------- textures
namespace {
gnd::ColorTex constColor(V3 v) {
    gnd::ColorTex t{};
    t.kind = 0;
    t.v1[0] = v.x; t.v1[1] = v.y; t.v1[2] = v.z;
    t.scale[0] = t.scale[1] = 1.f;
    return t;
}
// matte.cpp:33-43, area.cpp:31-43: the magenta "missing texture" checkerboard
gnd::ColorTex missingTexture() {
    gnd::ColorTex t{};
    t.kind = 1;
    t.v1[0] = t.v1[1] = t.v1[2] = 0.f;
    t.v2[0] = 1.f; t.v2[1] = 0.f; t.v2[2] = 1.f;
    t.scale[0] = t.scale[1] = 0.1f;
    return t;
}
}  // namespace

// constant.h:9-32
struct ConstantColor : ColorTexture {
    explicit ConstantColor(const PropertyList& p) { rec = constColor(p.getColor("value", gnd::v3s(1.f))); }
};
struct ConstantFloat : FloatTexture {
    explicit ConstantFloat(const PropertyList& p) {
        value = p.getFloat("value", 1.0f);
        tree = std::make_shared<ColorTexture>();
        tree->rec = constColor(gnd::v3s(value));
    }
};
// checkerboard.h:20-48
struct CheckerboardColor : ColorTexture {
    explicit CheckerboardColor(const PropertyList& p, bool flt = false) {
        V3 a = flt ? gnd::v3s(p.getFloat("value1", 1.0f)) : p.getColor("value1", gnd::v3s(1.f));
        V3 b = flt ? gnd::v3s(p.getFloat("value2", 0.0f)) : p.getColor("value2", gnd::v3s(0.f));
        V2 sc = p.getVector2("scale", V2{1.f, 1.f}), de = p.getPoint2("delta", V2{0.f, 0.f});
        rec.kind = 1;
        rec.v1[0] = a.x; rec.v1[1] = a.y; rec.v1[2] = a.z;
        rec.v2[0] = b.x; rec.v2[1] = b.y; rec.v2[2] = b.z;
        rec.scale[0] = sc.x; rec.scale[1] = sc.y;
        rec.delta[0] = de.x; rec.delta[1] = de.y;
    }
};
GND_REGISTER_CLASS(ConstantColor, "constant_color")
GND_REGISTER_CLASS(ConstantFloat, "constant_float")
GND_REGISTER_CLASS(CheckerboardColor, "checkerboard_color")

gnd::TexNode ColorTexture::node(TexTables&) const {
    gnd::TexNode n{};
    n.kind = rec.kind == gnd::kTexChecker ? gnd::kTnChecker : gnd::kTnConstant;
    for (int k = 0; k < 3; ++k) { n.v1[k] = rec.v1[k]; n.v2[k] = rec.v2[k]; }
    n.cscale[0] = rec.scale[0]; n.cscale[1] = rec.scale[1];
    n.delta[0] = rec.delta[0]; n.delta[1] = rec.delta[1];
    return n;
}
int32_t ColorTexture::flatten(TexTables& t) const {
    auto it = t.done.find(this);
    if (it != t.done.end()) return it->second;
    gnd::TexNode n = node(t);   // flattens the inputs first
    const int32_t idx = (int32_t)t.nodes.size();
    t.nodes.push_back(n);
    t.done.emplace(this, idx);
    return idx;
}

namespace {
// The value1 / value2 pair and p / scale of the procedural color textures
struct ProceduralColor : ColorTexture {
    V3 v1{}, v2{};
    float scale = 1.0f;
    int octaves = 6;
    bool flt = false;   // float texture: value1 / value2 are floats (default 0 and 1)
    ProceduralColor(const PropertyList& p, V3 d1, V3 d2, bool isFloat) : flt(isFloat) {
        rec.kind = gnd::kTexNode;
        v1 = flt ? gnd::v3s(p.getFloat("value1", 0.0f)) : p.getColor("value1", d1);
        v2 = flt ? gnd::v3s(p.getFloat("value2", 1.0f)) : p.getColor("value2", d2);
        scale = p.getFloat("scale", 1.0f);
    }
    gnd::TexNode base(int32_t kind) const {
        gnd::TexNode n{};
        n.kind = kind;
        if (flt) n.flags = gnd::kTnFloatLerp;
        n.v1[0] = v1.x; n.v1[1] = v1.y; n.v1[2] = v1.z;
        n.v2[0] = v2.x; n.v2[1] = v2.y; n.v2[2] = v2.z;
        n.scale = scale;
        n.octaves = octaves;
        return n;
    }
};
// perlin.h (texture):15-37: value1 .. value2 by turbulence(p / scale)
struct PerlinColor : ProceduralColor {
    explicit PerlinColor(const PropertyList& p, bool flt = false) : ProceduralColor(p, gnd::v3s(0.0f), gnd::v3s(1.0f), flt) {
        octaves = p.getInteger("octaves", 6);
    }
    gnd::TexNode node(TexTables&) const override { return base(gnd::kTnPerlin); }
};
// marble.h:15-46 and wood.h:15-46: veins along / around an axis, perturbed by turbulence
struct VeinColor : ProceduralColor {
    int32_t kind;
    float veinFreq, turbScale;
    V3 axis;
    VeinColor(const PropertyList& p, int32_t k, V3 d1, V3 d2, float turbDefault, bool flt)
        : ProceduralColor(p, d1, d2, flt), kind(k) {
        octaves = p.getInteger("octaves", 6);
        veinFreq = p.getFloat("vein_freq", 10.0f);
        turbScale = p.getFloat("turb_scale", turbDefault);
        axis = gnd::normalize(p.getVector3("axis", gnd::v3(0.0f, 1.0f, 0.0f)));
    }
    gnd::TexNode node(TexTables&) const override {
        gnd::TexNode n = base(kind);
        n.veinFreq = veinFreq;
        n.turbScale = turbScale;
        n.axis[0] = axis.x; n.axis[1] = axis.y; n.axis[2] = axis.z;
        return n;
    }
};
struct MarbleColor : VeinColor {
    explicit MarbleColor(const PropertyList& p, bool flt = false)
        : VeinColor(p, gnd::kTnMarble, gnd::v3s(0.1f), gnd::v3s(0.9f), 5.0f, flt) {}
};
struct WoodColor : VeinColor {
    explicit WoodColor(const PropertyList& p, bool flt = false)
        : VeinColor(p, gnd::kTnWood, gnd::v3(0.6f, 0.4f, 0.2f), gnd::v3(0.3f, 0.15f, 0.05f), 2.0f, flt) {}
};
// cellular.h:17-58: Worley F1 (distance) or F2 - F1 (cracks), unknown names fall back
struct CellularColor : ProceduralColor {
    int32_t flags = 0;
    explicit CellularColor(const PropertyList& p, bool flt = false) : ProceduralColor(p, gnd::v3s(0.0f), gnd::v3s(1.0f), flt) {
        if (p.getString("mode", "distance") == "cracks") flags |= gnd::kTnCracks;
        const std::string m = p.getString("metric", "euclidean");
        const int metric = m == "manhattan" ? 1 : (m == "chebyshev" ? 2 : 0);
        flags |= metric << gnd::kTnMetricShift;
    }
    gnd::TexNode node(TexTables&) const override {
        gnd::TexNode n = base(gnd::kTnCellular);
        n.flags = flags;   // Lerp (constants.h:41-44) for both flavours, never std::lerp
        return n;
    }
};
// domainWarp.h:13-58: the base texture evaluated at p and uv moved by the warp texture
struct DomainWarpColor : ColorTexture {
    float strength;
    std::shared_ptr<ColorTexture> baseTex, warpTex;
    bool flt = false;
    explicit DomainWarpColor(const PropertyList& p, bool isFloat = false) : strength(p.getFloat("strength", 1.0f)), flt(isFloat) {
        rec.kind = gnd::kTexNode;
    }
    void addChild(std::shared_ptr<GndObject> c) override {
        if (c->getClassType() != ETexture) throw std::runtime_error("WarpTexture: cannot add specified child!");
        auto t = std::dynamic_pointer_cast<ColorTexture>(c);
        if (c->getName() == "base") {
            if (baseTex) throw std::runtime_error("WarpTexture: base texture already defined!");
            if (flt) {
                auto f = std::dynamic_pointer_cast<FloatTexture>(c);
                if (!f) throw std::runtime_error("WarpTexture: the base of a float warp must be a float texture");
                t = f->tree;
            }
            if (!t) throw std::runtime_error("WarpTexture: the base of a color warp must be a color texture");
            baseTex = t;
        } else if (c->getName() == "warp") {
            if (warpTex) throw std::runtime_error("WarpTexture: warp texture already defined!");
            if (!t) throw std::runtime_error("WarpTexture: the warp input must be a color texture");
            warpTex = t;
        }
    }
    void activate() override {
        if (!baseTex) throw std::runtime_error("WarpTexture: missing base texture!");
        if (!warpTex) throw std::runtime_error("WarpTexture: missing warp texture!");
    }
    gnd::TexNode node(TexTables& t) const override {
        gnd::TexNode n{};
        n.kind = gnd::kTnWarp;
        n.strength = strength;
        n.a = baseTex->flatten(t);
        n.b = warpTex->flatten(t);
        return n;
    }
};
// imageTexture.cpp:11-143 with the texels of textureCache.h
struct ImageColor : ColorTexture {
    std::string filename, baseDir;
    bool linear = false, clamp = false, srgb = false;
    int width = 0, height = 0, channels = 0;
    std::vector<float> texels;
    // float image textures read the first channel (imageTexture.cpp:93-95), which is the
    // first texel channel here as well
    bool normal = false;   // image_normal
    bool isNormalMap() const override { return normal; }
    explicit ImageColor(const PropertyList& p, bool = false, bool isNormal = false) : filename(p.getString("filename")), normal(isNormal) {
        rec.kind = gnd::kTexNode;
        const std::string interp = p.getString("interpolation_mode", "closest");
        if (interp == "linear") linear = true;
        else if (interp != "closest") throw std::runtime_error("ImageTexture: Unknown interpolation mode " + interp);
        const std::string cs = p.getString("color_space", "linear");
        if (cs == "sRGB") srgb = true;
        else if (cs != "linear") throw std::runtime_error("ImageTexture: Unknown color space " + cs);
        const std::string rep = p.getString("repeat_mode", "repeat");
        if (rep == "clamp") clamp = true;
        else if (rep != "repeat") throw std::runtime_error("ImageTexture: Unknown repeat mode " + rep);
    }
    void setBaseDir(const std::string& d) override { baseDir = d; }
    void activate() override {
        std::filesystem::path abs(filename);
        if (abs.is_relative() && !baseDir.empty()) abs = std::filesystem::path(baseDir) / abs;
        readTextureImage(abs.string(), srgb, width, height, channels, texels);
    }
    gnd::TexNode node(TexTables& t) const override {
        gnd::TexNode n{};
        n.kind = gnd::kTnImage;
        n.flags = (linear ? gnd::kTnLinear : 0) | (clamp ? gnd::kTnClamp : 0) | (normal ? gnd::kTnNormal : 0);
        if (t.texels.size() / 4 + (size_t)width * height > (size_t)INT32_MAX)
            throw std::runtime_error("ImageTexture: image textures larger than 2^31 texels in total");
        n.a = (int32_t)(t.texels.size() / 4);
        n.b = channels;
        n.w = width;
        n.h = height;
        // extractValue (imageTexture.cpp:96-100): rgb of 3-4 channel images, the first
        // channel repeated otherwise
        for (size_t i = 0; i < (size_t)width * height; ++i) {
            const float* q = &texels[4 * i];
            const bool rgb = channels >= 3;
            t.texels.push_back(q[0]);
            t.texels.push_back(rgb ? q[1] : q[0]);
            t.texels.push_back(rgb ? q[2] : q[0]);
            t.texels.push_back(q[3]);
        }
        return n;
    }
};
// The float variants: the color texture classes built with float values, as a tree.
template <class C>
struct TreeFloat : FloatTexture {
    explicit TreeFloat(const PropertyList& p) {
        constant = false;
        tree = std::make_shared<C>(p, true);
    }
    void addChild(std::shared_ptr<GndObject> c) override { tree->addChild(c); }
    void activate() override { tree->activate(); }
    void setBaseDir(const std::string& d) override { tree->setBaseDir(d); }
};
using CheckerboardFloat = TreeFloat<CheckerboardColor>;
using PerlinFloat = TreeFloat<PerlinColor>;
using MarbleFloat = TreeFloat<MarbleColor>;
using WoodFloat = TreeFloat<WoodColor>;
using CellularFloat = TreeFloat<CellularColor>;
using DomainWarpFloat = TreeFloat<DomainWarpColor>;
using ImageFloat = TreeFloat<ImageColor>;
// imageTexture.cpp:101-104 (ImageTexture<Normal3f>)
struct ImageNormal : ImageColor {
    explicit ImageNormal(const PropertyList& p) : ImageColor(p, false, true) {}
};
}  // namespace
GND_REGISTER_CLASS(PerlinColor, "perlin_color")
GND_REGISTER_CLASS(MarbleColor, "marble_color")
GND_REGISTER_CLASS(WoodColor, "wood_color")
GND_REGISTER_CLASS(CellularColor, "cellular_color")
GND_REGISTER_CLASS(DomainWarpColor, "domainWarp_color")
GND_REGISTER_CLASS(ImageColor, "image_color")
GND_REGISTER_CLASS(CheckerboardFloat, "checkerboard_float")
GND_REGISTER_CLASS(PerlinFloat, "perlin_float")
GND_REGISTER_CLASS(MarbleFloat, "marble_float")
GND_REGISTER_CLASS(WoodFloat, "wood_float")
GND_REGISTER_CLASS(CellularFloat, "cellular_float")
GND_REGISTER_CLASS(DomainWarpFloat, "domainWarp_float")
GND_REGISTER_CLASS(ImageFloat, "image_float")
GND_REGISTER_CLASS(ImageNormal, "image_normal")

// ---------------------------------------------------------------- media
// homogeneous.cpp:14-20
struct HomogeneousMediumObj : MediumObj {
    explicit HomogeneousMediumObj(const PropertyList& p) {
        V3 a = p.getColor("sigma_a", gnd::v3s(0.1f)), s = p.getColor("sigma_s", gnd::v3s(0.1f));
        V3 t = a + s;
        rec.sigA[0] = a.x; rec.sigA[1] = a.y; rec.sigA[2] = a.z;
        rec.sigS[0] = s.x; rec.sigS[1] = s.y; rec.sigS[2] = s.z;
        rec.sigT[0] = t.x; rec.sigT[1] = t.y; rec.sigT[2] = t.z;
        rec.g = p.getFloat("g", 0.0f);
    }
};
GND_REGISTER_CLASS(HomogeneousMediumObj, "homogeneous")

// ---------------------------------------------------------------- materials
// material.h:36-59 (normal and bump maps are not part of the GPU path)
void MaterialObj::addChild(std::shared_ptr<GndObject> c) {
    if (c->getClassType() == ETexture && c->getName() == "normal") {
        if (normalTex) throw std::runtime_error("Material: normal map already defined!");
        auto t = std::dynamic_pointer_cast<ColorTexture>(c);
        if (!t || !t->isNormalMap()) throw std::runtime_error("Material: the normal map must be an image_normal texture");
        normalTex = t;
    } else if (c->getClassType() == ETexture && c->getName() == "bump") {
        if (bumpTex) throw std::runtime_error("Material: bump map already defined!");
        auto f = std::dynamic_pointer_cast<FloatTexture>(c);
        if (!f) throw std::runtime_error("Material: the bump map must be a float texture");
        bumpTex = f->tree;
    } else if (c->getClassType() == EMedium && c->getName() == "inside") {
        if (inside) throw std::runtime_error("Material: inside medium already defined!");
        inside = std::static_pointer_cast<MediumObj>(c);
    } else if (c->getClassType() == EMedium && c->getName() == "outside") {
        if (outside) throw std::runtime_error("Material: outside medium already defined!");
        outside = std::static_pointer_cast<MediumObj>(c);
    } else {
        throw std::runtime_error("Material: cannot add specified child (" + c->getName() + ")!");
    }
}

namespace {
void setColorSlot(gnd::ColorTex& slot, bool& have, const std::shared_ptr<GndObject>& c, std::shared_ptr<ColorTexture>& keep) {
    auto t = std::dynamic_pointer_cast<ColorTexture>(c);
    if (!t) throw std::runtime_error("Material: texture '" + c->getName() + "' must be a color texture");
    slot = t->rec;
    keep = t;
    have = true;
}
void setFloatSlot(float& slot, bool& have, const std::shared_ptr<GndObject>& c, std::shared_ptr<ColorTexture>& keep) {
    auto t = std::dynamic_pointer_cast<FloatTexture>(c);
    if (!t) throw std::runtime_error("Material: texture '" + c->getName() + "' must be a float texture");
    if (!t->constant) {
        keep = t->tree;
        have = true;
        return;
    }
    slot = t->value;
    have = true;
}
}  // namespace

// matte.cpp:7-53
struct MatteMat : MaterialObj {
    bool hasA = false;
    explicit MatteMat(const PropertyList& p) {
        rec.type = gnd::kMatMatte;
        rec.bumpScale = p.getFloat("bump_scale", 1.0f);   // material.h:14
        if (p.hasColor("albedo")) { rec.a = constColor(p.getColor("albedo", gnd::v3s(0.f))); hasA = true; }
    }
    void addChild(std::shared_ptr<GndObject> c) override {
        if (c->getClassType() != ETexture) return MaterialObj::addChild(c);
        if (c->getName() == "albedo") {
            if (hasA) throw std::runtime_error("Matte: there's already an albedo defined!");
            setColorSlot(rec.a, hasA, c, texA);
        } else MaterialObj::addChild(c);
    }
    void activate() override { if (!hasA) rec.a = missingTexture(); }
};
// plastic.cpp:8-91
struct PlasticMat : MaterialObj {
    bool hKd = false, hKs = false, hR = false, hE = false;
    explicit PlasticMat(const PropertyList& p) {
        rec.type = gnd::kMatPlastic;
        rec.bumpScale = p.getFloat("bump_scale", 1.0f);   // material.h:14
        if (p.hasColor("Kd")) { rec.a = constColor(p.getColor("Kd", gnd::v3s(0.f))); hKd = true; }
        if (p.hasColor("Ks")) { rec.b = constColor(p.getColor("Ks", gnd::v3s(0.f))); hKs = true; }
        if (p.hasFloat("roughness")) { rec.roughness = p.getFloat("roughness"); hR = true; }
        if (p.hasFloat("eta")) { rec.eta = p.getFloat("eta"); hE = true; }
    }
    void addChild(std::shared_ptr<GndObject> c) override {
        if (c->getClassType() != ETexture) return;   // plastic.cpp:30
        const std::string& n = c->getName();
        if (n == "Kd") setColorSlot(rec.a, hKd, c, texA);
        else if (n == "Ks") setColorSlot(rec.b, hKs, c, texB);
        else if (n == "roughness") setFloatSlot(rec.roughness, hR, c, roughTex);
        else if (n == "eta") setFloatSlot(rec.eta, hE, c, etaTex);
        else MaterialObj::addChild(c);
    }
    void activate() override {
        if (!hKd) rec.a = constColor(gnd::v3s(0.25f));
        if (!hKs) rec.b = constColor(gnd::v3s(0.25f));
        if (!hR) rec.roughness = 0.1f;
        if (!hE) rec.eta = 1.5f;
    }
};
// conductor.cpp:9-120
struct ConductorMat : MaterialObj {
    bool hR = false, hE = false, hK = false, hRo = false;
    V3 eta{1, 1, 1}, k{1, 1, 1};
    explicit ConductorMat(const PropertyList& p) {
        rec.type = gnd::kMatConductor;
        rec.bumpScale = p.getFloat("bump_scale", 1.0f);   // material.h:14
        if (p.hasColor("R")) { rec.a = constColor(p.getColor("R", gnd::v3s(0.f))); hR = true; }
        if (p.hasColor("eta")) { eta = p.getColor("eta", eta); hE = true; }
        if (p.hasColor("k")) { k = p.getColor("k", k); hK = true; }
        if (p.hasFloat("roughness")) { rec.roughness = p.getFloat("roughness"); hRo = true; }
    }
    void addChild(std::shared_ptr<GndObject> c) override {
        if (c->getClassType() != ETexture) throw std::runtime_error("Conductor: cannot add specified child!");
        const std::string& n = c->getName();
        if (n == "R") setColorSlot(rec.a, hR, c, texA);
        else if (n == "roughness") setFloatSlot(rec.roughness, hRo, c, roughTex);
        else if (n == "eta" || n == "k") {
            auto t = std::dynamic_pointer_cast<ColorTexture>(c);
            if (!t) throw std::runtime_error("Conductor: eta/k must be color textures");
            bool& have = n == "eta" ? hE : hK;
            if (t->rec.kind == gnd::kTexConstant) {
                (n == "eta" ? eta : k) = gnd::v3(t->rec.v1[0], t->rec.v1[1], t->rec.v1[2]);
            } else {
                (n == "eta" ? etaTex : kTex) = t;   // evaluated per shading point
            }
            have = true;
        } else MaterialObj::addChild(c);
    }
    void activate() override {
        if (!hR) rec.a = constColor(gnd::v3s(1.f));
        if (!hRo) rec.roughness = 0.f;
        rec.condEta[0] = eta.x; rec.condEta[1] = eta.y; rec.condEta[2] = eta.z;
        rec.condK[0] = k.x; rec.condK[1] = k.y; rec.condK[2] = k.z;
    }
};
// glass.cpp:8-115
struct GlassMat : MaterialObj {
    bool hR = false, hT = false, hRo = false, hE = false;
    explicit GlassMat(const PropertyList& p) {
        rec.type = gnd::kMatGlass;
        rec.bumpScale = p.getFloat("bump_scale", 1.0f);   // material.h:14
        if (p.hasColor("R")) { rec.a = constColor(p.getColor("R", gnd::v3s(0.f))); hR = true; }
        if (p.hasColor("T")) { rec.b = constColor(p.getColor("T", gnd::v3s(0.f))); hT = true; }
        if (p.hasFloat("roughness")) { rec.roughness = p.getFloat("roughness"); hRo = true; }
        if (p.hasFloat("eta")) { rec.eta = p.getFloat("eta"); hE = true; }
    }
    void addChild(std::shared_ptr<GndObject> c) override {
        const std::string& n = c->getName();
        if (n == "R") setColorSlot(rec.a, hR, c, texA);
        else if (n == "T") setColorSlot(rec.b, hT, c, texB);
        else if (n == "roughness") setFloatSlot(rec.roughness, hRo, c, roughTex);
        else if (n == "eta") setFloatSlot(rec.eta, hE, c, etaTex);
        else MaterialObj::addChild(c);
    }
    void activate() override {
        if (!hR) rec.a = constColor(gnd::v3s(1.f));
        if (!hT) rec.b = constColor(gnd::v3s(1.f));
        if (!hRo) rec.roughness = 0.f;
        if (!hE) rec.eta = 1.5f;
    }
};
// index.cpp:6-16 (null BSDF: medium boundary only)
struct IndexMat : MaterialObj {
    explicit IndexMat(const PropertyList& p) {
        rec.type = gnd::kMatIndex;
        rec.bumpScale = p.getFloat("bump_scale", 1.0f);
    }
};
GND_REGISTER_CLASS(MatteMat, "matte")
GND_REGISTER_CLASS(PlasticMat, "plastic")
GND_REGISTER_CLASS(ConductorMat, "conductor")
GND_REGISTER_CLASS(GlassMat, "glass")
GND_REGISTER_CLASS(IndexMat, "index")

// ---------------------------------------------------------------- emitter
// area.cpp:7-43
void EmitterObj::addChild(std::shared_ptr<GndObject> c) {
    if (c->getClassType() != ETexture) throw std::runtime_error("AreaLight: cannot add specified child!");
    if (c->getName() == "radiance") {
        if (hasRadiance) throw std::runtime_error("AreaLight: there's already a radiance value defined!");
        setColorSlot(radiance, hasRadiance, c, radianceTex);
    }
}
void EmitterObj::activate() {
    if (type == gnd::kEmitArea && !hasRadiance) radiance = missingTexture();
    if (type != gnd::kEmitEnv) return;
    // environment.cpp:15-27 and buildPDFs (environment.cpp:111-124)
    std::filesystem::path abs = std::filesystem::path(filename);
    if (abs.is_relative()) abs = std::filesystem::path(baseDir) / abs;
    if (!std::filesystem::is_regular_file(abs)) throw std::runtime_error("EnvMap: Invalid environment map path.");
    if (abs.extension() != ".exr") throw std::runtime_error("EnvMap: Invalid environment map extension.");
    readEXR(abs.string(), envWidth, envHeight, envTexels);
    const int rows = envHeight, cols = envWidth;
    std::vector<float> img((size_t)rows * cols);
    for (int i = 0; i < rows; i++) {
        const float sinTheta = (float)std::sin(M_PI * (i + 0.5f) / rows);
        for (int j = 0; j < cols; j++) {
            const float* t = &envTexels[3 * ((size_t)i * cols + j)];
            img[(size_t)i * cols + j] = gnd::luminance(gnd::v3(t[0], t[1], t[2])) * sinTheta;
        }
    }
    // distribution.cpp:6-64: one 1D distribution per row, the marginal over row integrals
    auto build1D = [](const float* f, int n, float* func, float* cdf, float& funcInt) {
        for (int i = 0; i < n; ++i) func[i] = f[i];
        cdf[0] = 0.0f;
        for (int i = 1; i < n + 1; ++i) cdf[i] = cdf[i - 1] + func[i - 1] / n;
        funcInt = cdf[n];
        if (funcInt == 0.0f) {
            for (int i = 1; i < n + 1; ++i) cdf[i] = float(i) / float(n);
        } else {
            for (int i = 1; i < n + 1; ++i) cdf[i] /= funcInt;
        }
    };
    const size_t mf = 0, mc = mf + rows, cf = mc + rows + 1, cc = cf + (size_t)rows * cols, ci = cc + (size_t)rows * (cols + 1);
    envDist.assign(ci + rows, 0.0f);
    for (int v = 0; v < rows; ++v)
        build1D(&img[(size_t)v * cols], cols, &envDist[cf + (size_t)v * cols], &envDist[cc + (size_t)v * (cols + 1)], envDist[ci + v]);
    build1D(&envDist[ci], rows, &envDist[mf], &envDist[mc], envMarginalIntegral);
}
struct AreaLightObj : EmitterObj {
    explicit AreaLightObj(const PropertyList& p) {
        if (p.hasColor("radiance")) { radiance = constColor(p.getColor("radiance", gnd::v3s(0.f))); hasRadiance = true; }
    }
};
// pointlight.cpp:9-12
struct PointLightObj : EmitterObj {
    explicit PointLightObj(const PropertyList& p) {
        type = gnd::kEmitPoint;
        position = p.getPoint3("position", gnd::v3s(0.0f));
        color = p.getColor("power", gnd::v3s(10.0f));
    }
};
// spotlight.cpp:11-24
struct SpotLightObj : EmitterObj {
    explicit SpotLightObj(const PropertyList& p) {
        type = gnd::kEmitSpot;
        position = p.getPoint3("position", gnd::v3s(0.0f));
        direction = gnd::normalize(p.getVector3("direction", gnd::v3(0.0f, 0.0f, -1.0f)));
        color = p.getColor("power", gnd::v3s(10.0f));
        const float spotSize = p.getFloat("spot_size", 45.0f);
        const float blend = p.getFloat("blend", 0.15f);
        const float halfAngle = spotSize * 0.5f;
        const float innerAngle = halfAngle * (1.0f - blend);
        cosTotal = std::cos((gnd::kPi / 180.f) * halfAngle);
        cosFalloff = std::cos((gnd::kPi / 180.f) * innerAngle);
    }
};
// directional.cpp:9-12
struct DirectionalLightObj : EmitterObj {
    explicit DirectionalLightObj(const PropertyList& p) {
        type = gnd::kEmitDirectional;
        direction = -gnd::normalize(p.getVector3("direction", gnd::v3(0.0f, -1.0f, 0.0f)));
        color = p.getColor("irradiance", gnd::v3s(1.0f));
    }
};
// environment.cpp:15-27
struct EnvironmentObj : EmitterObj {
    explicit EnvironmentObj(const PropertyList& p) {
        type = gnd::kEmitEnv;
        filename = p.getString("filename");
        strength = p.getFloat("strength", 1.0f);
    }
};
GND_REGISTER_CLASS(AreaLightObj, "area")
GND_REGISTER_CLASS(PointLightObj, "point")
GND_REGISTER_CLASS(SpotLightObj, "spot")
GND_REGISTER_CLASS(DirectionalLightObj, "directional")
GND_REGISTER_CLASS(EnvironmentObj, "environment")

// ---------------------------------------------------------------- shapes
Bounds ShapeObj::objectBounds() const {
    Bounds b;
    if (kind == gnd::kShapeSphere) {
        b.lo = gnd::v3s(-radius); b.hi = gnd::v3s(radius);
    } else if (kind == gnd::kShapeCube) {
        b.lo = -extents; b.hi = extents;
    } else {
        for (const V3& p : positions) b.grow(p);
    }
    return b;
}
void ShapeObj::activate() {
    if (kind != gnd::kShapeMesh) return;
    if (!positions.empty()) return;   // geometry supplied in memory
    if (filename.empty()) throw std::runtime_error("Mesh: filename missing!");
    loadOBJ(filename, *this);
    if (positions.empty()) throw std::runtime_error("Mesh: no geometry loaded!");
}
struct MeshShape : ShapeObj {
    explicit MeshShape(const PropertyList& p) { kind = gnd::kShapeMesh; filename = p.getString("filename", ""); }
};
struct SphereShape : ShapeObj {
    explicit SphereShape(const PropertyList& p) { kind = gnd::kShapeSphere; radius = p.getFloat("radius", 1.0f); }
};
struct CubeShape : ShapeObj {
    explicit CubeShape(const PropertyList& p) { kind = gnd::kShapeCube; extents = p.getVector3("extents", gnd::v3s(1.f)); }
};
GND_REGISTER_CLASS(MeshShape, "mesh")
GND_REGISTER_CLASS(SphereShape, "sphere")
GND_REGISTER_CLASS(CubeShape, "cube")

// ---------------------------------------------------------------- primitive
// primitive.cpp:6-11
PrimitiveObj::PrimitiveObj(const PropertyList& p) {
    toWorld = p.getTransform("toWorld", Transform());
    toWorldEnd = p.getTransform("toWorldEnd", toWorld);
    animated = !(toWorldEnd == toWorld);
}

gnd::InstMotion makeMotion(const Transform& a, const Transform& b) {
    gnd::InstMotion k{};
    gnd::motionDecompose(a.m.toXf34(), k.t0, k.s0, k.q0);
    gnd::motionDecompose(b.m.toXf34(), k.t1, k.s1, k.q1);
    k.endO2W = b.m.toXf34();
    k.endW2O = b.mInv.toXf34();
    return k;
}
Transform motionMid(const gnd::InstMotion& k) {
    gnd::Xf34 m, mi;
    gnd::motionCompose(k, (0.5f - 0.0f) / (1.0f - 0.0f), m, mi);
    Transform t;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) {
            t.m.c[c][r] = m.r[r][c];
            t.mInv.c[c][r] = mi.r[r][c];
        }
    return t;
}
void PrimitiveObj::addChild(std::shared_ptr<GndObject> c) {
    switch (c->getClassType()) {
        case EShape:
            if (shape) throw std::runtime_error("Primitive: shape already registered!");
            shape = std::static_pointer_cast<ShapeObj>(c);
            break;
        case EMaterial:
            if (material) throw std::runtime_error("Primitive: material already registered!");
            material = std::static_pointer_cast<MaterialObj>(c);
            break;
        case EEmitter:
            if (emitter) throw std::runtime_error("Primitive: emitter already registered!");
            emitter = std::static_pointer_cast<EmitterObj>(c);
            break;
        default:
            throw std::runtime_error("Primitive: invalid child class! Expected Shape.");
    }
}
void PrimitiveObj::activate() {
    if (!shape) throw std::runtime_error("Primitive: defined without a Shape!");
    if (!material) {
        auto m = std::make_shared<MatteMat>(PropertyList());
        m->activate();
        material = m;
    }
}
struct PrimitiveReg : PrimitiveObj {
    explicit PrimitiveReg(const PropertyList& p) : PrimitiveObj(p) {}
};
GND_REGISTER_CLASS(PrimitiveReg, "primitive")

// ---------------------------------------------------------------- camera, filters, sampler
CameraObj::CameraObj(const PropertyList& p) {
    toWorld = p.getTransform("toWorld", Transform());
    toWorldEnd = p.getTransform("toWorldEnd", toWorld);   // camera.h:20-25
    animated = !(toWorldEnd == toWorld);
    width = p.getInteger("width", 1280);
    height = p.getInteger("height", 720);
    fov = p.getFloat("fov", 45.0f);
}
void CameraObj::addChild(std::shared_ptr<GndObject> c) {
    if (c->getClassType() == EFilter) {
        if (filter) throw std::runtime_error("Camera: cannot define multiple films!");
        filter = std::static_pointer_cast<FilterObj>(c);
    }
}
struct PerspectiveCameraObj : CameraObj {
    explicit PerspectiveCameraObj(const PropertyList& p) : CameraObj(p) {}
};
// thinLens.cpp:13-31
struct ThinLensCameraObj : CameraObj {
    explicit ThinLensCameraObj(const PropertyList& p) : CameraObj(p) {
        kind = gnd::kCamThinLens;
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
};
// filter.h:20-54
struct BoxFilterObj : FilterObj {
    explicit BoxFilterObj(const PropertyList&) { type = 0; rx = ry = 0.5f; }
};
struct GaussianFilterObj : FilterObj {
    explicit GaussianFilterObj(const PropertyList& p) {
        type = 1;
        V2 r = p.getVector2("radius", V2{2.f, 2.f});
        rx = r.x; ry = r.y;
        alpha = p.getFloat("alpha", 2.0f);
    }
};
struct IndependentSamplerObj : SamplerObj {
    explicit IndependentSamplerObj(const PropertyList& p) : SamplerObj(p) {}
};
GND_REGISTER_CLASS(PerspectiveCameraObj, "perspective")
GND_REGISTER_CLASS(ThinLensCameraObj, "thinlens")
GND_REGISTER_CLASS(BoxFilterObj, "box")
GND_REGISTER_CLASS(GaussianFilterObj, "gaussian")
GND_REGISTER_CLASS(IndependentSamplerObj, "independent")
struct SceneReg : Scene {
    explicit SceneReg(const PropertyList& p) : Scene(p) {}
};
GND_REGISTER_CLASS(SceneReg, "scene")

// ---------------------------------------------------------------- scene
// scene.cpp:9-44
void Scene::addChild(std::shared_ptr<GndObject> c) {
    switch (c->getClassType()) {
        case EPrimitive: {
            auto prim = std::static_pointer_cast<PrimitiveObj>(c);
            if (prim->emitter) m_emitterOrder.push_back(EmitterEntry{(int)m_primitives.size(), nullptr});
            m_primitives.push_back(prim);
            break;
        }
        case ECamera:
            if (m_camera) throw std::runtime_error("Scene: cannot add multiple cameras!");
            m_camera = std::static_pointer_cast<CameraObj>(c);
            break;
        case EIntegrator:
            if (m_integrator) throw std::runtime_error("Scene: cannot add multiple integrators!");
            m_integrator = std::static_pointer_cast<Integrator>(c);
            break;
        case ESampler:
            if (m_sampler) throw std::runtime_error("Scene: cannot add multiple samplers!");
            m_sampler = std::static_pointer_cast<SamplerObj>(c);
            break;
        case EEmitter: {   // scene.cpp:33-40
            auto em = std::static_pointer_cast<EmitterObj>(c);
            if (em->type == gnd::kEmitArea) throw std::runtime_error("Scene: an area emitter must be attached to a primitive");
            m_emitterOrder.push_back(EmitterEntry{-1, em});
            if (em->isInfiniteAreaLight()) {
                if (m_envMap) throw std::runtime_error("Scene: cannot add multiple infinite area lights!");
                m_envMap = em;
            }
            break;
        }
        default:
            throw std::runtime_error("Scene: cannot add specified child!");
    }
}

// scene.cpp:46-62
void Scene::activate() {
    if (!m_camera) throw std::runtime_error("Scene: no camera specified!");
    if (!m_integrator) throw std::runtime_error("Scene: no integrator specified!");
    if (!m_sampler) throw std::runtime_error("Scene: no sampler specified!");
    build();
    if (!deferPreprocess) {
        ensureFilm();
        m_integrator->preprocess(this);
    }
}

// camera.h:63-66: the camera's film (its filter travels in the flattened scene). Scenes
// loaded only for their flattened description (deferPreprocess) get it when first rendered.
Film* Scene::ensureFilm() {
    if (!m_camera) throw std::runtime_error("Scene: no camera specified!");
    if (!m_camera->film) {
        m_camera->film = std::make_unique<Film>(m_camera->width, m_camera->height);
        m_camera->film->outputPath = outputPath;
        m_camera->film->outputName = outputName;
    }
    return m_camera->film.get();
}

namespace {

struct MeshBuild {
    std::vector<gnd::Node4> nodes;   // node refs relative to this vector
    uint32_t root = gnd::kEmpty;
    std::vector<uint32_t> order;     // leaf order -> original triangle
};

template <typename F>
void parallelFor(size_t n, F&& f) {
    unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)n));
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (;;) {
            size_t i = next.fetch_add(1);
            if (i >= n) break;
            f(i);
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

}  // namespace

void Scene::build() {
    auto fs = std::make_unique<FlatScene>();
    // unique meshes, materials, media
    std::unordered_map<const ShapeObj*, int> meshIdx;
    std::vector<const ShapeObj*> meshes;
    std::unordered_map<const MaterialObj*, int> matIdx;
    std::unordered_map<const MediumObj*, int> medIdx;
    auto mediumIndex = [&](const std::shared_ptr<MediumObj>& m) -> int {
        if (!m) return -1;
        auto it = medIdx.find(m.get());
        if (it != medIdx.end()) return it->second;
        int k = (int)fs->media.size();
        fs->media.push_back(m->rec);
        medIdx[m.get()] = k;
        return k;
    };
    for (auto& p : m_primitives) {
        if (p->shape->kind == gnd::kShapeMesh && !meshIdx.count(p->shape.get())) {
            meshIdx[p->shape.get()] = (int)meshes.size();
            meshes.push_back(p->shape.get());
        }
    }
    // bottom-level trees, built in parallel per mesh
    std::vector<MeshBuild> mb(meshes.size());
    std::vector<uint32_t> triBase(meshes.size() + 1, 0);
    for (size_t i = 0; i < meshes.size(); ++i) {
        size_t nt = meshes[i]->numTris();
        if (triBase[i] + nt >= gnd::kLeafFirstMask) throw std::runtime_error("Scene: too many triangles for the device layout");
        triBase[i + 1] = triBase[i] + (uint32_t)nt;
    }
    int parDepth = meshes.size() == 1 ? 4 : 0;
    if (deviceBlas) {
        // the device builds the mesh trees: keep the original order
        parallelFor(meshes.size(), [&](size_t i) {
            mb[i].order.resize(meshes[i]->numTris());
            for (size_t t = 0; t < mb[i].order.size(); ++t) mb[i].order[t] = (uint32_t)t;
        });
    } else parallelFor(meshes.size(), [&](size_t i) {
        const ShapeObj& m = *meshes[i];
        size_t nt = m.numTris();
        std::vector<Bounds> pb(nt);
        std::vector<V3> pc(nt);
        for (size_t t = 0; t < nt; ++t) {
            Bounds b;
            b.grow(m.positions[3 * t]); b.grow(m.positions[3 * t + 1]); b.grow(m.positions[3 * t + 2]);
            pb[t] = b;
            pc[t] = b.centroid();
        }
        BinTree bt = buildSAH(pb, pc, parDepth);
        mb[i].root = collapseToNode4(bt, triBase[i], pb, mb[i].nodes);
        mb[i].order = std::move(bt.order);
    });
    // top-level tree over primitive world bounds (bvh.cpp:10-36); it goes first
    size_t np = m_primitives.size();
    std::vector<Bounds> wb(np);
    std::vector<V3> wc(np);
    parallelFor(np, [&](size_t i) {
        const PrimitiveObj& pr = *m_primitives[i];
        const Bounds ob = pr.shape->objectBounds();
        wb[i] = ob.transformed(pr.toWorld);
        if (pr.animated) {   // motionBounds (animated.cpp:49-58): start, end and the middle
            wb[i].grow(ob.transformed(pr.toWorldEnd));
            wb[i].grow(ob.transformed(motionMid(makeMotion(pr.toWorld, pr.toWorldEnd))));
        }
        wc[i] = wb[i].lo * 0.5f + wb[i].hi * 0.5f;
    });
    if (np > 0) {
        BinTree tl = buildSAH(wb, wc, 0);
        std::vector<gnd::Node4> tlasNodes;
        fs->tlasRoot = collapseToNode4(tl, 0, wb, tlasNodes);
        fs->nodes.assign(tlasNodes.begin(), tlasNodes.end());
        fs->tlasList = tl.order;
    }
    // concatenate the meshes: every output offset first, then the meshes (node arrays,
    // area CDFs) and their triangles (in chunks of kChunk) written on all host cores
    const size_t nm = meshes.size();
    std::vector<uint32_t> blasRoot(nm);
    std::vector<size_t> nodeBase(nm + 1), cdfBase(nm + 1, 0);
    nodeBase[0] = fs->nodes.size();
    for (size_t i = 0; i < nm; ++i) {
        nodeBase[i + 1] = nodeBase[i] + mb[i].nodes.size();
        cdfBase[i + 1] = cdfBase[i] + meshes[i]->numTris() + 1;
        blasRoot[i] = mb[i].root == gnd::kEmpty ? gnd::kEmpty : mb[i].root + (uint32_t)nodeBase[i];
    }
    fs->nodes.resize(nodeBase[nm]);
    fs->tris.resize(triBase.back());
    fs->attrs.resize(triBase.back());
    fs->origToLeaf.resize(triBase.back());
    fs->cdf.resize(cdfBase[nm]);
    fs->meshes.resize(nm);
    parallelFor(nm, [&](size_t i) {
        const uint32_t base = (uint32_t)nodeBase[i];
        gnd::Node4* dst = fs->nodes.data() + base;
        for (gnd::Node4 n : mb[i].nodes) {   // inner-node references rebased
            for (int c = 0; c < 4; ++c)
                if (n.child[c] != gnd::kEmpty && !gnd::isLeaf(n.child[c])) n.child[c] += base;
            *dst++ = n;
        }
        const ShapeObj& m = *meshes[i];
        gnd::MeshRec& rec = fs->meshes[i];
        rec = gnd::MeshRec{};
        rec.cdfOffset = (uint32_t)cdfBase[i];
        rec.numTris = (uint32_t)m.numTris();
        rec.origToLeaf = triBase[i];
        // area CDF in original triangle order (mesh.cpp:120-145)
        float* cdf = fs->cdf.data() + cdfBase[i];
        cdf[0] = 0.0f;
        float total = 0.0f;
        for (size_t t = 0; t < m.numTris(); ++t) {
            V3 e1 = m.positions[3 * t + 1] - m.positions[3 * t];
            V3 e2 = m.positions[3 * t + 2] - m.positions[3 * t];
            total += 0.5f * gnd::length(gnd::cross(e1, e2));
            cdf[t + 1] = total;
        }
        if (total > 0.0f)
            for (size_t t = 1; t <= m.numTris(); ++t) cdf[t] /= total;
        rec.totalArea = total;
    });
    constexpr size_t kChunk = size_t(1) << 16;
    struct Piece { size_t mesh, lo, hi; };
    std::vector<Piece> pieces;
    for (size_t i = 0; i < nm; ++i)
        for (size_t lo = 0; lo < meshes[i]->numTris(); lo += kChunk)
            pieces.push_back(Piece{i, lo, std::min(lo + kChunk, meshes[i]->numTris())});
    parallelFor(pieces.size(), [&](size_t k) {
        const size_t i = pieces[k].mesh;
        const ShapeObj& m = *meshes[i];
        bool hasN = !m.normals.empty(), hasUV = !m.uvs.empty();
        for (size_t s = pieces[k].lo; s < pieces[k].hi; ++s) {
            uint32_t orig = mb[i].order[s];
            uint32_t slot = triBase[i] + (uint32_t)s;
            fs->origToLeaf[triBase[i] + orig] = slot;
            const V3* P = &m.positions[3 * orig];
            gnd::Tri& t = fs->tris[slot];
            t.v0x = P[0].x; t.v0y = P[0].y; t.v0z = P[0].z; t.prim = orig;
            t.v1x = P[1].x; t.v1y = P[1].y; t.v1z = P[1].z; t.pad1 = 0;
            t.v2x = P[2].x; t.v2y = P[2].y; t.v2z = P[2].z; t.pad2 = 0;
            gnd::TriAttr& a = fs->attrs[slot];
            std::memset(&a, 0, sizeof(a));
            if (hasN) {
                const V3* N = &m.normals[3 * orig];
                a.n0x = N[0].x; a.n0y = N[0].y; a.n0z = N[0].z;
                a.n1x = N[1].x; a.n1y = N[1].y; a.n1z = N[1].z;
                a.n2x = N[2].x; a.n2y = N[2].y; a.n2z = N[2].z;
            }
            if (hasUV) {
                const V2* U = &m.uvs[3 * orig];
                a.u0 = U[0].x; a.v0_ = U[0].y; a.u1 = U[1].x; a.v1_ = U[1].y; a.u2 = U[2].x; a.v2_ = U[2].y;
            }
            a.flags = (float)((hasN ? 1 : 0) | (hasUV ? 2 : 0));
        }
    });
    // emitters in scene-file order (scene.cpp:9-43): area lights of primitives and the
    // standalone point, spot, directional and environment emitters
    std::vector<int32_t> primEmitter(np, -1);
    for (const EmitterEntry& en : m_emitterOrder) {
        gnd::Emitter e{};
        e.instance = -1;
        if (en.prim >= 0) {
            e.type = gnd::kEmitArea;
            e.instance = en.prim;
            const EmitterObj& o = *m_primitives[en.prim]->emitter;
            e.radiance = o.radiance;
            if (o.radianceTex && e.radiance.kind == gnd::kTexNode) e.radiance.node = (uint32_t)o.radianceTex->flatten(fs->textures);
            primEmitter[en.prim] = (int32_t)fs->emitters.size();
        } else {
            const EmitterObj& o = *en.emitter;
            e.type = o.type;
            e.cosTotal = o.cosTotal;
            e.cosFalloff = o.cosFalloff;
            e.pos[0] = o.position.x; e.pos[1] = o.position.y; e.pos[2] = o.position.z;
            e.dir[0] = o.direction.x; e.dir[1] = o.direction.y; e.dir[2] = o.direction.z;
            e.color[0] = o.color.x; e.color[1] = o.color.y; e.color[2] = o.color.z;
            e.strength = o.strength;
            if (o.type == gnd::kEmitEnv) {
                fs->envEmitter = (int)fs->emitters.size();
                fs->envWidth = o.envWidth;
                fs->envHeight = o.envHeight;
                fs->envTexels = o.envTexels;
                fs->envDist = o.envDist;
                fs->envMarginalIntegral = o.envMarginalIntegral;
                fs->envStrength = o.strength;
            }
        }
        fs->emitters.push_back(e);
    }
    // instances, materials
    for (size_t i = 0; i < np; ++i) {
        const PrimitiveObj& p = *m_primitives[i];
        gnd::InstTrav it{};
        gnd::InstShade is{};
        it.w2o = p.toWorld.mInv.toXf34();
        is.o2w = p.toWorld.m.toXf34();
        it.kind = p.shape->kind;
        if (p.animated) {   // the start matrices above; the motion record for times > 0
            if (fs->motion.empty()) fs->motion.resize(np);
            fs->motion[i] = makeMotion(p.toWorld, p.toWorldEnd);
            it.kind |= gnd::kInstAnimated;
        }
        it.blasRoot = gnd::kEmpty;
        is.meshId = 0xFFFFFFFFu;
        if (p.shape->kind == gnd::kShapeMesh) {
            int mi = meshIdx[p.shape.get()];
            it.blasRoot = blasRoot[mi];
            is.triBase = triBase[mi];
            is.meshId = (uint32_t)mi;
        } else if (p.shape->kind == gnd::kShapeSphere) {
            it.p0 = p.shape->radius;
            is.radius = p.shape->radius;
        } else {
            it.p0 = p.shape->extents.x;
            it.p1 = p.shape->extents.y;
            is.ext[0] = p.shape->extents.x; is.ext[1] = p.shape->extents.y; is.ext[2] = p.shape->extents.z;
        }
        const MaterialObj* mat = p.material.get();
        auto mit = matIdx.find(mat);
        if (mit == matIdx.end()) {
            int k = (int)fs->materials.size();
            gnd::Material m = mat->rec;
            if (mat->texA && m.a.kind == gnd::kTexNode) m.a.node = (uint32_t)mat->texA->flatten(fs->textures);
            if (mat->texB && m.b.kind == gnd::kTexNode) m.b.node = (uint32_t)mat->texB->flatten(fs->textures);
            m.roughTex = mat->roughTex ? 1u + (uint32_t)mat->roughTex->flatten(fs->textures) : 0u;
            m.etaTex = mat->etaTex ? 1u + (uint32_t)mat->etaTex->flatten(fs->textures) : 0u;
            m.kTex = mat->kTex ? 1u + (uint32_t)mat->kTex->flatten(fs->textures) : 0u;
            m.normalTex = mat->normalTex ? 1u + (uint32_t)mat->normalTex->flatten(fs->textures) : 0u;
            m.bumpTex = (mat->bumpTex && !mat->normalTex) ? 1u + (uint32_t)mat->bumpTex->flatten(fs->textures) : 0u;
            fs->materials.push_back(m);
            mit = matIdx.emplace(mat, k).first;
        }
        is.material = mit->second;
        // glass / index attach their media (material.h:119-126); others keep none
        bool attaches = mat->rec.type == gnd::kMatGlass || mat->rec.type == gnd::kMatIndex;
        is.hasMedia = (attaches && (mat->inside || mat->outside)) ? 1u : 0u;
        is.mediumIn = is.hasMedia ? mediumIndex(mat->inside) : -1;
        is.mediumOut = is.hasMedia ? mediumIndex(mat->outside) : -1;
        is.emitter = primEmitter[i];
        fs->instT.push_back(it);
        fs->instS.push_back(is);
    }
    // camera (perspective.cpp:9-12)
    if (m_camera) {
        fs->camera.toWorld = m_camera->toWorld.m.toXf34();
        fs->camera.width = m_camera->width;
        fs->camera.height = m_camera->height;
        fs->camera.scale = std::tan((gnd::kPi / 180.f) * (m_camera->fov * 0.5f));
        fs->camera.aspect = m_camera->width / (float)m_camera->height;
        V3 org = m_camera->toWorld.point(gnd::v3s(0.0f));
        fs->camera.origin[0] = org.x; fs->camera.origin[1] = org.y; fs->camera.origin[2] = org.z;
        fs->camera.kind = m_camera->kind;
        fs->camera.blades = m_camera->blades;
        fs->camera.lensRadius = m_camera->lensRadius;
        fs->camera.focalDistance = m_camera->focalDistance;
        fs->camera.k1 = m_camera->k1;
        fs->camera.caAxial = m_camera->caAxial;
        fs->camera.caLateral = m_camera->caLateral;
        fs->camera.vignetting = m_camera->vignetting ? 1 : 0;
        fs->camera.rollingShutter = m_camera->rollingShutter ? 1 : 0;
        fs->camera.scanDuration = m_camera->scanDuration;
        fs->camera.exposureDuration = m_camera->exposureDuration;
        fs->camera.animated = m_camera->animated ? 1 : 0;
        if (m_camera->animated) fs->camera.motion = makeMotion(m_camera->toWorld, m_camera->toWorldEnd);
    }
    fs->fillDesc();
    gnd_scene_desc& d = fs->desc;
    d.width = m_camera ? m_camera->width : 0;
    d.height = m_camera ? m_camera->height : 0;
    d.spp = m_sampler ? m_sampler->spp : 1;
    d.max_depth = m_integrator ? m_integrator->maxDepth : 1000;
    d.integrator = m_integrator ? m_integrator->kind : 0;
    auto filt = m_camera ? m_camera->filter : nullptr;
    d.filter = filt ? filt->type : 1;   // film.cpp:29: Gaussian when no filter is given
    d.filter_radius[0] = filt ? filt->rx : 2.f;
    d.filter_radius[1] = filt ? filt->ry : 2.f;
    d.filter_alpha = filt ? filt->alpha : 2.f;
    d.blas_on_device = deviceBlas ? 1 : 0;
    m_flat = std::move(fs);
}

void FlatScene::fillDesc() {
    desc.nodes = nodes.data();
    desc.num_nodes = (int64_t)nodes.size();
    desc.tris = tris.data();
    desc.tri_attrs = attrs.data();
    desc.num_tris = (int64_t)tris.size();
    desc.inst_trav = instT.data();
    desc.inst_shade = instS.data();
    desc.num_instances = (int32_t)instT.size();
    desc.tlas_root = tlasRoot;
    desc.tlas_list = tlasList.data();
    desc.tlas_list_len = (int64_t)tlasList.size();
    desc.materials = materials.data();
    desc.num_materials = (int32_t)materials.size();
    desc.emitters = emitters.data();
    desc.num_emitters = (int32_t)emitters.size();
    desc.media = media.data();
    desc.num_media = (int32_t)media.size();
    desc.meshes = meshes.data();
    desc.num_meshes = (int32_t)meshes.size();
    desc.cdf = cdf.data();
    desc.cdf_len = (int64_t)cdf.size();
    desc.orig_to_leaf = origToLeaf.data();
    desc.orig_to_leaf_len = (int64_t)origToLeaf.size();
    desc.camera = &camera;
    desc.inst_motion = motion.empty() ? nullptr : motion.data();
    desc.env_emitter = envEmitter;
    desc.env_width = envWidth;
    desc.env_height = envHeight;
    desc.env_marginal_integral = envMarginalIntegral;
    desc.env_strength = envStrength;
    desc.env_texels = envTexels.empty() ? nullptr : envTexels.data();
    desc.env_dist = envDist.empty() ? nullptr : envDist.data();
    desc.tex_nodes = textures.nodes.empty() ? nullptr : textures.nodes.data();
    desc.num_tex_nodes = (int32_t)textures.nodes.size();
    desc.tex_texels = textures.texels.empty() ? nullptr : textures.texels.data();
    desc.num_tex_texels = (int64_t)(textures.texels.size() / 4);
}

}  // namespace gndh
