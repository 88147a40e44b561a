// Oracle (test infrastructure only): the reference's procedural and image textures
// restated on the CPU: Perlin noise, fBm and turbulence (math/perlin.h), Worley noise
// (math/worley.h), the perlin / marble / wood / cellular textures (textures/*.h), the
// domain warp (domainWarp.h) and image textures (imageTexture.cpp, textureCache.h) read
// from OpenEXR (uncompressed) or PNG files.
#pragma once
#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "oscene.h"

namespace orc {

// perlin.h: Ken Perlin's improved noise with his published permutation table
namespace perlin {
extern const int P[512];
inline float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
inline float grad(int hash, float x, float y, float z) {
    int h = hash & 15;
    float u = h < 8 ? x : y;
    float v = h < 4 ? y : (h == 12 || h == 14) ? x : z;
    return ((h & 1) == 0 ? u : -u) + ((h & 2) == 0 ? v : -v);
}
inline float lerp(float t, float a, float b) { return (1.f - t) * a + t * b; }   // constants.h:41-44
inline float noise(const Vec3& p) {
    int X = static_cast<int>(std::floor(p.x)) & 255;
    int Y = static_cast<int>(std::floor(p.y)) & 255;
    int Z = static_cast<int>(std::floor(p.z)) & 255;
    float x = p.x - std::floor(p.x), y = p.y - std::floor(p.y), z = p.z - std::floor(p.z);
    float u = fade(x), v = fade(y), w = fade(z);
    int A = P[X] + Y, AA = P[A] + Z, AB = P[A + 1] + Z;
    int B = P[X + 1] + Y, BA = P[B] + Z, BB = P[B + 1] + Z;
    float g000 = grad(P[AA], x, y, z), g100 = grad(P[BA], x - 1.0f, y, z);
    float g010 = grad(P[AB], x, y - 1.0f, z), g110 = grad(P[BB], x - 1.0f, y - 1.0f, z);
    float g001 = grad(P[AA + 1], x, y, z - 1.0f), g101 = grad(P[BA + 1], x - 1.0f, y, z - 1.0f);
    float g011 = grad(P[AB + 1], x, y - 1.0f, z - 1.0f), g111 = grad(P[BB + 1], x - 1.0f, y - 1.0f, z - 1.0f);
    float x00 = lerp(u, g000, g100), x10 = lerp(u, g010, g110), x01 = lerp(u, g001, g101), x11 = lerp(u, g011, g111);
    float y0 = lerp(v, x00, x10), y1 = lerp(v, x01, x11);
    return lerp(w, y0, y1);
}
inline float turbulence(const Vec3& p, int octaves) {
    float accum = 0.0f, weight = 1.0f;
    Vec3 t = p;
    for (int i = 0; i < octaves; ++i) {
        accum += weight * std::abs(noise(t));
        weight *= 0.5f;
        t = t * 2.0f;
    }
    return std::clamp(accum, 0.0f, 1.0f);
}
}  // namespace perlin

// worley.h
namespace worley {
inline Vec3 hash3(int x, int y, int z) {
    auto hash1 = [](uint32_t n) {
        n = (n << 13U) ^ n;
        n = n * (n * n * 15731U + 789221U) + 1376312589U;
        return float(n & 0x7fffffffU) / float(0x7fffffff);
    };
    uint32_t n = (uint32_t)x * 73856093U ^ (uint32_t)y * 19349663U ^ (uint32_t)z * 83492791U;
    return Vec3(hash1(n), hash1(n + 1), hash1(n + 2));
}
inline void noise(const Vec3& p, int metric, float& f1, float& f2) {
    int x0 = (int)std::floor(p.x), y0 = (int)std::floor(p.y), z0 = (int)std::floor(p.z);
    f1 = 1e8f;
    f2 = 1e8f;
    for (int k = -1; k <= 1; ++k)
        for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i) {
                int cx = x0 + i, cy = y0 + j, cz = z0 + k;
                Vec3 fp = Vec3((float)cx, (float)cy, (float)cz) + hash3(cx, cy, cz);
                Vec3 diff = p - fp;
                float dist;
                if (metric == 0) dist = diff.length();
                else if (metric == 1) dist = std::abs(diff.x) + std::abs(diff.y) + std::abs(diff.z);
                else dist = std::max({std::abs(diff.x), std::abs(diff.y), std::abs(diff.z)});
                if (dist < f1) { f2 = f1; f1 = dist; }
                else if (dist < f2) f2 = dist;
            }
}
}  // namespace worley

template <typename T>
inline T texLerp(float t, const T& a, const T& b) {   // m_value1 * (1 - t) + m_value2 * t
    return a * (1.0f - t) + b * t;
}

// perlin.h (texture): value1 .. value2 by turbulence(p / scale)
template <typename T>
struct PerlinTexture : Texture<T> {
    T v1, v2;
    float scale;
    int octaves;
    explicit PerlinTexture(const PropertyList& p);
    T evaluate(const SurfaceInteraction& si) const override {
        float n = perlin::turbulence(si.p / scale, octaves);
        if constexpr (std::is_same_v<T, float>) return std::lerp(v1, v2, n);
        else return texLerp(n, v1, v2);
    }
};
// marble.h
template <typename T>
struct MarbleTexture : Texture<T> {
    T v1, v2;
    float scale, veinFreq, turbScale;
    int octaves;
    Vec3 axis;
    explicit MarbleTexture(const PropertyList& p);
    T evaluate(const SurfaceInteraction& si) const override {
        float turb = perlin::turbulence(si.p / scale, octaves);
        float val = Dot(si.p, axis) + turb * turbScale;
        float sineval = std::sin(val * veinFreq);
        float t = 0.5f * (1.0f + sineval);
        if constexpr (std::is_same_v<T, float>) return std::lerp(v1, v2, t);
        else return texLerp(t, v1, v2);
    }
};
// wood.h
template <typename T>
struct WoodTexture : Texture<T> {
    T v1, v2;
    float scale, veinFreq, turbScale;
    int octaves;
    Vec3 axis;
    explicit WoodTexture(const PropertyList& p);
    T evaluate(const SurfaceInteraction& si) const override {
        float turb = perlin::turbulence(si.p / scale, octaves);
        float radius = Cross(si.p, axis).length();
        radius += turb * turbScale;
        float t = std::abs(std::sin(radius * veinFreq));
        if constexpr (std::is_same_v<T, float>) return std::lerp(v1, v2, t);
        else return texLerp(t, v1, v2);
    }
};
// cellular.h
template <typename T>
struct CellularTexture : Texture<T> {
    T v1, v2;
    float scale;
    int cracks, metric;
    explicit CellularTexture(const PropertyList& p);
    T evaluate(const SurfaceInteraction& si) const override {
        float f1, f2;
        worley::noise(si.p / scale, metric, f1, f2);
        float n = cracks ? f2 - f1 : f1;
        n = std::clamp(n, 0.0f, 1.0f);
        return (1.f - n) * v1 + n * v2;   // Lerp (constants.h:41-44)
    }
};
// domainWarp.h
template <typename T>
struct DomainWarpTexture : Texture<T> {
    float strength;
    std::shared_ptr<Texture<T>> base;
    std::shared_ptr<Texture<Color>> warp;
    explicit DomainWarpTexture(const PropertyList& p) : strength(p.getFloat("strength", 1.0f)) {}
    void addChild(ObjectPtr c) override;
    void activate() override;
    T evaluate(const SurfaceInteraction& si) const override {
        Color w = warp->evaluate(si);
        Vec3 d((w.r * 2.0f - 1.0f) * strength, (w.g * 2.0f - 1.0f) * strength, (w.b * 2.0f - 1.0f) * strength);
        SurfaceInteraction ws = si;
        ws.p = si.p + d;
        Vec3 dpdv = Cross(si.n, si.dpdu);
        float lu = si.dpdu.lengthSquared(), lv = dpdv.lengthSquared();
        float du = (lu > 0.0f) ? Dot(d, si.dpdu) / lu : 0.0f;
        float dv = (lv > 0.0f) ? Dot(d, dpdv) / lv : 0.0f;
        ws.uv.x += du;
        ws.uv.y += dv;
        return base->evaluate(ws);
    }
};
// uncompressed scanline OpenEXR, R, G, B (oobjects.cpp)
void loadEXR(const std::string& path, int& w, int& h, std::vector<Color>& px);

// imageTexture.cpp + textureCache.h
struct ImageData {
    int width = 0, height = 0, channels = 0;
    std::vector<float> data;
};
std::shared_ptr<ImageData> loadTextureImage(const std::string& path, bool srgb);
template <typename T>
struct ImageTexture : Texture<T> {
    std::string filename, baseDir;
    bool linear = false, clamp = false, srgb = false;
    bool normal = false;   // image_normal (imageTexture.cpp:101-104)
    std::shared_ptr<ImageData> img;
    explicit ImageTexture(const PropertyList& p);
    void setBaseDir(const std::string& d) override { baseDir = d; }
    void activate() override;
    Vec2 getUV(const Vec2& uv) const {
        if (clamp) return Vec2(std::clamp(uv.x, 0.0f, 1.0f), std::clamp(uv.y, 0.0f, 1.0f));
        return Vec2(uv.x - std::floor(uv.x), uv.y - std::floor(uv.y));
    }
    T extract(int x, int y) const {
        int w = img->width, h = img->height, c = img->channels;
        if (!clamp) { x = ((x % w) + w) % w; y = ((y % h) + h) % h; }
        else { x = std::clamp(x, 0, w - 1); y = std::clamp(y, 0, h - 1); }
        const float* ptr = &img->data[(size_t)(y * w + x) * c];
        if constexpr (std::is_same_v<T, float>) return ptr[0];
        else if (normal) return c >= 3 ? Color(ptr[0] * 2.0f - 1.0f, ptr[1] * 2.0f - 1.0f, ptr[2] * 2.0f - 1.0f) : Color(0.0f, 0.0f, 1.0f);
        else return c >= 3 ? Color(ptr[0], ptr[1], ptr[2]) : Color(ptr[0]);
    }
    T evaluate(const SurfaceInteraction& si) const override {
        Vec2 l = getUV(si.uv);
        if (!linear) return extract((int)std::floor(l.x * img->width), (int)std::floor(l.y * img->height));
        int w = img->width, h = img->height;
        float xc = l.x * w - 0.5f, yc = l.y * h - 0.5f;
        int x0 = (int)std::floor(xc), y0 = (int)std::floor(yc);
        float tx = xc - (float)x0, ty = yc - (float)y0;
        T c00 = extract(x0, y0), c10 = extract(x0 + 1, y0), c01 = extract(x0, y0 + 1), c11 = extract(x0 + 1, y0 + 1);
        T top = c00 * (1.0f - tx) + c10 * tx;
        T bottom = c01 * (1.0f - tx) + c11 * tx;
        return top * (1.0f - ty) + bottom * ty;
    }
};

}  // namespace orc
