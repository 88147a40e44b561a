// Oracle (test infrastructure only): constructors, the permutation table and the image
// loading of otextures.h.
#include "otextures.h"

#include <zlib.h>

#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <stdexcept>

namespace orc {

// perlin.h:98-121: Ken Perlin's published permutation of 0..255, repeated to avoid modulos
#define ORC_PERLIN_PERM                                                                                                    \
    151, 160, 137, 91, 90, 15, 131, 13, 201, 95, 96, 53, 194, 233, 7, 225, 140, 36, 103, 30, 69, 142, 8, 99, 37, 240, 21,  \
        10, 23, 190, 6, 148, 247, 120, 234, 75, 0, 26, 197, 62, 94, 252, 219, 203, 117, 35, 11, 32, 57, 177, 33, 88, 237,  \
        149, 56, 87, 174, 20, 125, 136, 171, 168, 68, 175, 74, 165, 71, 134, 139, 48, 27, 166, 77, 146, 158, 231, 83, 111, \
        229, 122, 60, 211, 133, 230, 220, 105, 92, 41, 55, 46, 245, 40, 244, 102, 143, 54, 65, 25, 63, 161, 1, 216, 80, 73, \
        209, 76, 132, 187, 208, 89, 18, 169, 200, 196, 135, 130, 116, 188, 159, 86, 164, 100, 109, 198, 173, 186, 3, 64,   \
        52, 217, 226, 250, 124, 123, 5, 202, 38, 147, 118, 126, 255, 82, 85, 212, 207, 206, 59, 227, 47, 16, 58, 17, 182,   \
        189, 28, 42, 223, 183, 170, 213, 119, 248, 152, 2, 44, 154, 163, 70, 221, 153, 101, 155, 167, 43, 172, 9, 129, 22,  \
        39, 253, 19, 98, 108, 110, 79, 113, 224, 232, 178, 185, 112, 104, 218, 246, 97, 228, 251, 34, 242, 193, 238, 210,   \
        144, 12, 191, 179, 162, 241, 81, 51, 145, 235, 249, 14, 239, 107, 49, 192, 214, 31, 181, 199, 106, 157, 184, 84,    \
        204, 176, 115, 121, 50, 45, 127, 4, 150, 254, 138, 236, 205, 93, 222, 114, 67, 29, 24, 72, 243, 141, 128, 195, 78,  \
        66, 215, 61, 156, 180
const int perlin::P[512] = {ORC_PERLIN_PERM, ORC_PERLIN_PERM};
#undef ORC_PERLIN_PERM

template <typename T>
static void values(const PropertyList& p, T& v1, T& v2, float d1, float d2, Color c1, Color c2) {
    if constexpr (std::is_same_v<T, float>) { v1 = p.getFloat("value1", d1); v2 = p.getFloat("value2", d2); }
    else { v1 = p.getColor("value1", c1); v2 = p.getColor("value2", c2); }
}

template <typename T>
PerlinTexture<T>::PerlinTexture(const PropertyList& p) {   // perlin.h:15-27
    values(p, v1, v2, 0.0f, 1.0f, Color(0.0f), Color(1.0f));
    scale = p.getFloat("scale", 1.0f);
    octaves = p.getInteger("octaves", 6);
}
template <typename T>
MarbleTexture<T>::MarbleTexture(const PropertyList& p) {   // marble.h:15-33
    values(p, v1, v2, 0.0f, 1.0f, Color(0.1f), Color(0.9f));
    scale = p.getFloat("scale", 1.0f);
    octaves = p.getInteger("octaves", 6);
    veinFreq = p.getFloat("vein_freq", 10.0f);
    turbScale = p.getFloat("turb_scale", 5.0f);
    axis = Normalize(p.getVector3("axis", Vec3(0.0f, 1.0f, 0.0f)));
}
template <typename T>
WoodTexture<T>::WoodTexture(const PropertyList& p) {   // wood.h:15-33
    values(p, v1, v2, 0.0f, 1.0f, Color(0.6f, 0.4f, 0.2f), Color(0.3f, 0.15f, 0.05f));
    scale = p.getFloat("scale", 1.0f);
    octaves = p.getInteger("octaves", 6);
    veinFreq = p.getFloat("vein_freq", 10.0f);
    turbScale = p.getFloat("turb_scale", 2.0f);
    axis = Normalize(p.getVector3("axis", Vec3(0.0f, 1.0f, 0.0f)));
}
template <typename T>
CellularTexture<T>::CellularTexture(const PropertyList& p) {   // cellular.h:17-45
    values(p, v1, v2, 0.0f, 1.0f, Color(0.0f), Color(1.0f));
    scale = p.getFloat("scale", 1.0f);
    cracks = p.getString("mode", "distance") == "cracks" ? 1 : 0;
    const std::string m = p.getString("metric", "euclidean");
    metric = m == "manhattan" ? 1 : (m == "chebyshev" ? 2 : 0);
}
template <typename T>
void DomainWarpTexture<T>::addChild(ObjectPtr c) {   // domainWarp.h:18-31
    if (c->classType() != ETexture) throw std::runtime_error("WarpTexture: cannot add specified child!");
    if (c->name == "base") {
        if (base) throw std::runtime_error("WarpTexture: base texture already defined!");
        base = std::static_pointer_cast<Texture<T>>(c);
    } else if (c->name == "warp") {
        if (warp) throw std::runtime_error("WarpTexture: warp texture already defined!");
        warp = std::static_pointer_cast<Texture<Color>>(c);
    }
}
template <typename T>
void DomainWarpTexture<T>::activate() {
    if (!base) throw std::runtime_error("WarpTexture: missing base texture!");
    if (!warp) throw std::runtime_error("WarpTexture: missing warp texture!");
}
template <typename T>
ImageTexture<T>::ImageTexture(const PropertyList& p) {   // imageTexture.cpp:11-32
    filename = p.getString("filename");
    const std::string interp = p.getString("interpolation_mode", "closest");
    if (interp == "closest") linear = false;
    else if (interp == "linear") linear = true;
    else throw std::runtime_error("ImageTexture: Unknown interpolation mode " + interp);
    const std::string cs = p.getString("color_space", "linear");
    if (cs == "sRGB") srgb = true;
    else if (cs == "linear") srgb = false;
    else throw std::runtime_error("ImageTexture: Unknown color space " + cs);
    const std::string rep = p.getString("repeat_mode", "repeat");
    if (rep == "repeat") clamp = false;
    else if (rep == "clamp") clamp = true;
    else throw std::runtime_error("ImageTexture: Unknown repeat mode " + rep);
}
template <typename T>
void ImageTexture<T>::activate() {
    std::filesystem::path abs(filename);
    if (abs.is_relative()) abs = std::filesystem::path(baseDir) / abs;
    img = loadTextureImage(abs.string(), srgb);
}

template struct PerlinTexture<Color>;
template struct PerlinTexture<float>;
template struct MarbleTexture<Color>;
template struct MarbleTexture<float>;
template struct WoodTexture<Color>;
template struct WoodTexture<float>;
template struct CellularTexture<Color>;
template struct CellularTexture<float>;
template struct DomainWarpTexture<Color>;
template struct DomainWarpTexture<float>;
template struct ImageTexture<Color>;
template struct ImageTexture<float>;

// PNG: 8- or 16-bit greyscale, grey + alpha, RGB or RGBA, not interlaced; rows unfiltered
// (none, sub, up, average, Paeth) from one zlib stream; 16-bit samples keep their high
// byte (stb's conversion to 8 bits).
static void loadPNG(const std::string& path, int& w, int& h, int& channels, std::vector<uint8_t>& px) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("TextureCache: Failed to load image " + path);
    std::vector<uint8_t> d((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (d.size() < 8 || std::memcmp(d.data(), sig, 8) != 0) throw std::runtime_error("TextureCache: Failed to load image " + path);
    auto be32 = [&](size_t at) {
        if (at + 4 > d.size()) throw std::runtime_error("PNG: truncated");
        return (uint32_t)d[at] << 24 | (uint32_t)d[at + 1] << 16 | (uint32_t)d[at + 2] << 8 | d[at + 3];
    };
    size_t pos = 8;
    int depth = 0, ctype = 0, inter = 0;
    std::vector<uint8_t> z;
    for (;;) {
        uint32_t n = be32(pos);
        if (pos + 12 + n > d.size()) throw std::runtime_error("PNG: truncated");
        std::string type(reinterpret_cast<const char*>(&d[pos + 4]), 4);
        const uint8_t* body = &d[pos + 8];
        if (type == "IHDR") {
            w = (int)be32(pos + 8);
            h = (int)be32(pos + 12);
            depth = body[8];
            ctype = body[9];
            inter = body[12];
        } else if (type == "IDAT") {
            z.insert(z.end(), body, body + n);
        } else if (type == "IEND") {
            break;
        }
        pos += 12 + n;
    }
    if (inter != 0 || (depth != 8 && depth != 16)) throw std::runtime_error("PNG: only 8/16-bit non-interlaced images");
    channels = ctype == 0 ? 1 : ctype == 4 ? 2 : ctype == 2 ? 3 : ctype == 6 ? 4 : 0;
    if (!channels) throw std::runtime_error("PNG: unsupported colour type");
    const size_t bpp = (size_t)channels * (depth / 8), stride = (size_t)w * bpp;
    std::vector<uint8_t> raw((stride + 1) * h);
    uLongf len = (uLongf)raw.size();
    if (uncompress(raw.data(), &len, z.data(), (uLong)z.size()) != Z_OK || len != raw.size())
        throw std::runtime_error("PNG: corrupt image data");
    std::vector<uint8_t> img(stride * h), prev(stride, 0);
    for (int y = 0; y < h; ++y) {
        const uint8_t ft = raw[y * (stride + 1)];
        const uint8_t* in = &raw[y * (stride + 1) + 1];
        uint8_t* out = &img[y * stride];
        for (size_t i = 0; i < stride; ++i) {
            const int a = i >= bpp ? out[i - bpp] : 0, b = prev[i], c = i >= bpp ? prev[i - bpp] : 0;
            int v = in[i];
            if (ft == 1) v += a;
            else if (ft == 2) v += b;
            else if (ft == 3) v += (a + b) / 2;
            else if (ft == 4) {
                const int pp = a + b - c, pa = std::abs(pp - a), pb = std::abs(pp - b), pc = std::abs(pp - c);
                v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
            }
            out[i] = (uint8_t)v;
        }
        std::memcpy(prev.data(), out, stride);
    }
    px.resize((size_t)w * h * channels);
    const size_t step = depth / 8;
    for (size_t i = 0; i < px.size(); ++i) px[i] = img[i * step];   // 16 bit: the high byte
}

extern "C" float orc_round_half(float x);   // opost.cpp: float -> binary16 -> float

// textureCache.h:23-95: EXR files as RGBA halves, other files 8-bit with the optional
// sRGB decode of colour channels; both flipped vertically (row 0 = the bottom row).
std::shared_ptr<ImageData> loadTextureImage(const std::string& path, bool srgb) {
    auto img = std::make_shared<ImageData>();
    if (path.size() >= 4 && path.compare(path.size() - 4, 4, ".exr") == 0) {
        std::vector<Color> px;
        loadEXR(path, img->width, img->height, px);
        img->channels = 4;
        img->data.resize((size_t)img->width * img->height * 4);
        for (int y = 0; y < img->height; ++y) {
            const int dy = img->height - 1 - y;
            for (int x = 0; x < img->width; ++x) {
                const Color& c = px[(size_t)y * img->width + x];
                float* o = &img->data[((size_t)dy * img->width + x) * 4];
                // Imf::RgbaInputFile reads into half-precision Rgba pixels
                o[0] = orc_round_half(c.r); o[1] = orc_round_half(c.g); o[2] = orc_round_half(c.b); o[3] = 1.0f;
            }
        }
        return img;
    }
    std::vector<uint8_t> px;
    loadPNG(path, img->width, img->height, img->channels, px);
    const int w = img->width, h = img->height, c = img->channels;
    img->data.resize(px.size());
    auto toLinear = [](float v) { return v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f); };
    for (int y = 0; y < h; ++y) {
        const int sy = h - 1 - y;   // stbi_set_flip_vertically_on_load(true)
        for (int i = 0; i < w * c; ++i) {
            const size_t k = (size_t)y * w * c + i;
            float v = px[(size_t)sy * w * c + i] / 255.0f;
            if (srgb && (c <= 3 || (int)(k % c) < 3)) v = toLinear(v);
            img->data[k] = v;
        }
    }
    return img;
}

}  // namespace orc

// Ken Perlin's permutation table as the oracle holds it (512 entries)
extern "C" void orc_perlin_perm(int32_t* out) {
    for (int i = 0; i < 512; ++i) out[i] = orc::perlin::P[i];
}

// Texture probe: a scene file whose root element is a color or float texture, evaluated at
// n surface points given as p (3), n (3), dpdu (3), uv (2); out: rgb (float textures
// repeat their value). Returns 0, or -1 with the message in err.
extern "C" int orc_tex_eval(const char* path, int64_t n, const float* pts, float* out, char* err, int errlen) {
    using namespace orc;
    try {
        auto obj = loadSceneXML(path);
        auto ct = std::dynamic_pointer_cast<Texture<Color>>(obj);
        auto ft = std::dynamic_pointer_cast<Texture<float>>(obj);
        if (!ct && !ft) throw std::runtime_error("root element is not a texture");
        for (int64_t i = 0; i < n; ++i) {
            const float* q = pts + 11 * i;
            SurfaceInteraction si;
            si.p = Vec3(q[0], q[1], q[2]);
            si.n = Vec3(q[3], q[4], q[5]);
            si.dpdu = Vec3(q[6], q[7], q[8]);
            si.uv = Vec2(q[9], q[10]);
            if (ct) {
                Color c = ct->evaluate(si);
                out[3 * i] = c.r; out[3 * i + 1] = c.g; out[3 * i + 2] = c.b;
            } else {
                out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = ft->evaluate(si);
            }
        }
        return 0;
    } catch (const std::exception& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return -1;
    }
}
