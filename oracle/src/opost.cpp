// Oracle (test infrastructure only): CPU restatement of the reference's post-processing,
// the GLSL passes that postProcessor.cpp:148-235 runs on the film (bloom_prefilter.frag,
// bloom_downsample.frag, bloom_upsample.frag, tonemap.frag, gammaCorrect.frag) and the
// 8-bit conversion of Film::savePNG (film.cpp:154-171, color.h:84-95).
//
// The shaders run through OpenGL, which is unavailable here, so their arithmetic is
// restated with the texture unit made explicit: GL_LINEAR sampling with exact fp32
// weights, clamp to edge, texel centres at (i + 0.5) / size; the bloom pyramid's RGB16F
// targets round every stored value to binary16 (round to nearest even); the additive
// blend of the upsample pass adds in fp32 and stores to binary16. Matrix-vector products
// and dot products sum left to right.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Tex {
    int w = 0, h = 0;
    std::vector<float> px;   // rgb per texel, row-major
    const float* at(int x, int y) const { return &px[3 * ((size_t)y * w + x)]; }
};

// float -> binary16 -> float, round to nearest even (IEEE 754 conversion)
float roundHalf(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t sign = u & 0x80000000u;
    uint32_t a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return f;                                   // inf, NaN
    if (a >= 0x477ff000u) return sign ? -INFINITY : INFINITY;         // >= 65520: overflow
    if (a < 0x38800000u) {                                            // below 2^-14: subnormal
        const float q = std::nearbyint(std::fabs(f) * 16777216.0f) * (1.0f / 16777216.0f);
        return sign ? -q : q;
    }
    a += 0x0fffu + ((a >> 13) & 1u);
    a &= ~0x1fffu;
    a |= sign;
    float r;
    std::memcpy(&r, &a, 4);
    return r;
}

// GL_LINEAR sample at texture coordinate (u, v), clamp to edge
void sample(const Tex& t, float u, float v, float out[3]) {
    const float x = u * (float)t.w - 0.5f, y = v * (float)t.h - 0.5f;
    const float x0f = std::floor(x), y0f = std::floor(y);
    const float fx = x - x0f, fy = y - y0f;
    const int x0 = std::clamp((int)x0f, 0, t.w - 1), x1 = std::clamp((int)x0f + 1, 0, t.w - 1);
    const int y0 = std::clamp((int)y0f, 0, t.h - 1), y1 = std::clamp((int)y0f + 1, 0, t.h - 1);
    const float *a = t.at(x0, y0), *b = t.at(x1, y0), *c = t.at(x0, y1), *d = t.at(x1, y1);
    for (int k = 0; k < 3; ++k) {
        const float c0 = a[k] * (1.0f - fx) + b[k] * fx;
        const float c1 = c[k] * (1.0f - fx) + d[k] * fx;
        out[k] = c0 * (1.0f - fy) + c1 * fy;
    }
}

// bloom_prefilter.frag
void prefilter(const Tex& src, Tex& dst, float threshold) {
    for (int j = 0; j < dst.h; ++j)
        for (int i = 0; i < dst.w; ++i) {
            float c[3];
            sample(src, ((float)i + 0.5f) / (float)dst.w, ((float)j + 0.5f) / (float)dst.h, c);
            const float bright = std::max(c[0], std::max(c[1], c[2]));
            float* o = &dst.px[3 * ((size_t)j * dst.w + i)];
            for (int k = 0; k < 3; ++k) o[k] = roundHalf(bright > threshold ? c[k] : 0.0f);
        }
}

// bloom_downsample.frag: 13 taps at 1 and 2 source texels
void downsample(const Tex& src, Tex& dst) {
    const float x = 1.0f / (float)src.w, y = 1.0f / (float)src.h;
    for (int j = 0; j < dst.h; ++j)
        for (int i = 0; i < dst.w; ++i) {
            const float u = ((float)i + 0.5f) / (float)dst.w, v = ((float)j + 0.5f) / (float)dst.h;
            float a[3], b[3], c[3], d[3], e[3], f[3], g[3], h[3], ii[3], jj[3], kk[3], ll[3], mm[3];
            sample(src, u - 2 * x, v + 2 * y, a);
            sample(src, u, v + 2 * y, b);
            sample(src, u + 2 * x, v + 2 * y, c);
            sample(src, u - 2 * x, v, d);
            sample(src, u, v, e);
            sample(src, u + 2 * x, v, f);
            sample(src, u - 2 * x, v - 2 * y, g);
            sample(src, u, v - 2 * y, h);
            sample(src, u + 2 * x, v - 2 * y, ii);
            sample(src, u - x, v + y, jj);
            sample(src, u + x, v + y, kk);
            sample(src, u - x, v - y, ll);
            sample(src, u + x, v - y, mm);
            float* o = &dst.px[3 * ((size_t)j * dst.w + i)];
            for (int k = 0; k < 3; ++k) {
                float s = e[k] * 0.125f;
                s += (((a[k] + c[k]) + g[k]) + ii[k]) * 0.03125f;
                s += (((b[k] + d[k]) + f[k]) + h[k]) * 0.0625f;
                s += (((jj[k] + kk[k]) + ll[k]) + mm[k]) * 0.125f;
                o[k] = roundHalf(s);
            }
        }
}

// bloom_upsample.frag with the additive blend (GL_ONE, GL_ONE) into dst
void upsampleAdd(const Tex& src, Tex& dst, float radius) {
    const float x = radius * (1.0f / (float)src.w), y = radius * (1.0f / (float)src.h);
    for (int j = 0; j < dst.h; ++j)
        for (int i = 0; i < dst.w; ++i) {
            const float u = ((float)i + 0.5f) / (float)dst.w, v = ((float)j + 0.5f) / (float)dst.h;
            float a[3], b[3], c[3], d[3], e[3], f[3], g[3], h[3], ii[3];
            sample(src, u - x, v + y, a);
            sample(src, u, v + y, b);
            sample(src, u + x, v + y, c);
            sample(src, u - x, v, d);
            sample(src, u, v, e);
            sample(src, u + x, v, f);
            sample(src, u - x, v - y, g);
            sample(src, u, v - y, h);
            sample(src, u + x, v - y, ii);
            float* o = &dst.px[3 * ((size_t)j * dst.w + i)];
            for (int k = 0; k < 3; ++k) {
                float s = e[k] * 4.0f;
                s += (((b[k] + d[k]) + f[k]) + h[k]) * 2.0f;
                s += (((a[k] + c[k]) + g[k]) + ii[k]) * 1.0f;
                s *= 1.0f / 16.0f;
                o[k] = roundHalf(o[k] + s);
            }
        }
}

// ---------------------------------------------------------------- tonemap.frag operators
struct V {
    float r, g, b;
};
V mul3(const float m[9], V c) {   // GLSL mat3(m0..m8) is column-major
    return V{(m[0] * c.r + m[3] * c.g) + m[6] * c.b, (m[1] * c.r + m[4] * c.g) + m[7] * c.b,
             (m[2] * c.r + m[5] * c.g) + m[8] * c.b};
}
float clamp01(float x) { return std::fmin(std::fmax(x, 0.0f), 1.0f); }

V reinhard(V c) {
    const float luma = (c.r * 0.2126f + c.g * 0.7152f) + c.b * 0.0722f;
    const float tl = luma / (1.0f + luma);
    const float s = tl / std::fmax(luma, 0.00001f);
    return V{c.r * s, c.g * s, c.b * s};
}
float u2curve(float x) {
    const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, F = 0.30f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
}
V uncharted2(V c) {
    const float bias = 2.0f;
    const float ws = 1.0f / u2curve(11.2f);
    return V{u2curve(bias * c.r) * ws, u2curve(bias * c.g) * ws, u2curve(bias * c.b) * ws};
}
const float kAcesIn[9] = {0.59719f, 0.07600f, 0.02840f, 0.35458f, 0.90834f, 0.13383f, 0.04823f, 0.01566f, 0.83777f};
const float kAcesOut[9] = {1.60475f, -0.10208f, -0.00327f, -0.53108f, 1.10813f, -0.07276f, -0.07367f, -0.00605f, 1.07602f};
float rrtOdt(float v) {
    const float a = v * (v + 0.0245786f) - 0.000090537f;
    const float b = v * (0.983729f * v + 0.432951f) + 0.238081f;
    return a / b;
}
V aces(V c) {
    c = mul3(kAcesIn, c);
    c = V{rrtOdt(c.r), rrtOdt(c.g), rrtOdt(c.b)};
    c = mul3(kAcesOut, c);
    return V{clamp01(c.r), clamp01(c.g), clamp01(c.b)};
}
V khronos(V c) {
    const float startCompression = 0.8f - 0.04f;
    const float desaturation = 0.15f;
    const float x = std::fmin(c.r, std::fmin(c.g, c.b));
    const float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    c = V{c.r - offset, c.g - offset, c.b - offset};
    const float peak = std::fmax(c.r, std::fmax(c.g, c.b));
    if (peak < startCompression) return c;
    const float d = 1.0f - startCompression;
    const float newPeak = 1.0f - d * d / (peak + d - startCompression);
    const float s = newPeak / peak;
    c = V{c.r * s, c.g * s, c.b * s};
    const float g = 1.0f - 1.0f / (desaturation * (peak - newPeak) + 1.0f);
    // mix(c, vec3(newPeak), g) = c * (1 - g) + newPeak * g
    return V{c.r * (1.0f - g) + newPeak * g, c.g * (1.0f - g) + newPeak * g, c.b * (1.0f - g) + newPeak * g};
}
const float kRec2020ToSrgb[9] = {1.6605f, -0.1246f, -0.0182f, -0.5876f, 1.1329f, -0.1006f, -0.0728f, -0.0083f, 1.1187f};
const float kSrgbToRec2020[9] = {0.6274f, 0.0691f, 0.0164f, 0.3293f, 0.9195f, 0.0880f, 0.0433f, 0.0113f, 0.8956f};
const float kAgxInset[9] = {0.856627153315983f, 0.137318972929847f, 0.11189821299995f,
                            0.0951212405381588f, 0.761241990602591f, 0.0767994186031903f,
                            0.0482516061458583f, 0.101439036467562f, 0.811302368396859f};
const float kAgxOutset[9] = {1.1271005818144368f, -0.1413297634984383f, -0.14132976349843826f,
                             -0.11060664309660323f, 1.157823702216272f, -0.11060664309660294f,
                             -0.016493938717834573f, -0.016493938717834257f, 1.2519364065950405f};
float agxChannel(float x) {
    const float minEv = -12.47393f, maxEv = 4.026069f;
    x = std::fmax(x, 1e-10f);
    x = std::fmin(std::fmax(std::log2(x), minEv), maxEv);
    x = (x - minEv) / (maxEv - minEv);
    x = clamp01(x);
    const float x2 = x * x, x4 = x2 * x2;
    return ((((((15.5f * x4 * x2 - 40.14f * x4 * x) + 31.96f * x4) - 6.868f * x2 * x) + 0.4298f * x2) + 0.1191f * x) - 0.00232f);
}
V agx(V c, float power, float saturation) {
    c = mul3(kSrgbToRec2020, c);
    c = mul3(kAgxInset, c);
    c = V{agxChannel(c.r), agxChannel(c.g), agxChannel(c.b)};
    // CDL with slope 1, offset 0
    c = V{std::pow(c.r * 1.0f + 0.0f, power), std::pow(c.g * 1.0f + 0.0f, power), std::pow(c.b * 1.0f + 0.0f, power)};
    const float luma = (c.r * 0.2126f + c.g * 0.7152f) + c.b * 0.0722f;
    c = V{luma + saturation * (c.r - luma), luma + saturation * (c.g - luma), luma + saturation * (c.b - luma)};
    c = mul3(kAgxOutset, c);
    c = V{std::pow(std::fmax(0.0f, c.r), 2.2f), std::pow(std::fmax(0.0f, c.g), 2.2f), std::pow(std::fmax(0.0f, c.b), 2.2f)};
    c = mul3(kRec2020ToSrgb, c);
    return V{clamp01(c.r), clamp01(c.g), clamp01(c.b)};
}

V tonemap(V c, int op) {
    switch (op) {
        case 1: return reinhard(c);
        case 2: return uncharted2(c);
        case 3: return aces(c);
        case 4: return khronos(c);
        case 5: return agx(c, 1.0f, 1.0f);
        case 6: return agx(c, 1.35f, 1.4f);
        default: return c;
    }
}

// color.h:84-95 + film.cpp:161-169 (NaN -> 0)
uint8_t exportByte(float x) {
    const float s = x <= 0.0031308f ? 12.92f * x : 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f;
    const float v = std::fmin(std::fmax(s * 255.0f + 0.5f, 0.0f), 255.0f);
    return (uint8_t)v;
}
// gammaCorrect.frag + the unsigned normalised store of the 8-bit target
uint8_t displayByte(float x) {
    const float s = x <= 0.0031308f ? 12.92f * x : 1.055f * std::pow(x, 0.41666f) - 0.055f;
    return (uint8_t)std::nearbyint(clamp01(s) * 255.0f);
}

}  // namespace

extern "C" {

// Post-processing of a linear RGB image (w x h x 3): optional bloom pyramid, exposure,
// tonemap operator; outputs the tonemapped float image (hdr, nullable) and 8-bit RGB
// (rgb8, nullable; output 0: Film::savePNG conversion, 1: the display gamma pass).
// params: tonemapper, bloom, mips, output (ints); exposure, threshold, radius, intensity.
void orc_post(const float* rgb, int w, int h, int tonemapper, float exposure, int bloom, float threshold,
              float radius, float intensity, int mips, int output, float* hdr, uint8_t* rgb8) {
    Tex in;
    in.w = w; in.h = h;
    in.px.assign(rgb, rgb + 3 * (size_t)w * h);
    // postProcessor.cpp:116-143: pyramid from half size, halving while both sides >= 2, at most 6
    std::vector<Tex> pyr;
    for (int mw = w / 2, mh = h / 2, i = 0; i < 6; ++i) {
        Tex t;
        t.w = mw; t.h = mh;
        t.px.assign(3 * (size_t)std::max(mw, 0) * std::max(mh, 0), 0.0f);
        pyr.push_back(t);
        mw /= 2; mh /= 2;
        if (mw < 2 || mh < 2) break;
    }
    const bool doBloom = bloom && !pyr.empty() && pyr[0].w > 0 && pyr[0].h > 0;
    if (doBloom) {
        const int n = std::min(mips, (int)pyr.size());
        prefilter(in, pyr[0], threshold);
        for (int i = 1; i < n; ++i) downsample(pyr[i - 1], pyr[i]);
        for (int i = n - 1; i > 0; --i) upsampleAdd(pyr[i], pyr[i - 1], radius);
    }
    const float scale = std::exp2(exposure);
    for (int j = 0; j < h; ++j)
        for (int i = 0; i < w; ++i) {
            const float* p = in.at(i, j);
            V c{p[0], p[1], p[2]};
            if (doBloom) {
                float b[3];
                sample(pyr[0], ((float)i + 0.5f) / (float)w, ((float)j + 0.5f) / (float)h, b);
                c = V{c.r + b[0] * intensity, c.g + b[1] * intensity, c.b + b[2] * intensity};
            }
            c = V{c.r * scale, c.g * scale, c.b * scale};
            c = tonemap(c, tonemapper);
            const size_t o = 3 * ((size_t)j * w + i);
            if (hdr) { hdr[o] = c.r; hdr[o + 1] = c.g; hdr[o + 2] = c.b; }
            if (rgb8) {
                const float v[3] = {c.r, c.g, c.b};
                for (int k = 0; k < 3; ++k) rgb8[o + k] = output == 1 ? displayByte(v[k]) : exportByte(v[k]);
            }
        }
}

float orc_round_half(float x) { return roundHalf(x); }

}  // extern "C"
