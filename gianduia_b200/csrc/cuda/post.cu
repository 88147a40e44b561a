// Post-processing of a rendered image on the device (gnd_gpu_post): the reference's GL
// post pipeline (postProcessor.cpp:148-235 running bloom_prefilter.frag,
// bloom_downsample.frag, bloom_upsample.frag, tonemap.frag and gammaCorrect.frag) and the
// 8-bit conversion of Film::savePNG (film.cpp:154-171), as CUDA kernels on plain device
// buffers (no graphics stack).
//
// Texture sampling is GL_LINEAR made explicit: texel centres at (i + 0.5) / size, exact
// fp32 bilinear weights, clamp to edge. The bloom pyramid (half size, halving while both
// sides stay >= 2, at most 6 levels) is stored in binary16 like the reference's RGB16F
// targets; the upsample pass adds into the finer level in fp32 and stores binary16, as
// the additive blend does. Every kernel is one thread per output texel; the images are
// small next to HBM bandwidth (a 1024^2 frame is 12 MB), so the pass is launch-bound.
#include <cuda_fp16.h>

#include <algorithm>
#include <vector>

#include "runtime.h"

namespace gnd {

namespace {

constexpr int kPostBlock = 256;
constexpr int kMaxBloomMips = 6;

struct Img {
    int w, h;
};

template <typename T>
__device__ __forceinline__ float ld(const T* p);
template <>
__device__ __forceinline__ float ld<float>(const float* p) { return __ldg(p); }
template <>
__device__ __forceinline__ float ld<__half>(const __half* p) { return __half2float(*p); }

// GL_LINEAR sample of an rgb texture at (u, v), clamp to edge
template <typename T>
__device__ __forceinline__ void sample(const T* tex, Img t, float u, float v, float out[3]) {
    const float x = u * (float)t.w - 0.5f, y = v * (float)t.h - 0.5f;
    const float x0f = floorf(x), y0f = floorf(y);
    const float fx = x - x0f, fy = y - y0f;
    const int x0 = min(max((int)x0f, 0), t.w - 1), x1 = min(max((int)x0f + 1, 0), t.w - 1);
    const int y0 = min(max((int)y0f, 0), t.h - 1), y1 = min(max((int)y0f + 1, 0), t.h - 1);
    const T* a = tex + 3 * ((size_t)y0 * t.w + x0);
    const T* b = tex + 3 * ((size_t)y0 * t.w + x1);
    const T* c = tex + 3 * ((size_t)y1 * t.w + x0);
    const T* d = tex + 3 * ((size_t)y1 * t.w + x1);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float c0 = ld(a + k) * (1.0f - fx) + ld(b + k) * fx;
        const float c1 = ld(c + k) * (1.0f - fx) + ld(d + k) * fx;
        out[k] = c0 * (1.0f - fy) + c1 * fy;
    }
}

// bloom_prefilter.frag: the input sampled at the half-size texel centres, kept where its
// brightest channel exceeds the threshold
__global__ void kBloomPrefilter(const float* __restrict__ in, Img ii, __half* dst, Img di, float threshold) {
    const int n = di.w * di.h;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = q % di.w, j = q / di.w;
    float c[3];
    sample(in, ii, ((float)i + 0.5f) / (float)di.w, ((float)j + 0.5f) / (float)di.h, c);
    const float bright = fmaxf(c[0], fmaxf(c[1], c[2]));
    __half* o = dst + 3 * (size_t)q;
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = __float2half_rn(bright > threshold ? c[k] : 0.0f);
}

// bloom_downsample.frag: 13 taps at one and two source texels
__global__ void kBloomDown(const __half* __restrict__ src, Img si, __half* dst, Img di) {
    const int n = di.w * di.h;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = q % di.w, j = q / di.w;
    const float x = 1.0f / (float)si.w, y = 1.0f / (float)si.h;
    const float u = ((float)i + 0.5f) / (float)di.w, v = ((float)j + 0.5f) / (float)di.h;
    float a[3], b[3], c[3], d[3], e[3], f[3], g[3], h[3], ii[3], jj[3], kk[3], ll[3], mm[3];
    sample(src, si, u - 2 * x, v + 2 * y, a);
    sample(src, si, u, v + 2 * y, b);
    sample(src, si, u + 2 * x, v + 2 * y, c);
    sample(src, si, u - 2 * x, v, d);
    sample(src, si, u, v, e);
    sample(src, si, u + 2 * x, v, f);
    sample(src, si, u - 2 * x, v - 2 * y, g);
    sample(src, si, u, v - 2 * y, h);
    sample(src, si, u + 2 * x, v - 2 * y, ii);
    sample(src, si, u - x, v + y, jj);
    sample(src, si, u + x, v + y, kk);
    sample(src, si, u - x, v - y, ll);
    sample(src, si, u + x, v - y, mm);
    __half* o = dst + 3 * (size_t)q;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float s = e[k] * 0.125f;
        s += (((a[k] + c[k]) + g[k]) + ii[k]) * 0.03125f;
        s += (((b[k] + d[k]) + f[k]) + h[k]) * 0.0625f;
        s += (((jj[k] + kk[k]) + ll[k]) + mm[k]) * 0.125f;
        o[k] = __float2half_rn(s);
    }
}

// bloom_upsample.frag (3x3 tent of `radius` source texels) added into the finer level
__global__ void kBloomUpAdd(const __half* __restrict__ src, Img si, __half* dst, Img di, float radius) {
    const int n = di.w * di.h;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = q % di.w, j = q / di.w;
    const float x = radius * (1.0f / (float)si.w), y = radius * (1.0f / (float)si.h);
    const float u = ((float)i + 0.5f) / (float)di.w, v = ((float)j + 0.5f) / (float)di.h;
    float a[3], b[3], c[3], d[3], e[3], f[3], g[3], h[3], ii[3];
    sample(src, si, u - x, v + y, a);
    sample(src, si, u, v + y, b);
    sample(src, si, u + x, v + y, c);
    sample(src, si, u - x, v, d);
    sample(src, si, u, v, e);
    sample(src, si, u + x, v, f);
    sample(src, si, u - x, v - y, g);
    sample(src, si, u, v - y, h);
    sample(src, si, u + x, v - y, ii);
    __half* o = dst + 3 * (size_t)q;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float s = e[k] * 4.0f;
        s += (((b[k] + d[k]) + f[k]) + h[k]) * 2.0f;
        s += (((a[k] + c[k]) + g[k]) + ii[k]) * 1.0f;
        s *= 1.0f / 16.0f;
        o[k] = __float2half_rn(__half2float(o[k]) + s);
    }
}

// ---------------------------------------------------------------- tonemap.frag operators
struct C3 {
    float r, g, b;
};
// GLSL mat3(m0..m8) is column-major; products summed left to right
__device__ __forceinline__ C3 mul3(const float* m, C3 c) {
    return C3{(m[0] * c.r + m[3] * c.g) + m[6] * c.b, (m[1] * c.r + m[4] * c.g) + m[7] * c.b,
              (m[2] * c.r + m[5] * c.g) + m[8] * c.b};
}
__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

__constant__ float kAcesIn[9] = {0.59719f, 0.07600f, 0.02840f, 0.35458f, 0.90834f, 0.13383f, 0.04823f, 0.01566f, 0.83777f};
__constant__ float kAcesOut[9] = {1.60475f, -0.10208f, -0.00327f, -0.53108f, 1.10813f, -0.07276f, -0.07367f, -0.00605f, 1.07602f};
__constant__ float kRec2020ToSrgb[9] = {1.6605f, -0.1246f, -0.0182f, -0.5876f, 1.1329f, -0.1006f, -0.0728f, -0.0083f, 1.1187f};
__constant__ float kSrgbToRec2020[9] = {0.6274f, 0.0691f, 0.0164f, 0.3293f, 0.9195f, 0.0880f, 0.0433f, 0.0113f, 0.8956f};
__constant__ float kAgxInset[9] = {0.856627153315983f, 0.137318972929847f, 0.11189821299995f,
                                   0.0951212405381588f, 0.761241990602591f, 0.0767994186031903f,
                                   0.0482516061458583f, 0.101439036467562f, 0.811302368396859f};
__constant__ float kAgxOutset[9] = {1.1271005818144368f, -0.1413297634984383f, -0.14132976349843826f,
                                    -0.11060664309660323f, 1.157823702216272f, -0.11060664309660294f,
                                    -0.016493938717834573f, -0.016493938717834257f, 1.2519364065950405f};

__device__ __forceinline__ C3 reinhard(C3 c) {
    const float luma = (c.r * 0.2126f + c.g * 0.7152f) + c.b * 0.0722f;
    const float s = (luma / (1.0f + luma)) / fmaxf(luma, 0.00001f);
    return C3{c.r * s, c.g * s, c.b * s};
}
__device__ __forceinline__ float u2curve(float x) {
    const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, F = 0.30f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
}
__device__ __forceinline__ C3 uncharted2(C3 c) {
    const float ws = 1.0f / u2curve(11.2f);
    return C3{u2curve(2.0f * c.r) * ws, u2curve(2.0f * c.g) * ws, u2curve(2.0f * c.b) * ws};
}
__device__ __forceinline__ float rrtOdt(float v) {
    const float a = v * (v + 0.0245786f) - 0.000090537f;
    const float b = v * (0.983729f * v + 0.432951f) + 0.238081f;
    return a / b;
}
__device__ __forceinline__ C3 aces(C3 c) {
    c = mul3(kAcesIn, c);
    c = C3{rrtOdt(c.r), rrtOdt(c.g), rrtOdt(c.b)};
    c = mul3(kAcesOut, c);
    return C3{clamp01(c.r), clamp01(c.g), clamp01(c.b)};
}
__device__ __forceinline__ C3 khronosNeutral(C3 c) {
    const float startCompression = 0.8f - 0.04f, desaturation = 0.15f;
    const float x = fminf(c.r, fminf(c.g, c.b));
    const float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    c = C3{c.r - offset, c.g - offset, c.b - offset};
    const float peak = fmaxf(c.r, fmaxf(c.g, c.b));
    if (peak < startCompression) return c;
    const float d = 1.0f - startCompression;
    const float newPeak = 1.0f - d * d / (peak + d - startCompression);
    const float s = newPeak / peak;
    c = C3{c.r * s, c.g * s, c.b * s};
    const float g = 1.0f - 1.0f / (desaturation * (peak - newPeak) + 1.0f);
    return C3{c.r * (1.0f - g) + newPeak * g, c.g * (1.0f - g) + newPeak * g, c.b * (1.0f - g) + newPeak * g};
}
__device__ __forceinline__ float agxChannel(float x) {
    const float minEv = -12.47393f, maxEv = 4.026069f;
    x = fmaxf(x, 1e-10f);
    x = fminf(fmaxf(log2f(x), minEv), maxEv);
    x = clamp01((x - minEv) / (maxEv - minEv));
    const float x2 = x * x, x4 = x2 * x2;
    return ((((((15.5f * x4 * x2 - 40.14f * x4 * x) + 31.96f * x4) - 6.868f * x2 * x) + 0.4298f * x2) + 0.1191f * x) - 0.00232f);
}
__device__ __forceinline__ C3 agx(C3 c, float power, float saturation) {
    c = mul3(kSrgbToRec2020, c);
    c = mul3(kAgxInset, c);
    c = C3{agxChannel(c.r), agxChannel(c.g), agxChannel(c.b)};
    c = C3{powf(c.r * 1.0f + 0.0f, power), powf(c.g * 1.0f + 0.0f, power), powf(c.b * 1.0f + 0.0f, power)};
    const float luma = (c.r * 0.2126f + c.g * 0.7152f) + c.b * 0.0722f;
    c = C3{luma + saturation * (c.r - luma), luma + saturation * (c.g - luma), luma + saturation * (c.b - luma)};
    c = mul3(kAgxOutset, c);
    c = C3{powf(fmaxf(0.0f, c.r), 2.2f), powf(fmaxf(0.0f, c.g), 2.2f), powf(fmaxf(0.0f, c.b), 2.2f)};
    c = mul3(kRec2020ToSrgb, c);
    return C3{clamp01(c.r), clamp01(c.g), clamp01(c.b)};
}

// color.h:84-95 then film.cpp:164-169 (x 255 + 0.5, clamp, truncate; NaN -> 0)
__device__ __forceinline__ uint8_t exportByte(float x) {
    const float s = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
    return (uint8_t)fminf(fmaxf(s * 255.0f + 0.5f, 0.0f), 255.0f);
}
// gammaCorrect.frag + the unsigned normalised 8-bit store (round to nearest)
__device__ __forceinline__ uint8_t displayByte(float x) {
    const float s = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 0.41666f) - 0.055f;
    return (uint8_t)rintf(clamp01(s) * 255.0f);
}

// tonemap.frag main(): + bloom * intensity, * exp2(exposure), operator; then the 8-bit
// conversion of the export (output 0) or display (output 1) path
__global__ void kTonemap(const float* __restrict__ in, Img ii, const __half* __restrict__ bloom, Img bi, float intensity,
                         float scale, int op, int output, float* hdr, uint8_t* rgb8) {
    const int n = ii.w * ii.h;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = q % ii.w, j = q / ii.w;
    const float* p = in + 3 * (size_t)q;
    C3 c{p[0], p[1], p[2]};
    if (bloom) {
        float b[3];
        sample(bloom, bi, ((float)i + 0.5f) / (float)ii.w, ((float)j + 0.5f) / (float)ii.h, b);
        c = C3{c.r + b[0] * intensity, c.g + b[1] * intensity, c.b + b[2] * intensity};
    }
    c = C3{c.r * scale, c.g * scale, c.b * scale};
    switch (op) {
        case 1: c = reinhard(c); break;
        case 2: c = uncharted2(c); break;
        case 3: c = aces(c); break;
        case 4: c = khronosNeutral(c); break;
        case 5: c = agx(c, 1.0f, 1.0f); break;
        case 6: c = agx(c, 1.35f, 1.4f); break;
        default: break;
    }
    const size_t o = 3 * (size_t)q;
    if (hdr) { hdr[o] = c.r; hdr[o + 1] = c.g; hdr[o + 2] = c.b; }
    if (rgb8) {
        rgb8[o] = output == 1 ? displayByte(c.r) : exportByte(c.r);
        rgb8[o + 1] = output == 1 ? displayByte(c.g) : exportByte(c.g);
        rgb8[o + 2] = output == 1 ? displayByte(c.b) : exportByte(c.b);
    }
}

inline unsigned blocks(int n) { return (unsigned)((n + kPostBlock - 1) / kPostBlock); }

void checkParams(int w, int h, const gnd_post_params* p) {
    if (w <= 0 || h <= 0 || (int64_t)w * h > (int64_t)1 << 28) throw Error(GND_ERR_INVALID, "post: image size out of range");
    if (!p) throw Error(GND_ERR_INVALID, "post: null parameters");
    if (p->tonemapper < 0 || p->tonemapper > 6) throw Error(GND_ERR_INVALID, "post: unknown tonemapper");
    if (p->output != 0 && p->output != 1) throw Error(GND_ERR_INVALID, "post: output must be 0 (export) or 1 (display)");
    if (p->bloom && (p->bloom_mips < 1 || p->bloom_mips > kMaxBloomMips)) throw Error(GND_ERR_INVALID, "post: bloom_mips out of range (1..6)");
}

// Runs the passes on `st` over device buffers; scratch from the pool.
void postDevice(const float* rgb, int w, int h, const gnd_post_params* p, float* hdr, uint8_t* rgb8, cudaStream_t st) {
    // postProcessor.cpp:116-143: the pyramid
    std::vector<Img> mips;
    for (int mw = w / 2, mh = h / 2, i = 0; i < kMaxBloomMips; ++i) {
        mips.push_back(Img{mw, mh});
        mw /= 2;
        mh /= 2;
        if (mw < 2 || mh < 2) break;
    }
    const bool doBloom = p->bloom && !mips.empty() && mips[0].w > 0 && mips[0].h > 0;
    std::vector<PoolBuf> levels;
    if (doBloom) {
        const int n = std::min<int>(p->bloom_mips, (int)mips.size());
        for (int i = 0; i < n; ++i) {
            levels.emplace_back((size_t)mips[i].w * mips[i].h * 3 * sizeof(__half), st);
            if (i > 0) GND_CUDA(cudaMemsetAsync(levels.back().ptr, 0, levels.back().bytes, st));
        }
        kBloomPrefilter<<<blocks(mips[0].w * mips[0].h), kPostBlock, 0, st>>>(rgb, Img{w, h}, levels[0].as<__half>(), mips[0],
                                                                               p->bloom_threshold);
        for (int i = 1; i < n; ++i)
            kBloomDown<<<blocks(mips[i].w * mips[i].h), kPostBlock, 0, st>>>(levels[i - 1].as<__half>(), mips[i - 1],
                                                                              levels[i].as<__half>(), mips[i]);
        for (int i = n - 1; i > 0; --i)
            kBloomUpAdd<<<blocks(mips[i - 1].w * mips[i - 1].h), kPostBlock, 0, st>>>(levels[i].as<__half>(), mips[i],
                                                                                      levels[i - 1].as<__half>(), mips[i - 1],
                                                                                      p->bloom_radius);
        GND_CUDA(cudaGetLastError());
    }
    kTonemap<<<blocks(w * h), kPostBlock, 0, st>>>(rgb, Img{w, h}, doBloom ? levels[0].as<__half>() : nullptr,
                                                   doBloom ? mips[0] : Img{1, 1}, p->bloom_intensity, exp2f(p->exposure),
                                                   p->tonemapper, p->output, hdr, rgb8);
    GND_CUDA(cudaGetLastError());
}

}  // namespace

}  // namespace gnd

using namespace gnd;

extern "C" {

gnd_status gnd_gpu_post(gnd_gpu_ctx* ctxh, const float* rgb, int32_t width, int32_t height, const gnd_post_params* params,
                        float* hdr, uint8_t* rgb8) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        checkParams(width, height, params);
        if (!rgb) throw Error(GND_ERR_INVALID, "post: null input");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        const size_t n = (size_t)width * height;
        PoolBuf din(n * 12, c->stream), dhdr(hdr ? n * 12 : 0, c->stream), d8(rgb8 ? n * 3 : 0, c->stream);
        GND_CUDA(cudaMemcpyAsync(din.ptr, rgb, n * 12, cudaMemcpyHostToDevice, c->stream));
        postDevice(din.as<float>(), width, height, params, hdr ? dhdr.as<float>() : nullptr, rgb8 ? d8.as<uint8_t>() : nullptr,
                   c->stream);
        if (hdr) GND_CUDA(cudaMemcpyAsync(hdr, dhdr.ptr, n * 12, cudaMemcpyDeviceToHost, c->stream));
        if (rgb8) GND_CUDA(cudaMemcpyAsync(rgb8, d8.ptr, n * 3, cudaMemcpyDeviceToHost, c->stream));
        GND_CUDA(cudaStreamSynchronize(c->stream));
    });
}

gnd_status gnd_gpu_post_dev(gnd_gpu_ctx* ctxh, const float* d_rgb, int32_t width, int32_t height,
                            const gnd_post_params* params, float* d_hdr, uint8_t* d_rgb8, void* stream) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        checkParams(width, height, params);
        if (!d_rgb) throw Error(GND_ERR_INVALID, "post: null input");
        c->bind();
        postDevice(d_rgb, width, height, params, d_hdr, d_rgb8, reinterpret_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
