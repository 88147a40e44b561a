// Texture trees on the device: Perlin turbulence (math/perlin.h), Worley F1 / F2
// (math/worley.h), the perlin / marble / wood / cellular color textures, image lookups
// (imageTexture.cpp: closest or bilinear, repeat or clamp) and the domain warp
// (domainWarp.h), evaluated at a surface point (p, n, dpdu, uv). Float arithmetic in the
// reference's order; sinf is the device's, so marble and wood can differ from the host in
// the last bits.
#pragma once
#include "gnd/layout.h"
#include "gnd/vmath.h"

namespace gnd {

// Ken Perlin's permutation of 0..255 from "Improving Noise" (2002); indices up to 511 wrap.
__device__ const uint8_t kPerlinPerm[256] = {
    151, 160, 137, 91, 90, 15, 131, 13, 201, 95, 96, 53, 194, 233, 7, 225, 140, 36, 103, 30, 69, 142, 8,
    99, 37, 240, 21, 10, 23, 190, 6, 148, 247, 120, 234, 75, 0, 26, 197, 62, 94, 252, 219, 203, 117, 35,
    11, 32, 57, 177, 33, 88, 237, 149, 56, 87, 174, 20, 125, 136, 171, 168, 68, 175, 74, 165, 71, 134,
    139, 48, 27, 166, 77, 146, 158, 231, 83, 111, 229, 122, 60, 211, 133, 230, 220, 105, 92, 41, 55, 46,
    245, 40, 244, 102, 143, 54, 65, 25, 63, 161, 1, 216, 80, 73, 209, 76, 132, 187, 208, 89, 18, 169,
    200, 196, 135, 130, 116, 188, 159, 86, 164, 100, 109, 198, 173, 186, 3, 64, 52, 217, 226, 250, 124,
    123, 5, 202, 38, 147, 118, 126, 255, 82, 85, 212, 207, 206, 59, 227, 47, 16, 58, 17, 182, 189, 28,
    42, 223, 183, 170, 213, 119, 248, 152, 2, 44, 154, 163, 70, 221, 153, 101, 155, 167, 43, 172, 9,
    129, 22, 39, 253, 19, 98, 108, 110, 79, 113, 224, 232, 178, 185, 112, 104, 218, 246, 97, 228, 251,
    34, 242, 193, 238, 210, 144, 12, 191, 179, 162, 241, 81, 51, 145, 235, 249, 14, 239, 107, 49, 192,
    214, 31, 181, 199, 106, 157, 184, 84, 204, 176, 115, 121, 50, 45, 127, 4, 150, 254, 138, 236, 205,
    93, 222, 114, 67, 29, 24, 72, 243, 141, 128, 195, 78, 66, 215, 61, 156, 180};

__device__ __forceinline__ int perm(int i) { return (int)__ldg(&kPerlinPerm[i & 255]); }
__device__ __forceinline__ float nFade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
__device__ __forceinline__ float nLerp(float t, float a, float b) { return (1.0f - t) * a + t * b; }   // constants.h:41-44
// gradient of hash h dotted with (x, y, z): one of the 12 cube-edge directions
__device__ __forceinline__ float nGrad(int h, float x, float y, float z) {
    h &= 15;
    const float u = h < 8 ? x : y;
    const float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}

// Perlin::noise (perlin.h:12-50), in [-1, 1]
__device__ __forceinline__ float perlinNoise(V3 p) {
    const float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
    const int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
    const float x = p.x - fx, y = p.y - fy, z = p.z - fz;
    const float u = nFade(x), v = nFade(y), w = nFade(z);
    const int A = perm(X) + Y, AA = perm(A) + Z, AB = perm(A + 1) + Z;
    const int B = perm(X + 1) + Y, BA = perm(B) + Z, BB = perm(B + 1) + Z;
    const float x00 = nLerp(u, nGrad(perm(AA), x, y, z), nGrad(perm(BA), x - 1.0f, y, z));
    const float x10 = nLerp(u, nGrad(perm(AB), x, y - 1.0f, z), nGrad(perm(BB), x - 1.0f, y - 1.0f, z));
    const float x01 = nLerp(u, nGrad(perm(AA + 1), x, y, z - 1.0f), nGrad(perm(BA + 1), x - 1.0f, y, z - 1.0f));
    const float x11 = nLerp(u, nGrad(perm(AB + 1), x, y - 1.0f, z - 1.0f), nGrad(perm(BB + 1), x - 1.0f, y - 1.0f, z - 1.0f));
    return nLerp(w, nLerp(v, x00, x10), nLerp(v, x01, x11));
}

// Perlin::turbulence (perlin.h:71-85), clamped to [0, 1]
__device__ __forceinline__ float turbulence(V3 p, int octaves) {
    float acc = 0.0f, weight = 1.0f;
    for (int i = 0; i < octaves; ++i) {
        acc += weight * fabsf(perlinNoise(p));
        weight *= 0.5f;
        p = p * 2.0f;
    }
    return clampf(acc, 0.0f, 1.0f);
}

// Worley::hash3's per-component hash (worley.h:67-72)
__device__ __forceinline__ float worleyHash(uint32_t n) {
    n = (n << 13U) ^ n;
    n = n * (n * n * 15731U + 789221U) + 1376312589U;
    return (float)(n & 0x7fffffffU) / (float)0x7fffffff;
}
// Worley::noise (worley.h:22-64): distances to the nearest and second nearest feature
// points of the 27 cells around p, one feature point per cell
__device__ __forceinline__ void worleyNoise(V3 p, int metric, float& f1, float& f2) {
    const int x0 = (int)floorf(p.x), y0 = (int)floorf(p.y), z0 = (int)floorf(p.z);
    f1 = 1e8f;
    f2 = 1e8f;
    for (int k = -1; k <= 1; ++k)
        for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i) {
                const int cx = x0 + i, cy = y0 + j, cz = z0 + k;
                const uint32_t n = (uint32_t)cx * 73856093U ^ (uint32_t)cy * 19349663U ^ (uint32_t)cz * 83492791U;
                const V3 fp = v3((float)cx + worleyHash(n), (float)cy + worleyHash(n + 1), (float)cz + worleyHash(n + 2));
                const V3 d = p - fp;
                float dist;
                if (metric == 0) dist = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
                else if (metric == 1) dist = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
                else dist = fmaxf_(fmaxf_(fabsf(d.x), fabsf(d.y)), fabsf(d.z));
                if (dist < f1) { f2 = f1; f1 = dist; }
                else if (dist < f2) f2 = dist;
            }
}

// std::lerp(a, b, t) as P0811R3 specifies it: exact at t = 0 and t = 1, monotonic,
// a + t (b - a) unless a and b straddle zero
__device__ __forceinline__ float stdLerp(float a, float b, float t) {
    if ((a <= 0.0f && b >= 0.0f) || (a >= 0.0f && b <= 0.0f)) return t * b + (1.0f - t) * a;
    if (t == 1.0f) return b;
    const float x = a + t * (b - a);
    return (t > 1.0f) == (b > a) ? (b < x ? x : b) : (b > x ? x : b);
}
// value1 * (1 - t) + value2 * t for color textures; the float perlin / marble / wood
// textures blend with std::lerp (perlin.h:33, marble.h:42, wood.h:42)
__device__ __forceinline__ V3 texMix(const TexNode& t, float x) {
    if (t.flags & kTnFloatLerp) return v3s(stdLerp(t.v1[0], t.v2[0], x));
    return v3(t.v1[0], t.v1[1], t.v1[2]) * (1.0f - x) + v3(t.v2[0], t.v2[1], t.v2[2]) * x;
}

// ImageTexture::extractValue (imageTexture.cpp:84-107) on rgba texels
__device__ __forceinline__ V3 imageTexel(const SceneView& s, const TexNode& t, int x, int y) {
    const int w = t.w, h = t.h;
    if (t.flags & kTnClamp) {
        x = x < 0 ? 0 : (x > w - 1 ? w - 1 : x);
        y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
    } else {
        x = ((x % w) + w) % w;
        y = ((y % h) + h) % h;
    }
    const float4 c = __ldg(reinterpret_cast<const float4*>(s.texels) + t.a + (int64_t)y * w + x);
    if (t.flags & kTnNormal)   // imageTexture.cpp:101-104
        return t.b >= 3 ? v3(c.x * 2.0f - 1.0f, c.y * 2.0f - 1.0f, c.z * 2.0f - 1.0f) : v3(0.0f, 0.0f, 1.0f);
    return v3(c.x, c.y, c.z);
}
// ImageTexture::sampleClosest / sampleLinear (imageTexture.cpp:109-143)
__device__ __forceinline__ V3 imageLookup(const SceneView& s, const TexNode& t, V2 uv) {
    V2 l;
    if (t.flags & kTnClamp) l = V2{clampf(uv.x, 0.0f, 1.0f), clampf(uv.y, 0.0f, 1.0f)};
    else l = V2{uv.x - floorf(uv.x), uv.y - floorf(uv.y)};
    if (!(t.flags & kTnLinear)) return imageTexel(s, t, (int)floorf(l.x * (float)t.w), (int)floorf(l.y * (float)t.h));
    const float xc = l.x * (float)t.w - 0.5f, yc = l.y * (float)t.h - 0.5f;
    const int x0 = (int)floorf(xc), y0 = (int)floorf(yc);
    const float tx = xc - (float)x0, ty = yc - (float)y0;
    const V3 top = imageTexel(s, t, x0, y0) * (1.0f - tx) + imageTexel(s, t, x0 + 1, y0) * tx;
    const V3 bottom = imageTexel(s, t, x0, y0 + 1) * (1.0f - tx) + imageTexel(s, t, x0 + 1, y0 + 1) * tx;
    return top * (1.0f - ty) + bottom * ty;
}

// Every node kind but the warp, at point p with coordinates uv
__device__ __forceinline__ V3 texLeaf(const SceneView& s, const TexNode& t, V3 p, V2 uv) {
    switch (t.kind) {
        case kTnConstant:
            return v3(t.v1[0], t.v1[1], t.v1[2]);
        case kTnChecker: {   // checkerboard.h:36-48
            float x = uv.x / t.cscale[0], y = uv.y / t.cscale[1];
            x -= t.delta[0];
            y -= t.delta[1];
            const int a = (int)floorf(x), b = (int)floorf(y);
            return ((a + b) % 2 == 0) ? v3(t.v1[0], t.v1[1], t.v1[2]) : v3(t.v2[0], t.v2[1], t.v2[2]);
        }
        case kTnPerlin:   // perlin.h (texture):30-37
            return texMix(t, turbulence(divs(p, t.scale), t.octaves));
        case kTnMarble: {   // marble.h:36-46
            const float turb = turbulence(divs(p, t.scale), t.octaves);
            const float val = dot(p, v3(t.axis[0], t.axis[1], t.axis[2])) + turb * t.turbScale;
            return texMix(t, 0.5f * (1.0f + sinf(val * t.veinFreq)));
        }
        case kTnWood: {   // wood.h:36-46
            const float turb = turbulence(divs(p, t.scale), t.octaves);
            float radius = length(cross(p, v3(t.axis[0], t.axis[1], t.axis[2])));
            radius += turb * t.turbScale;
            return texMix(t, fabsf(sinf(radius * t.veinFreq)));
        }
        case kTnCellular: {   // cellular.h:48-58
            float f1, f2;
            worleyNoise(divs(p, t.scale), (t.flags >> kTnMetricShift) & 3, f1, f2);
            return texMix(t, clampf((t.flags & kTnCracks) ? f2 - f1 : f1, 0.0f, 1.0f));
        }
        case kTnImage:
            return imageLookup(s, t, uv);
        default:
            return v3s(0.0f);
    }
}

// A chain of warps ending in a leaf (domainWarp.h:38-58): each warp evaluates its warp
// input at the current point, moves p by (2 w - 1) strength and uv by that offset's
// projections on dpdu and n x dpdu (n and dpdu stay those of the surface), then continues
// with its base. LEVEL bounds the nesting of warps inside warp inputs.
template <int LEVEL>
__device__ __forceinline__ V3 texChain(const SceneView& s, uint32_t node, V3 p, V3 n, V3 dpdu, V2 uv) {
    for (int hop = 0; hop < s.numTexNodes; ++hop) {
        const TexNode t = s.texNodes[node];
        if (t.kind != kTnWarp) return texLeaf(s, t, p, uv);
        V3 w;
        if constexpr (LEVEL > 1) w = texChain<LEVEL - 1>(s, (uint32_t)t.b, p, n, dpdu, uv);
        else w = texLeaf(s, s.texNodes[t.b], p, uv);
        const V3 d = v3((w.x * 2.0f - 1.0f) * t.strength, (w.y * 2.0f - 1.0f) * t.strength, (w.z * 2.0f - 1.0f) * t.strength);
        const V3 dpdv = cross(n, dpdu);
        const float lu = lengthSq(dpdu), lv = lengthSq(dpdv);
        const float du = lu > 0.0f ? dot(d, dpdu) / lu : 0.0f;
        const float dv = lv > 0.0f ? dot(d, dpdv) / lv : 0.0f;
        p = p + d;
        uv.x += du;
        uv.y += dv;
        node = (uint32_t)t.a;
    }
    return v3s(0.0f);   // unreachable for the trees the host builds (no cycles)
}

// A texture tree, out of line so that the kernels without trees keep their registers.
__device__ __noinline__ V3 evalTexTree(const SceneView& s, uint32_t node, V3 p, V3 n, V3 dpdu, V2 uv) {
    return texChain<kTexWarpNesting>(s, node, p, n, dpdu, uv);
}

}  // namespace gnd
