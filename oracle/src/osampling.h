// Oracle (test infrastructure only): random numbers and sample warps of the
// reference's radiance path, restated on the CPU.
#pragma once
#include "omath.h"

namespace orc {

// pcg32.h:5-32 (PCG32, XSH-RR output, seeded with stream 1)
struct PCG32 {
    uint64_t state = 0, inc = 1;
    PCG32(uint64_t initstate = 0, uint64_t initseq = 1) { seed(initstate, initseq); }
    void seed(uint64_t initstate, uint64_t initseq = 1) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        nextUInt();
        state += initstate;
        nextUInt();
    }
    uint32_t nextUInt() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
    }
    // pcg32.h:107-109: ldexp((float)u, -32); can return exactly 1.0f
    float nextFloat() { return std::ldexp((float)nextUInt(), -32); }
};

// independent.cpp:39-44
inline uint64_t splitMix64(uint64_t index) {
    uint64_t z = index + 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// independent.cpp:22-32. The reference constructs Point2f(next, next); C++ leaves the
// order of those two calls unspecified. This restatement fixes x first, then y, and
// (integrators) the 2D sample before the 1D sample in BSDF::sample calls.
struct Sampler {
    PCG32 rng;
    uint64_t draws = 0;
    void seed(uint64_t idx) { rng.seed(splitMix64(idx)); }
    float next1D() { ++draws; return rng.nextFloat(); }
    Vec2 next2D() { float a = next1D(); float b = next1D(); return Vec2(a, b); }
};

namespace warp {
// warp.cpp:7-26 (concentric disk; M_PI terms evaluated in double as in the reference)
inline Vec2 squareToUniformDisk(const Vec2& s) {
    Vec2 p(2.0f * s.x - 1.0f, 2.0f * s.y - 1.0f);
    if (std::abs(p.x) < Epsilon && std::abs(p.y) < Epsilon) return Vec2(0, 0);
    float r, theta;
    if (std::abs(p.x) > std::abs(p.y)) {
        r = p.x;
        theta = (float)((M_PI / 4.0f) * (p.y / p.x));
    } else {
        r = p.y;
        theta = (float)((M_PI / 2.0f) - (M_PI / 4.0f) * (p.x / p.y));
    }
    return Vec2(r * std::cos(theta), r * std::sin(theta));
}
// warp.cpp:86-113: uniform point in a regular polygon with `blades` corners (one corner
// at the top), sampled as one of its triangles around the centre
inline Vec2 squareToUniformPolygon(const Vec2& s, int blades) {
    if (blades < 3) return squareToUniformDisk(s);
    float bladeFloat = s.x * blades;
    int bladeIdx = std::min(static_cast<int>(bladeFloat), blades - 1);
    float u0 = bladeFloat - bladeIdx;
    float u1 = s.y;
    float deltaTheta = 2.0f * Pi / blades;
    float theta1 = bladeIdx * deltaTheta;
    float theta2 = (bladeIdx + 1) * deltaTheta;
    float offset = Pi / 2.0f;
    theta1 += offset;
    theta2 += offset;
    Vec2 v1(std::cos(theta1), std::sin(theta1));
    Vec2 v2(std::cos(theta2), std::sin(theta2));
    float r = std::sqrt(u0);
    return Vec2(r * ((1.0f - u1) * v1.x + u1 * v2.x), r * ((1.0f - u1) * v1.y + u1 * v2.y));
}
// warp.cpp:35-44
inline Vec3 squareToUniformSphereCap(const Vec2& s, float cosThetaMax) {
    float theta = std::acos(1 - (1 - cosThetaMax) * s.x);
    float phi = (float)(2.0f * M_PI * s.y);
    return Vec3(std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta));
}
inline float squareToUniformSphereCapPdf(const Vec3& v, float cosThetaMax) {
    if (Dot(v, Vec3(0, 0, 1)) < cosThetaMax || std::abs(1 - v.lengthSquared()) > Epsilon) return 0.0f;
    return 1 / (2.0f * Pi * (1 - cosThetaMax));
}
inline Vec3 squareToUniformSphere(const Vec2& s) { return squareToUniformSphereCap(s, -1.0f); }
inline Vec3 squareToUniformHemisphere(const Vec2& s) { return squareToUniformSphereCap(s, 0.0f); }
// warp.cpp:69-78
inline Vec3 squareToCosineHemisphere(const Vec2& s) {
    Vec2 d = squareToUniformDisk(s);
    float r = d.lengthSquared();
    float z = std::sqrt(1 - r);
    return Vec3(d.x, d.y, z);
}
// warp.cpp:80-85
inline float squareToCosineHemispherePdf(const Vec3& v) {
    if (v.z <= 0.0f || std::abs(1 - v.lengthSquared()) > Epsilon) return 0.0f;
    return InvPi * v.z;
}
}  // namespace warp

}  // namespace orc
