// Host/device vector math for the GPU integrators and the host scene builder.
//
// Operation order follows the reference's glm/Highway arithmetic so that geometry
// (transforms, slab and triangle tests) is bit-reproducible between host and device:
// every translation unit is compiled without multiply-add contraction
// (nvcc -fmad=false, g++ -ffp-contract=off).
//   dot(a,b)       = (a.x*b.x + a.y*b.y) + a.z*b.z          (geometry.h:243)
//   normalize(v)   = v * (1/sqrt(dot(v,v)))                 (geometry.h:253)
//   M*(x,y,z,w)    = (c0*x + c1*y) + (c2*z + c3*w)          (transform.h:330-343)
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define GND_HD __host__ __device__ __forceinline__
#else
#define GND_HD inline
#endif

namespace gnd {

constexpr float kEpsilon = 0.0001f;                          // constants.h:13
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInv2Pi = 0.15915494309189533577f;
constexpr float kInv4Pi = 0.07957747154594766788f;
constexpr float kInvPiD = (float)0.318309886183790671538;    // M_1_PI as a float
constexpr double kPiD = 3.14159265358979323846;

struct V3 {
    float x, y, z;
};
struct V2 {
    float x, y;
};

GND_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
GND_HD V3 v3s(float s) { return V3{s, s, s}; }
GND_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
GND_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
GND_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
GND_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
GND_HD V3 operator*(float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
GND_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
// vector / scalar divides each component (glm vec3 / s)
GND_HD V3 divs(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
// Color / scalar multiplies by the reciprocal (color.h:41)
GND_HD V3 cdiv(V3 a, float s) { float inv = 1.0f / s; return V3{a.x * inv, a.y * inv, a.z * inv}; }
GND_HD float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
GND_HD float lengthSq(V3 a) { return dot(a, a); }
GND_HD float length(V3 a) { return sqrtf(dot(a, a)); }
GND_HD V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
GND_HD V3 normalize(V3 v) {
    float inv = 1.0f / sqrtf(dot(v, v));
    return v * inv;
}
GND_HD float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
GND_HD bool isBlack(V3 c) { return c.x <= 0.0f && c.y <= 0.0f && c.z <= 0.0f; }   // color.h:52-54
GND_HD float luminance(V3 c) { return c.x * 0.212671f + c.y * 0.715160f + c.z * 0.072169f; }  // color.h:48-50
GND_HD float fminf_(float a, float b) { return a < b ? a : b; }
GND_HD float fmaxf_(float a, float b) { return a > b ? a : b; }
GND_HD float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Affine 3x4 transform stored as rows: r[k] = (m[0][k], m[1][k], m[2][k], m[3][k]) of the
// column-major 4x4 matrix, so a point maps with the glm column sum order.
struct Xf34 {
    float r[3][4];
};
GND_HD V3 xfPoint(const Xf34& m, V3 p) {
    // w of an affine matrix is exactly 1, so no perspective division
    V3 o;
    o.x = (m.r[0][0] * p.x + m.r[0][1] * p.y) + (m.r[0][2] * p.z + m.r[0][3]);
    o.y = (m.r[1][0] * p.x + m.r[1][1] * p.y) + (m.r[1][2] * p.z + m.r[1][3]);
    o.z = (m.r[2][0] * p.x + m.r[2][1] * p.y) + (m.r[2][2] * p.z + m.r[2][3]);
    return o;
}
GND_HD V3 xfVector(const Xf34& m, V3 v) {
    V3 o;
    o.x = (m.r[0][0] * v.x + m.r[0][1] * v.y) + (m.r[0][2] * v.z + m.r[0][3] * 0.0f);
    o.y = (m.r[1][0] * v.x + m.r[1][1] * v.y) + (m.r[1][2] * v.z + m.r[1][3] * 0.0f);
    o.z = (m.r[2][0] * v.x + m.r[2][1] * v.y) + (m.r[2][2] * v.z + m.r[2][3] * 0.0f);
    return o;
}
// Normal transform of the forward matrix F given its inverse I: transpose(mat3(I)) * n,
// rows summed left to right (transform.h:345-348): out[i] = I[0][i]*n.x + I[1][i]*n.y + I[2][i]*n.z
// with I[c][r] column-major, i.e. out[i] = I.r[0][i]... -> column i of the row storage.
GND_HD V3 xfNormal(const Xf34& inv, V3 n) {
    V3 o;
    o.x = inv.r[0][0] * n.x + inv.r[1][0] * n.y + inv.r[2][0] * n.z;
    o.y = inv.r[0][1] * n.x + inv.r[1][1] * n.y + inv.r[2][1] * n.z;
    o.z = inv.r[0][2] * n.x + inv.r[1][2] * n.y + inv.r[2][2] * n.z;
    return o;
}

// frame.h:17-33
struct Frame {
    V3 x, y, z;
};
GND_HD Frame frameFromNormal(V3 n) {
    Frame f;
    f.z = n;
    float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    f.x = v3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    f.y = v3(b, sign + n.y * n.y * a, -n.y);
    return f;
}
GND_HD V3 toLocal(const Frame& f, V3 v) { return v3(dot(v, f.x), dot(v, f.y), dot(v, f.z)); }
GND_HD V3 toWorld(const Frame& f, V3 v) { return (f.x * v.x + f.y * v.y) + f.z * v.z; }

}  // namespace gnd
