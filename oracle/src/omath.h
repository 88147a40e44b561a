// Oracle (test infrastructure only): scalar CPU restatement of the math layer the
// reference's radiance path runs on. Nothing in the product links this code; tests,
// the smoke check and the bench's CPU-baseline leg use it as the checker.
//
// The reference builds its vectors on glm and its 4-wide kernels on Highway; neither
// is present here, so this file restates the operations they perform, keeping the
// operation order so that results are bit-reproducible when compiled with
// -ffp-contract=off:
//   * dot = (x*x' + y*y') + z*z'                         (glm::dot, geometry.h:243)
//   * normalize = v * (1/sqrt(dot(v,v)))                 (glm::normalize, geometry.h:253)
//   * mat4 * vec4 = (c0*x + c1*y) + (c2*z + c3*w)        (glm mat4 product, transform.h:330-343)
//   * vec / scalar divides each component                (glm vec3 / s)
//   * Color / s multiplies by 1/s                        (color.h:41)
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <algorithm>
#include <string>

namespace orc {

constexpr float Infinity = std::numeric_limits<float>::infinity();
constexpr float Epsilon = 0.0001f;                       // constants.h:13
constexpr float Pi = 3.14159265358979323846f;            // constants.h:15
constexpr float InvPi = 0.31830988618379067154f;
constexpr float Inv2Pi = 0.15915494309189533577f;
constexpr float Inv4Pi = 0.07957747154594766788f;

struct Vec2 {
    float x = 0, y = 0;
    Vec2() = default;
    Vec2(float a, float b) : x(a), y(b) {}
    Vec2 operator+(const Vec2& o) const { return {x + o.x, y + o.y}; }
    Vec2 operator-(const Vec2& o) const { return {x - o.x, y - o.y}; }
    Vec2 operator*(float s) const { return {x * s, y * s}; }
    float lengthSquared() const { return x * x + y * y; }
};

struct Vec3 {
    float x = 0, y = 0, z = 0;
    Vec3() = default;
    explicit Vec3(float a) : x(a), y(a), z(a) {}
    Vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    Vec3 operator*(float s) const { return {x * s, y * s, z * s}; }
    Vec3 operator/(float s) const { return {x / s, y / s, z / s}; }
    Vec3 operator-() const { return {-x, -y, -z}; }
    Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    float lengthSquared() const { return (x * x + y * y) + z * z; }
    float length() const { return std::sqrt(lengthSquared()); }
    bool hasNaNs() const { return std::isnan(x) || std::isnan(y) || std::isnan(z); }
};
inline Vec3 operator*(float s, const Vec3& v) { return v * s; }
inline float Dot(const Vec3& a, const Vec3& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float AbsDot(const Vec3& a, const Vec3& b) { return std::abs(Dot(a, b)); }
inline Vec3 Cross(const Vec3& a, const Vec3& b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline Vec3 Normalize(const Vec3& v) {
    float inv = 1.0f / std::sqrt(Dot(v, v));
    return v * inv;
}

struct Color {
    float r = 0, g = 0, b = 0;
    Color() = default;
    Color(float v) : r(v), g(v), b(v) {}
    Color(float a, float b_, float c) : r(a), g(b_), b(c) {}
    float operator[](int i) const { return i == 0 ? r : (i == 1 ? g : b); }
    Color operator+(const Color& o) const { return {r + o.r, g + o.g, b + o.b}; }
    Color operator-(const Color& o) const { return {r - o.r, g - o.g, b - o.b}; }
    Color operator*(const Color& o) const { return {r * o.r, g * o.g, b * o.b}; }
    Color operator*(float s) const { return {r * s, g * s, b * s}; }
    Color operator/(float s) const { float inv = 1.0f / s; return {r * inv, g * inv, b * inv}; }
    Color& operator+=(const Color& o) { r += o.r; g += o.g; b += o.b; return *this; }
    Color& operator*=(const Color& o) { r *= o.r; g *= o.g; b *= o.b; return *this; }
    Color& operator*=(float s) { r *= s; g *= s; b *= s; return *this; }
    Color& operator/=(float s) { float inv = 1.0f / s; r *= inv; g *= inv; b *= inv; return *this; }
    // color.h:48-50
    float luminance() const { return r * 0.212671f + g * 0.715160f + b * 0.072169f; }
    // color.h:52-54
    bool isBlack() const { return r <= 0.0f && g <= 0.0f && b <= 0.0f; }
    // color.h:56-59 (NaN or Inf)
    bool hasNaNs() const {
        return std::isnan(r) || std::isnan(g) || std::isnan(b) || std::isinf(r) || std::isinf(g) ||
               std::isinf(b);
    }
};
inline Color operator*(float s, const Color& c) { return c * s; }

// Column-major 4x4 matrix, c[col][row], like glm::mat4.
struct Mat4 {
    float c[4][4];
    Mat4() { for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) c[i][j] = (i == j) ? 1.f : 0.f; }
    static Mat4 zero() { Mat4 m; for (auto& col : m.c) for (float& v : col) v = 0.f; return m; }
    // (c0*x + c1*y) + (c2*z + c3*w), per row
    void mulVec(const float v[4], float out[4]) const {
        for (int r = 0; r < 4; ++r) {
            float a0 = c[0][r] * v[0];
            float a1 = c[1][r] * v[1];
            float add0 = a0 + a1;
            float a2 = c[2][r] * v[2];
            float a3 = c[3][r] * v[3];
            float add1 = a2 + a3;
            out[r] = add0 + add1;
        }
    }
    Mat4 operator*(const Mat4& b) const {
        Mat4 m;
        for (int col = 0; col < 4; ++col) mulVec(b.c[col], m.c[col]);
        return m;
    }
    Mat4 transpose() const {
        Mat4 m;
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) m.c[i][j] = c[j][i];
        return m;
    }
    bool operator==(const Mat4& o) const {
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) if (c[i][j] != o.c[i][j]) return false;
        return true;
    }
};

// General 4x4 inverse by cofactor expansion (the role glm::inverse plays for LookAt,
// transform.h:428-431). Only the camera uses it; instance inverses are composed.
Mat4 Inverse(const Mat4& m);

struct Bounds3 {
    Vec3 pMin, pMax;
    // bounds.h:151-156: empty box is (max, lowest)
    Bounds3() {
        float lo = std::numeric_limits<float>::lowest(), hi = std::numeric_limits<float>::max();
        pMin = Vec3(hi); pMax = Vec3(lo);
    }
    explicit Bounds3(const Vec3& p) : pMin(p), pMax(p) {}
    Bounds3(const Vec3& a, const Vec3& b)
        : pMin(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)),
          pMax(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)) {}
    Vec3 diagonal() const { return pMax - pMin; }
    // bounds.h:184-187
    float surfaceArea() const { Vec3 d = diagonal(); return 2.f * (d.x * d.y + d.x * d.z + d.y * d.z); }
    // bounds.h:196-203
    int maximumExtent() const {
        Vec3 d = diagonal();
        if (d.x > d.y && d.x > d.z) return 0;
        if (d.y > d.z) return 1;
        return 2;
    }
    Vec3 corner(int i) const {
        return Vec3((i & 1) ? pMax.x : pMin.x, (i & 2) ? pMax.y : pMin.y, (i & 4) ? pMax.z : pMin.z);
    }
    // bounds.h:214-216
    Vec3 centroid() const { return pMin * 0.5f + pMax * 0.5f; }
};
inline Bounds3 Union(const Bounds3& a, const Bounds3& b) {
    Bounds3 r;
    r.pMin = Vec3(std::min(a.pMin.x, b.pMin.x), std::min(a.pMin.y, b.pMin.y), std::min(a.pMin.z, b.pMin.z));
    r.pMax = Vec3(std::max(a.pMax.x, b.pMax.x), std::max(a.pMax.y, b.pMax.y), std::max(a.pMax.z, b.pMax.z));
    return r;
}
inline Bounds3 Union(const Bounds3& a, const Vec3& p) {
    Bounds3 r;
    r.pMin = Vec3(std::min(a.pMin.x, p.x), std::min(a.pMin.y, p.y), std::min(a.pMin.z, p.z));
    r.pMax = Vec3(std::max(a.pMax.x, p.x), std::max(a.pMax.y, p.y), std::max(a.pMax.z, p.z));
    return r;
}

class Medium;

// ray.h:12-33: tMin/tMax are mutable (traversal shrinks tMax); tMin defaults to Epsilon.
struct Ray {
    Vec3 o, d;
    mutable float tMin = Epsilon;
    mutable float tMax = Infinity;
    const Medium* medium = nullptr;
    float time = 0.0f;
    Ray() = default;
    Ray(const Vec3& o_, const Vec3& d_, float tmax = Infinity) : o(o_), d(d_), tMin(Epsilon), tMax(tmax) {}
};

// bounds.h:244-264: scalar slab test used by the reference's unit tests.
inline bool BoundsIntersect(const Bounds3& b, const Ray& ray, float* hitt0, float* hitt1) {
    float t0 = 0.f, t1 = ray.tMax;
    for (int i = 0; i < 3; ++i) {
        float inv = 1.f / ray.d[i];
        float tn = (b.pMin[i] - ray.o[i]) * inv;
        float tf = (b.pMax[i] - ray.o[i]) * inv;
        if (tn > tf) std::swap(tn, tf);
        t0 = tn > t0 ? tn : t0;
        t1 = tf < t1 ? tf : t1;
        if (t0 > t1) return false;
    }
    if (hitt0) *hitt0 = t0;
    if (hitt1) *hitt1 = t1;
    return true;
}

// transform.h:299-437. Keeps both the matrix and its inverse; composition multiplies
// both (so instance inverses are products of exact step inverses, not glm::inverse).
struct Transform {
    Mat4 m, mInv;
    Transform() = default;
    Transform(const Mat4& a, const Mat4& b) : m(a), mInv(b) {}
    Transform inverse() const { return Transform(mInv, m); }
    Transform operator*(const Transform& t2) const { return Transform(m * t2.m, t2.mInv * mInv); }
    bool operator==(const Transform& o) const { return m == o.m; }
    Vec3 point(const Vec3& p) const {
        float in[4] = {p.x, p.y, p.z, 1.f}, out[4];
        m.mulVec(in, out);
        if (out[3] == 1.0f) return Vec3(out[0], out[1], out[2]);
        return Vec3(out[0] / out[3], out[1] / out[3], out[2] / out[3]);
    }
    Vec3 vector(const Vec3& v) const {
        float in[4] = {v.x, v.y, v.z, 0.f}, out[4];
        m.mulVec(in, out);
        return Vec3(out[0], out[1], out[2]);
    }
    // transform.h:345-348: transpose(mat3(mInv)) * n, rows summed left to right
    Vec3 normal(const Vec3& n) const {
        Vec3 r;
        for (int i = 0; i < 3; ++i) r[i] = mInv.c[i][0] * n.x + mInv.c[i][1] * n.y + mInv.c[i][2] * n.z;
        return r;
    }
    // transform.h:350-354: new Ray => tMin reset to Epsilon, d not renormalised
    Ray ray(const Ray& r) const { return Ray(point(r.o), vector(r.d), r.tMax); }
    Bounds3 bounds(const Bounds3& b) const {
        Bounds3 ret(point(b.corner(0)));
        for (int i = 1; i < 8; ++i) ret = Union(ret, point(b.corner(i)));
        return ret;
    }
    static Transform Translate(const Vec3& d);
    static Transform Scale(float x, float y, float z);
    static Transform Rotate(float degrees, const Vec3& axis);
    static Transform LookAt(const Vec3& pos, const Vec3& target, const Vec3& up);
};

// constants.h:46-54
inline bool SolveQuadratic(float a, float b, float c, float& r0, float& r1) {
    float discrim = b * b - 4.0f * a * c;
    if (discrim < 0) return false;
    float rd = std::sqrt(discrim);
    r0 = (-b - rd) / (2.0f * a);
    r1 = (-b + rd) / (2.0f * a);
    return true;
}

// frame.h:17-33
struct Frame {
    Vec3 x{1, 0, 0}, y{0, 1, 0}, z{0, 0, 1};
    Frame() = default;
    Frame(const Vec3& a, const Vec3& b, const Vec3& c) : x(a), y(b), z(c) {}
    static Frame fromNormal(const Vec3& n) {
        Frame f;
        f.z = n;
        float sign = std::copysign(1.0f, n.z);
        const float a = -1.0f / (sign + n.z);
        const float b = n.x * n.y * a;
        f.x = Vec3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
        f.y = Vec3(b, sign + n.y * n.y * a, -n.y);
        return f;
    }
    Vec3 toLocal(const Vec3& v) const { return Vec3(Dot(v, x), Dot(v, y), Dot(v, z)); }
    Vec3 toWorld(const Vec3& v) const { return (x * v.x + y * v.y) + z * v.z; }
};

}  // namespace orc
