// Oracle (test infrastructure only): AnimatedTransform (animated.cpp:7-60), the motion of
// a primitive or camera between toWorld (time 0) and toWorldEnd (time 1).
//
// The reference decomposes both matrices with glm::decompose, interpolates translation and
// scale linearly and the rotation by glm::slerp, recomposes T * R * S and inverts with
// glm::inverse. glm is not part of the reference sources, so its published algorithms are
// restated here: the unmatrix decomposition (scale and shear by Gram-Schmidt on the
// columns, a reflection folded into the scale, the rotation quaternion by Shoemake's
// largest-component method), slerp with the linear fallback when the quaternions are
// within FLT_EPSILON of parallel, and the inverse of the affine result by the adjugate of
// its 3x3 part. The GPU (gnd/motion.h) and the host framework run the same operations in
// the same order; bit parity with glm itself is not claimed (glm is absent here).
#pragma once
#include <cmath>

#include "omath.h"

namespace orc {

struct MotionKeys {
    float T[2][3], S[2][3], Q[2][4];   // translation, scale, rotation quaternion (x, y, z, w)
};

namespace motion {

inline float dot3(const float a[3], const float b[3]) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

// Affine matrix (column-major Mat4) -> translation, scale, rotation
inline void decompose(const Mat4& m, float T[3], float S[3], float Q[4]) {
    for (int r = 0; r < 3; ++r) T[r] = m.c[3][r];
    float c[3][3];   // columns of the 3x3 part
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) c[k][r] = m.c[k][r];
    S[0] = std::sqrt(dot3(c[0], c[0]));
    for (int r = 0; r < 3; ++r) c[0][r] = c[0][r] * (1.0f / S[0]);
    float skz = dot3(c[0], c[1]);
    for (int r = 0; r < 3; ++r) c[1][r] = c[1][r] + c[0][r] * (-skz);
    S[1] = std::sqrt(dot3(c[1], c[1]));
    for (int r = 0; r < 3; ++r) c[1][r] = c[1][r] * (1.0f / S[1]);
    float sky = dot3(c[0], c[2]);
    for (int r = 0; r < 3; ++r) c[2][r] = c[2][r] + c[0][r] * (-sky);
    float skx = dot3(c[1], c[2]);
    for (int r = 0; r < 3; ++r) c[2][r] = c[2][r] + c[1][r] * (-skx);
    S[2] = std::sqrt(dot3(c[2], c[2]));
    for (int r = 0; r < 3; ++r) c[2][r] = c[2][r] * (1.0f / S[2]);
    const float cr[3] = {c[1][1] * c[2][2] - c[1][2] * c[2][1], c[1][2] * c[2][0] - c[1][0] * c[2][2],
                         c[1][0] * c[2][1] - c[1][1] * c[2][0]};
    if (dot3(c[0], cr) < 0.0f) {
        for (int k = 0; k < 3; ++k) {
            S[k] = -S[k];
            for (int r = 0; r < 3; ++r) c[k][r] = -c[k][r];
        }
    }
    // rotation R[row][col] = c[col][row]
    const float r00 = c[0][0], r11 = c[1][1], r22 = c[2][2];
    const float trace = (r00 + r11) + r22;
    if (trace > 0.0f) {
        float root = std::sqrt(trace + 1.0f);
        Q[3] = 0.5f * root;
        root = 0.5f / root;
        Q[0] = root * (c[1][2] - c[2][1]);
        Q[1] = root * (c[2][0] - c[0][2]);
        Q[2] = root * (c[0][1] - c[1][0]);
    } else if (r00 >= r11 && r00 >= r22) {
        float root = std::sqrt(((1.0f + r00) - r11) - r22);
        Q[0] = 0.5f * root;
        root = 0.5f / root;
        Q[1] = (c[1][0] + c[0][1]) * root;
        Q[2] = (c[2][0] + c[0][2]) * root;
        Q[3] = (c[1][2] - c[2][1]) * root;
    } else if (r11 >= r22) {
        float root = std::sqrt(((1.0f + r11) - r00) - r22);
        Q[1] = 0.5f * root;
        root = 0.5f / root;
        Q[0] = (c[1][0] + c[0][1]) * root;
        Q[2] = (c[2][1] + c[1][2]) * root;
        Q[3] = (c[2][0] - c[0][2]) * root;
    } else {
        float root = std::sqrt(((1.0f + r22) - r00) - r11);
        Q[2] = 0.5f * root;
        root = 0.5f / root;
        Q[0] = (c[2][0] + c[0][2]) * root;
        Q[1] = (c[2][1] + c[1][2]) * root;
        Q[3] = (c[0][1] - c[1][0]) * root;
    }
}

// Interpolated matrix at dt in (0, 1): row-major 3x4 [A | t] and its inverse
inline void compose(const MotionKeys& k, float dt, float M[3][4], float Minv[3][4]) {
    float t[3], s[3], q[4], z[4];
    for (int i = 0; i < 3; ++i) {
        t[i] = k.T[0][i] * (1.0f - dt) + k.T[1][i] * dt;
        s[i] = k.S[0][i] * (1.0f - dt) + k.S[1][i] * dt;
    }
    float cosT = ((k.Q[0][0] * k.Q[1][0] + k.Q[0][1] * k.Q[1][1]) + k.Q[0][2] * k.Q[1][2]) + k.Q[0][3] * k.Q[1][3];
    for (int i = 0; i < 4; ++i) z[i] = k.Q[1][i];
    if (cosT < 0.0f) {
        for (int i = 0; i < 4; ++i) z[i] = -z[i];
        cosT = -cosT;
    }
    if (cosT > 1.0f - 1.1920929e-7f) {
        for (int i = 0; i < 4; ++i) q[i] = k.Q[0][i] * (1.0f - dt) + z[i] * dt;
    } else {
        const float angle = std::acos(cosT);
        const float s0 = std::sin((1.0f - dt) * angle), s1 = std::sin(dt * angle), sa = std::sin(angle);
        for (int i = 0; i < 4; ++i) q[i] = (k.Q[0][i] * s0 + z[i] * s1) / sa;
    }
    const float xx = q[0] * q[0], yy = q[1] * q[1], zz = q[2] * q[2];
    const float xy = q[0] * q[1], xz = q[0] * q[2], yz = q[1] * q[2];
    const float wx = q[3] * q[0], wy = q[3] * q[1], wz = q[3] * q[2];
    const float R[3][3] = {{1.0f - 2.0f * (yy + zz), 2.0f * (xy - wz), 2.0f * (xz + wy)},
                           {2.0f * (xy + wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz - wx)},
                           {2.0f * (xz - wy), 2.0f * (yz + wx), 1.0f - 2.0f * (xx + yy)}};
    float A[3][3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            A[r][c] = R[r][c] * s[c];
            M[r][c] = A[r][c];
        }
        M[r][3] = t[r];
    }
    const float c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    const float c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    const float c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    const float inv = 1.0f / ((A[0][0] * c00 + A[0][1] * c01) + A[0][2] * c02);
    float B[3][3];
    B[0][0] = c00 * inv;
    B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * inv;
    B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * inv;
    B[1][0] = c01 * inv;
    B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * inv;
    B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * inv;
    B[2][0] = c02 * inv;
    B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * inv;
    B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * inv;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) Minv[r][c] = B[r][c];
        Minv[r][3] = -((B[r][0] * t[0] + B[r][1] * t[1]) + B[r][2] * t[2]);
    }
}

inline Mat4 toMat4(const float M[3][4]) {
    Mat4 m;   // identity bottom row
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) m.c[c][r] = M[r][c];
    return m;
}

}  // namespace motion

// animated.cpp:7-60 with the start and end times 0 and 1 (primitive.cpp:7-11, camera.h:20-25)
struct AnimatedTransform {
    Transform start, end;
    bool animated = false;
    MotionKeys keys{};
    void set(const Transform& t1, const Transform& t2) {
        start = t1;
        end = t2;
        animated = !(t1 == t2);
        if (animated) {
            motion::decompose(t1.m, keys.T[0], keys.S[0], keys.Q[0]);
            motion::decompose(t2.m, keys.T[1], keys.S[1], keys.Q[1]);
        }
    }
    Transform interpolate(float time) const {
        if (!animated || time <= 0.0f) return start;
        if (time >= 1.0f) return end;
        const float dt = (time - 0.0f) / (1.0f - 0.0f);
        float M[3][4], Minv[3][4];
        motion::compose(keys, dt, M, Minv);
        return Transform(motion::toMat4(M), motion::toMat4(Minv));
    }
    Bounds3 motionBounds(const Bounds3& b) const {
        if (!animated) return start.bounds(b);
        Bounds3 r = Union(start.bounds(b), end.bounds(b));
        return Union(r, interpolate((0.0f + 1.0f) * 0.5f).bounds(b));
    }
};

}  // namespace orc
