// Motion blur: AnimatedTransform (animated.cpp:7-60) between a start transform (time 0)
// and an end transform (time 1) for instances and the camera. The reference decomposes
// both matrices with glm::decompose, interpolates translation and scale linearly and the
// rotation by glm::slerp, recomposes T * R * S and inverts it. The same algorithms are
// written out here: the unmatrix decomposition (scale and shear by Gram-Schmidt over the
// columns, a reflection folded into the scale, the quaternion by Shoemake's largest-
// component method), slerp with the linear fallback within FLT_EPSILON of parallel, and
// the inverse of the affine result by the adjugate of its 3x3 part. The host decomposes
// once per transform; kernels compose per ray.
#pragma once
#include "layout.h"

namespace gnd {

GND_HD float dot3a(const float a[3], const float b[3]) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

// Affine 3x4 matrix (row-major) -> translation t, scale s, rotation quaternion q (x,y,z,w)
GND_HD void motionDecompose(const Xf34& m, float t[3], float s[3], float q[4]) {
    for (int r = 0; r < 3; ++r) t[r] = m.r[r][3];
    float c[3][3];   // columns of the 3x3 part
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) c[k][r] = m.r[r][k];
    s[0] = sqrtf(dot3a(c[0], c[0]));
    for (int r = 0; r < 3; ++r) c[0][r] = c[0][r] * (1.0f / s[0]);
    const float skz = dot3a(c[0], c[1]);
    for (int r = 0; r < 3; ++r) c[1][r] = c[1][r] + c[0][r] * (-skz);
    s[1] = sqrtf(dot3a(c[1], c[1]));
    for (int r = 0; r < 3; ++r) c[1][r] = c[1][r] * (1.0f / s[1]);
    const float sky = dot3a(c[0], c[2]);
    for (int r = 0; r < 3; ++r) c[2][r] = c[2][r] + c[0][r] * (-sky);
    const float skx = dot3a(c[1], c[2]);
    for (int r = 0; r < 3; ++r) c[2][r] = c[2][r] + c[1][r] * (-skx);
    s[2] = sqrtf(dot3a(c[2], c[2]));
    for (int r = 0; r < 3; ++r) c[2][r] = c[2][r] * (1.0f / s[2]);
    const float cr[3] = {c[1][1] * c[2][2] - c[1][2] * c[2][1], c[1][2] * c[2][0] - c[1][0] * c[2][2],
                         c[1][0] * c[2][1] - c[1][1] * c[2][0]};
    if (dot3a(c[0], cr) < 0.0f) {
        for (int k = 0; k < 3; ++k) {
            s[k] = -s[k];
            for (int r = 0; r < 3; ++r) c[k][r] = -c[k][r];
        }
    }
    // rotation R[row][col] = c[col][row]
    const float r00 = c[0][0], r11 = c[1][1], r22 = c[2][2];
    const float trace = (r00 + r11) + r22;
    if (trace > 0.0f) {
        float root = sqrtf(trace + 1.0f);
        q[3] = 0.5f * root;
        root = 0.5f / root;
        q[0] = root * (c[1][2] - c[2][1]);
        q[1] = root * (c[2][0] - c[0][2]);
        q[2] = root * (c[0][1] - c[1][0]);
    } else if (r00 >= r11 && r00 >= r22) {
        float root = sqrtf(((1.0f + r00) - r11) - r22);
        q[0] = 0.5f * root;
        root = 0.5f / root;
        q[1] = (c[1][0] + c[0][1]) * root;
        q[2] = (c[2][0] + c[0][2]) * root;
        q[3] = (c[1][2] - c[2][1]) * root;
    } else if (r11 >= r22) {
        float root = sqrtf(((1.0f + r11) - r00) - r22);
        q[1] = 0.5f * root;
        root = 0.5f / root;
        q[0] = (c[1][0] + c[0][1]) * root;
        q[2] = (c[2][1] + c[1][2]) * root;
        q[3] = (c[2][0] - c[0][2]) * root;
    } else {
        float root = sqrtf(((1.0f + r22) - r00) - r11);
        q[2] = 0.5f * root;
        root = 0.5f / root;
        q[0] = (c[2][0] + c[0][2]) * root;
        q[1] = (c[2][1] + c[1][2]) * root;
        q[3] = (c[0][1] - c[1][0]) * root;
    }
}

// The matrix at dt in (0, 1) and its inverse (row-major 3x4)
GND_HD void motionCompose(const InstMotion& k, float dt, Xf34& M, Xf34& Minv) {
    float t[3], s[3], q[4], z[4];
    const float* t0 = k.t0; const float* t1 = k.t1;
    const float* s0 = k.s0; const float* s1 = k.s1;
    const float* q0 = k.q0; const float* q1 = k.q1;
    for (int i = 0; i < 3; ++i) {
        t[i] = t0[i] * (1.0f - dt) + t1[i] * dt;
        s[i] = s0[i] * (1.0f - dt) + s1[i] * dt;
    }
    float cosT = ((q0[0] * q1[0] + q0[1] * q1[1]) + q0[2] * q1[2]) + q0[3] * q1[3];
    for (int i = 0; i < 4; ++i) z[i] = q1[i];
    if (cosT < 0.0f) {
        for (int i = 0; i < 4; ++i) z[i] = -z[i];
        cosT = -cosT;
    }
    if (cosT > 1.0f - 1.1920929e-7f) {
        for (int i = 0; i < 4; ++i) q[i] = q0[i] * (1.0f - dt) + z[i] * dt;
    } else {
        const float angle = acosf(cosT);
        const float w0 = sinf((1.0f - dt) * angle), w1 = sinf(dt * angle), sa = sinf(angle);
        for (int i = 0; i < 4; ++i) q[i] = (q0[i] * w0 + z[i] * w1) / sa;
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
            M.r[r][c] = A[r][c];
        }
        M.r[r][3] = t[r];
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
        for (int c = 0; c < 3; ++c) Minv.r[r][c] = B[r][c];
        Minv.r[r][3] = -((B[r][0] * t[0] + B[r][1] * t[1]) + B[r][2] * t[2]);
    }
}

// AnimatedTransform::interpolate (animated.cpp:29-47) with start time 0 and end time 1:
// the start matrices at time <= 0, the end matrices at time >= 1, else the composition.
GND_HD void motionAt(const InstMotion& k, const Xf34& startO2W, const Xf34& startW2O, float time, Xf34& o2w, Xf34& w2o) {
    if (time <= 0.0f) { o2w = startO2W; w2o = startW2O; return; }
    if (time >= 1.0f) { o2w = k.endO2W; w2o = k.endW2O; return; }
    motionCompose(k, (time - 0.0f) / (1.0f - 0.0f), o2w, w2o);
}

}  // namespace gnd
