// pe_xform.h — 4×4 transforms of mesh instances, shared by the host scene builder and the kernels:
// Mat4f::inverse (src/core/math/mat.h:130-175), the determinant MeshInstance uses for texel
// density (mesh_instance.cpp:11-15) and the motion-blur interpolation of a moving instance,
// interpolateTransform (src/core/math/quat.cpp): translation and scale linear, rotation by SLERP
// of unit quaternions in double precision, recomposed as T·R·S and inverted again.
//
// The pose at a shutter time splits into what depends only on the two end poses (decomposeTRS of
// each, the quaternions normalised and put on the short arc, the arc angle and its sine: host,
// once per instance, with the C library's acos / sin as the reference calls them) and what
// depends on the time (motionPoseAt: two sines, a normalisation, the matrix and its inverse).
// Matrices are row-major float[16] with column vectors; everything is compiled without FMA
// contraction, in the reference's operand order.
#pragma once

#include "pe_math.h"

namespace pe {

// Mat4f::inverse: cofactors from the 2×2 minors of the top and bottom row pairs; the identity for
// a singular matrix.
PE_HD void mat4Inverse(const float* m, float* o) {
    const float s0 = m[0] * m[5] - m[4] * m[1];
    const float s1 = m[0] * m[6] - m[4] * m[2];
    const float s2 = m[0] * m[7] - m[4] * m[3];
    const float s3 = m[1] * m[6] - m[5] * m[2];
    const float s4 = m[1] * m[7] - m[5] * m[3];
    const float s5 = m[2] * m[7] - m[6] * m[3];
    const float c5 = m[10] * m[15] - m[14] * m[11];
    const float c4 = m[9] * m[15] - m[13] * m[11];
    const float c3 = m[9] * m[14] - m[13] * m[10];
    const float c2 = m[8] * m[15] - m[12] * m[11];
    const float c1 = m[8] * m[14] - m[12] * m[10];
    const float c0 = m[8] * m[13] - m[12] * m[9];
    const float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    if (det == 0.0f) {
        for (int k = 0; k < 16; ++k) o[k] = (k % 5 == 0) ? 1.0f : 0.0f;
        return;
    }
    const float id = 1.0f / det;
    o[0] = (m[5] * c5 - m[6] * c4 + m[7] * c3) * id;
    o[1] = (-m[1] * c5 + m[2] * c4 - m[3] * c3) * id;
    o[2] = (m[13] * s5 - m[14] * s4 + m[15] * s3) * id;
    o[3] = (-m[9] * s5 + m[10] * s4 - m[11] * s3) * id;
    o[4] = (-m[4] * c5 + m[6] * c2 - m[7] * c1) * id;
    o[5] = (m[0] * c5 - m[2] * c2 + m[3] * c1) * id;
    o[6] = (-m[12] * s5 + m[14] * s2 - m[15] * s1) * id;
    o[7] = (m[8] * s5 - m[10] * s2 + m[11] * s1) * id;
    o[8] = (m[4] * c4 - m[5] * c2 + m[7] * c0) * id;
    o[9] = (-m[0] * c4 + m[1] * c2 - m[3] * c0) * id;
    o[10] = (m[12] * s4 - m[13] * s2 + m[15] * s0) * id;
    o[11] = (-m[8] * s4 + m[9] * s2 - m[11] * s0) * id;
    o[12] = (-m[4] * c3 + m[5] * c1 - m[6] * c0) * id;
    o[13] = (m[0] * c3 - m[1] * c1 + m[2] * c0) * id;
    o[14] = (-m[12] * s3 + m[13] * s1 - m[14] * s0) * id;
    o[15] = (m[8] * s3 - m[9] * s1 + m[10] * s0) * id;
}

// det3x3 of the upper 3×3 block (mesh_instance.cpp:11-15).
PE_HD float det3x3(const float* m) {
    return m[0] * (m[5] * m[10] - m[6] * m[9]) - m[1] * (m[4] * m[10] - m[6] * m[8]) +
           m[2] * (m[4] * m[9] - m[5] * m[8]);
}

// Texel-density scale of a transform: cbrt(max(|det|, 1e-12)) (mesh_instance.cpp:95-98).
PE_HD float uvScaleOf(const float* m) {
    return cbrtf(smax(fabsf(det3x3(m)), 1e-12f));
}

// The time-independent half of interpolateTransform for one moving instance.
struct MotionTRS {
    float p0[3], p1[3];   // translations at t0 and t1
    float s0[3], s1[3];   // signed scales (a negative determinant flips z)
    double qa[4], qb[4];  // unit rotations (x, y, z, w) as doubles, qb on the short arc from qa
    double theta, sinT;   // SLERP arc angle and its sine
    int32_t linear;       // arcs with cos > 0.9995 are interpolated linearly
    int32_t pad;
};

// Quatf::normalized (quat.cpp): in double, identity for a near-zero quaternion.
PE_HD void quatNormalized(const float* q, float* out) {
    const double dx = q[0], dy = q[1], dz = q[2], dw = q[3];
    const double len2 = dx * dx + dy * dy + dz * dz + dw * dw;
    if (!(len2 > 1e-16)) {
        out[0] = out[1] = out[2] = 0.0f;
        out[3] = 1.0f;
        return;
    }
    const double inv = 1.0 / sqrt(len2);
    out[0] = static_cast<float>(dx * inv);
    out[1] = static_cast<float>(dy * inv);
    out[2] = static_cast<float>(dz * inv);
    out[3] = static_cast<float>(dw * inv);
}

// Quatf::toMat4 then composeTRS (quat.cpp): rotation of the re-normalised quaternion, columns
// scaled, translation in the last column; the bottom row 0 0 0 1.
PE_HD void composeTRS(const float* p, const float* qIn, const float* s, float* m) {
    float q[4];
    quatNormalized(qIn, q);
    const float xx = q[0] * q[0], yy = q[1] * q[1], zz = q[2] * q[2];
    const float xy = q[0] * q[1], xz = q[0] * q[2], yz = q[1] * q[2];
    const float wx = q[3] * q[0], wy = q[3] * q[1], wz = q[3] * q[2];
    m[0] = (1.0f - 2.0f * (yy + zz)) * s[0];
    m[1] = (2.0f * (xy - wz)) * s[1];
    m[2] = (2.0f * (xz + wy)) * s[2];
    m[3] = p[0];
    m[4] = (2.0f * (xy + wz)) * s[0];
    m[5] = (1.0f - 2.0f * (xx + zz)) * s[1];
    m[6] = (2.0f * (yz - wx)) * s[2];
    m[7] = p[1];
    m[8] = (2.0f * (xz - wy)) * s[0];
    m[9] = (2.0f * (yz + wx)) * s[1];
    m[10] = (1.0f - 2.0f * (xx + yy)) * s[2];
    m[11] = p[2];
    m[12] = 0.0f;
    m[13] = 0.0f;
    m[14] = 0.0f;
    m[15] = 1.0f;
}

// interpolateTransform(t0, t1, a) for 0 < a < 1: the matrix and (Transform(m)) its inverse.
PE_HD void motionPoseAt(const MotionTRS& M, float a, float* m, float* inv) {
    const float b = 1.0f - a;
    float p[3], s[3];
    for (int k = 0; k < 3; ++k) {
        p[k] = M.p0[k] * b + M.p1[k] * a;
        s[k] = M.s0[k] * b + M.s1[k] * a;
    }
    // Quatf::slerp
    const double td = static_cast<double>(a);
    double r[4];
    if (M.linear) {
        for (int k = 0; k < 4; ++k) r[k] = M.qa[k] + (M.qb[k] - M.qa[k]) * td;
    } else {
        const double wa = sin((1.0 - td) * M.theta) / M.sinT;
        const double wb = sin(td * M.theta) / M.sinT;
        for (int k = 0; k < 4; ++k) r[k] = M.qa[k] * wa + M.qb[k] * wb;
    }
    const double len2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3];
    float q[4] = {0.0f, 0.0f, 0.0f, 1.0f};
    if (len2 > 1e-16) {
        const double il = 1.0 / sqrt(len2);
        for (int k = 0; k < 4; ++k) q[k] = static_cast<float>(r[k] * il);
    }
    composeTRS(p, q, s, m);
    mat4Inverse(m, inv);
}

} // namespace pe
