// vx_device.cuh — device-side maths shared by the corotational-solve kernels.
//
// 3-vectors, symmetric 3x3 blocks stored as six values (xx, yy, zz, xy, xz, yz),
// full 3x3 matrices as three columns, and quaternions (x, y, z, w). These
// restate the glam operations the reference uses (Mat3::inverse, Quat * Vec3,
// Quat::from_mat3, Quat::slerp at 1/2), see src/solver.rs:27-122 and :327-417.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define VX_EMPTY_U32 0xFFFFFFFFu

namespace vx {

// f32 constants of the reference (src/scene.rs:10-11) and 2*AREA/CELL
// evaluated in f32 (src/solver.rs:72).
constexpr double kCell = 0.0099999997764825820922851562;
constexpr double kArea = 9.99999974737875163555145264e-05;
constexpr double kStiffScale = 0.0199999995529651641845703125;

struct v3 {
    double x, y, z;
};
__device__ __forceinline__ v3 mk(double x, double y, double z) { return v3{x, y, z}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator*(v3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ v3 normalize_or_zero(v3 v) {
    double rcp = 1.0 / sqrt(dot(v, v));
    if (isfinite(rcp) && rcp > 0.0) return v * rcp;
    return {0.0, 0.0, 0.0};
}
__device__ __forceinline__ double get(v3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Column-major 3x3 (c[k] is column k), as glam::Mat3.
struct m3 {
    v3 c[3];
};
__device__ __forceinline__ v3 mul(const m3& m, v3 v) {
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}
__device__ __forceinline__ v3 mul_t(const m3& m, v3 v) {  // m^T v
    return {dot(m.c[0], v), dot(m.c[1], v), dot(m.c[2], v)};
}
__device__ __forceinline__ double det(const m3& m) { return dot(m.c[2], cross(m.c[0], m.c[1])); }
// Rows of the inverse are (y x z, z x x, x x y) / det over the columns x, y, z.
__device__ __forceinline__ m3 inverse(const m3& m) {
    v3 t0 = cross(m.c[1], m.c[2]);
    v3 t1 = cross(m.c[2], m.c[0]);
    v3 t2 = cross(m.c[0], m.c[1]);
    double inv_det = 1.0 / dot(m.c[2], t2);
    m3 r;
    r.c[0] = mk(t0.x, t1.x, t2.x) * inv_det;
    r.c[1] = mk(t0.y, t1.y, t2.y) * inv_det;
    r.c[2] = mk(t0.z, t1.z, t2.z) * inv_det;
    return r;
}
__device__ __forceinline__ m3 transpose(const m3& m) {
    m3 r;
    r.c[0] = mk(m.c[0].x, m.c[1].x, m.c[2].x);
    r.c[1] = mk(m.c[0].y, m.c[1].y, m.c[2].y);
    r.c[2] = mk(m.c[0].z, m.c[1].z, m.c[2].z);
    return r;
}

// Symmetric 3x3: s[0..5] = xx, yy, zz, xy, xz, yz.
struct sym6 {
    double s[6];
};
__device__ __forceinline__ v3 mul(const sym6& a, v3 v) {
    return {a.s[0] * v.x + a.s[3] * v.y + a.s[4] * v.z, a.s[3] * v.x + a.s[1] * v.y + a.s[5] * v.z,
            a.s[4] * v.x + a.s[5] * v.y + a.s[2] * v.z};
}
// Inverse of a symmetric block by its adjugate (exactly symmetric).
__device__ __forceinline__ sym6 inverse(const sym6& a) {
    double xx = a.s[0], yy = a.s[1], zz = a.s[2], xy = a.s[3], xz = a.s[4], yz = a.s[5];
    double c00 = yy * zz - yz * yz;
    double c01 = xz * yz - xy * zz;
    double c02 = xy * yz - xz * yy;
    double c11 = xx * zz - xz * xz;
    double c12 = xy * xz - xx * yz;
    double c22 = xx * yy - xy * xy;
    double d = xx * c00 + xy * c01 + xz * c02;
    double inv = 1.0 / d;
    return sym6{{c00 * inv, c11 * inv, c22 * inv, c01 * inv, c02 * inv, c12 * inv}};
}

struct quat {
    double x, y, z, w;
};
// q * v = v (w^2 - b.b) + b (2 v.b) + (b x v)(2 w), b = (x, y, z).
__device__ __forceinline__ v3 rotate(quat q, v3 v) {
    v3 b = mk(q.x, q.y, q.z);
    double s = q.w * q.w - dot(b, b);
    return v * s + b * (2.0 * dot(v, b)) + cross(b, v) * (2.0 * q.w);
}
__device__ __forceinline__ m3 from_quat(quat q) {
    double x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    double xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    double yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    double wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    m3 m;
    m.c[0] = mk(1.0 - (yy + zz), xy + wz, xz - wy);
    m.c[1] = mk(xy - wz, 1.0 - (xx + zz), yz + wx);
    m.c[2] = mk(xz + wy, yz - wx, 1.0 - (xx + yy));
    return m;
}
__device__ __forceinline__ quat normalize(quat q) {
    double inv = 1.0 / sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
__device__ __forceinline__ double qdot(quat a, quat b) {
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
// slerp(a, b, 1/2) on the short arc = normalize(a + sign(a.b) b).
__device__ __forceinline__ quat slerp_half(quat a, quat b) {
    double s = qdot(a, b) < 0.0 ? -1.0 : 1.0;
    return normalize(quat{a.x + s * b.x, a.y + s * b.y, a.z + s * b.z, a.w + s * b.w});
}
// Rotation matrix (columns) -> quaternion, four-branch method of M. Day (2015).
__device__ __forceinline__ quat from_mat3(const m3& m) {
    double m00 = m.c[0].x, m01 = m.c[0].y, m02 = m.c[0].z;
    double m10 = m.c[1].x, m11 = m.c[1].y, m12 = m.c[1].z;
    double m20 = m.c[2].x, m21 = m.c[2].y, m22 = m.c[2].z;
    if (m22 <= 0.0) {
        double dif10 = m11 - m00, omm22 = 1.0 - m22;
        if (dif10 <= 0.0) {
            double f = omm22 - dif10, inv = 0.5 / sqrt(f);
            return {f * inv, (m01 + m10) * inv, (m02 + m20) * inv, (m12 - m21) * inv};
        }
        double f = omm22 + dif10, inv = 0.5 / sqrt(f);
        return {(m01 + m10) * inv, f * inv, (m12 + m21) * inv, (m20 - m02) * inv};
    }
    double sum10 = m11 + m00, opm22 = 1.0 + m22;
    if (sum10 <= 0.0) {
        double f = opm22 - sum10, inv = 0.5 / sqrt(f);
        return {(m02 + m20) * inv, (m12 + m21) * inv, f * inv, (m01 - m10) * inv};
    }
    double f = opm22 + sum10, inv = 0.5 / sqrt(f);
    return {(m12 - m21) * inv, (m20 - m02) * inv, (m01 - m10) * inv, f * inv};
}
// basis(axis, q), src/solver.rs:27-34.
__device__ __forceinline__ m3 basis(int axis, quat q) {
    m3 f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        int k = (axis + c) % 3;
        v3 e = mk(k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0);
        f.c[c] = rotate(q, e);
    }
    return f;
}

// Warp/block reductions ------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace vx
