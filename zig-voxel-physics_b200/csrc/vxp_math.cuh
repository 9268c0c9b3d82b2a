// vxp_math.cuh — device (and host) float math of the voxel contact path.
//
// Every function keeps the operation order of the Zig reference so that, with
// the library built by nvcc --fmad=false -prec-div=true -prec-sqrt=true, each
// result is bit-identical to the reference's strict-IEEE f32 arithmetic:
//   src/math.zig:33-176 (Vec3), 258-372 (Quat), 446-507 (Mat3),
//   543-554 (Transform), 673-747 (AABB/OBB vertices), 755-768 (integrateRotation).
// No operator is contracted into an FMA and nothing is reassociated.
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define VXP_HD __host__ __device__ __forceinline__
#else
#define VXP_HD inline
#endif

namespace vxp {

struct F3 {
    float x, y, z;
};
struct I3 {
    int32_t x, y, z;
};
struct Qt {
    float x, y, z, w;
};
struct M33 {
    float m[9];  // row-major
};

constexpr float kEpsilon = 1e-6f;  // math.zig:4

VXP_HD F3 f3(float x, float y, float z) { return F3{x, y, z}; }
VXP_HD F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
VXP_HD F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
VXP_HD F3 operator-(F3 a) { return F3{-a.x, -a.y, -a.z}; }
VXP_HD F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
VXP_HD float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VXP_HD F3 cross3(F3 a, F3 b) {
    return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
VXP_HD float lensq3(F3 a) { return dot3(a, a); }
VXP_HD float len3(F3 a) { return sqrtf(lensq3(a)); }
// Vec3.normalize: zero below EPSILON, else scale by 1/len.
VXP_HD F3 normalize3(F3 a) {
    const float l = len3(a);
    if (l < kEpsilon) return F3{0.f, 0.f, 0.f};
    return a * (1.0f / l);
}
// Vec3.normalizeOrZero.
VXP_HD F3 normalize_or_zero3(F3 a) {
    const float l2 = lensq3(a);
    if (l2 < kEpsilon * kEpsilon) return F3{0.f, 0.f, 0.f};
    return a * (1.0f / sqrtf(l2));
}
VXP_HD F3 min3(F3 a, F3 b) { return F3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
VXP_HD F3 max3(F3 a, F3 b) { return F3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
// std.math.clamp(v, lo, hi) == @max(lo, @min(v, hi)), per component.
VXP_HD float clampf_ref(float v, float lo, float hi) { return fmaxf(lo, fminf(v, hi)); }
VXP_HD F3 clamp3(F3 v, F3 lo, F3 hi) {
    return F3{clampf_ref(v.x, lo.x, hi.x), clampf_ref(v.y, lo.y, hi.y), clampf_ref(v.z, lo.z, hi.z)};
}
VXP_HD bool finite3(F3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// ---- quaternions -----------------------------------------------------------
VXP_HD Qt qmul(Qt s, Qt o) {
    return Qt{s.w * o.x + s.x * o.w + s.y * o.z - s.z * o.y,
              s.w * o.y - s.x * o.z + s.y * o.w + s.z * o.x,
              s.w * o.z + s.x * o.y - s.y * o.x + s.z * o.w,
              s.w * o.w - s.x * o.x - s.y * o.y - s.z * o.z};
}
VXP_HD Qt qconj(Qt q) { return Qt{-q.x, -q.y, -q.z, q.w}; }
VXP_HD Qt qnormalize(Qt q) {
    const float l = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (l < kEpsilon) return Qt{0.f, 0.f, 0.f, 1.f};
    const float inv = 1.0f / l;
    return Qt{q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
// Quat.rotate: renormalises only when |q|^2 is outside [0.99, 1.01].
VXP_HD F3 qrotate(Qt self, F3 v) {
    const float l2 = self.x * self.x + self.y * self.y + self.z * self.z + self.w * self.w;
    const Qt q = (l2 < 0.99f || l2 > 1.01f) ? qnormalize(self) : self;
    const F3 qv = F3{q.x, q.y, q.z};
    const F3 uv = cross3(qv, v);
    const F3 uuv = cross3(qv, uv);
    return (v + uv * (2.0f * q.w)) + uuv * 2.0f;
}
// Rotation by a quaternion already known to pass Quat.rotate's norm test
// unchanged, i.e. the output of qnormalize: skips the recheck.  Only valid when
// the caller computed q = qnormalize(x) and |q|^2 lies in [0.99, 1.01], which
// qnormalize guarantees to within a few ulp.
VXP_HD F3 qrotate_unit(Qt q, F3 v) {
    const F3 qv = F3{q.x, q.y, q.z};
    const F3 uv = cross3(qv, v);
    const F3 uuv = cross3(qv, uv);
    return (v + uv * (2.0f * q.w)) + uuv * 2.0f;
}

// ---- sin / cos (Cody-Waite reduction by pi/2, Taylor series in double) -----
// The solver's only transcendental use is Quat.fromAxisAngle inside
// integrateRotation.  Evaluating the series in double and rounding once gives
// the correctly rounded f32 result except in rare double-rounding cases, and
// the same bits on the host and the device.
VXP_HD double vxp_taylor_sin(double r) {
    const double r2 = r * r;
    double p = 0x1.952c77030ad4ap-49;
    p = -0x1.ae7f3e733b81fp-41 + r2 * p;
    p = 0x1.6124613a86d09p-33 + r2 * p;
    p = -0x1.ae64567f544e4p-26 + r2 * p;
    p = 0x1.71de3a556c734p-19 + r2 * p;
    p = -0x1.a01a01a01a01ap-13 + r2 * p;
    p = 0x1.1111111111111p-7 + r2 * p;
    p = -0x1.5555555555555p-3 + r2 * p;
    return r + (r * r2) * p;
}
VXP_HD double vxp_taylor_cos(double r) {
    const double r2 = r * r;
    double p = 0x1.6827863b97d97p-53;
    p = -0x1.ae7f3e733b81fp-45 + r2 * p;
    p = 0x1.93974a8c07c9dp-37 + r2 * p;
    p = -0x1.1eed8eff8d898p-29 + r2 * p;
    p = 0x1.27e4fb7789f5cp-22 + r2 * p;
    p = -0x1.a01a01a01a01ap-16 + r2 * p;
    p = 0x1.6c16c16c16c17p-10 + r2 * p;
    p = -0x1.5555555555555p-5 + r2 * p;
    p = 0x1.0000000000000p-1 + r2 * p;
    return 1.0 - r2 * p;
}
VXP_HD float vxp_sincos(float xf, int which) {
    const double x = (double)xf;
    if (!(fabs(x) < 1.0e6)) return which == 0 ? (float)sin(x) : (float)cos(x);
    const double k = rint(x * 0x1.45f306dc9c883p-1);
    double r = x - k * 0x1.921fb54400000p+0;
    r = r - k * 0x1.0b4611a600000p-34;
    r = r - k * 0x1.3198a2e037073p-69;
    const int q = ((int)k + which) & 3;
    double v;
    if (q == 0) v = vxp_taylor_sin(r);
    else if (q == 1) v = vxp_taylor_cos(r);
    else if (q == 2) v = -vxp_taylor_sin(r);
    else v = -vxp_taylor_cos(r);
    return (float)v;
}

// Quat.fromAxisAngle (math.zig:230-240).
VXP_HD Qt from_axis_angle(F3 axis, float angle) {
    const float half = angle * 0.5f;
    const float s = vxp_sincos(half, 0);
    const F3 n = normalize3(axis);
    return Qt{n.x * s, n.y * s, n.z * s, vxp_sincos(half, 1)};
}
// math.integrateRotation (math.zig:755-768).
VXP_HD Qt integrate_rotation(Qt rot, F3 w, float dt) {
    const F3 omega = w * dt;
    const float ol = len3(omega);
    if (ol < kEpsilon) return rot;
    const float half = ol * 0.5f;
    const F3 axis = omega * (1.0f / ol);
    const Qt delta = from_axis_angle(axis, half * 2.0f);
    return qnormalize(qmul(delta, rot));
}

// ---- matrices ----------------------------------------------------------------
VXP_HD M33 quat_to_mat3(Qt q) {  // Quat.toMat3
    const float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    const float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    const float yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    const float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    M33 r;
    r.m[0] = 1.0f - (yy + zz); r.m[1] = xy + wz; r.m[2] = xz - wy;
    r.m[3] = xy - wz; r.m[4] = 1.0f - (xx + zz); r.m[5] = yz + wx;
    r.m[6] = xz + wy; r.m[7] = yz - wx; r.m[8] = 1.0f - (xx + yy);
    return r;
}
VXP_HD M33 mat3_mul(const M33& a, const M33& b) {
    M33 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r.m[i * 3 + j] = a.m[i * 3 + 0] * b.m[0 * 3 + j] + a.m[i * 3 + 1] * b.m[1 * 3 + j] +
                             a.m[i * 3 + 2] * b.m[2 * 3 + j];
    return r;
}
VXP_HD M33 mat3_transpose(const M33& a) {
    M33 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i * 3 + j] = a.m[j * 3 + i];
    return r;
}
VXP_HD F3 mat3_mul_vec(const M33& a, F3 v) {
    return F3{a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
              a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z};
}
// R * I_local^-1 * R^T  (VoxelBody.getWorldInvInertia / BodyState.integratePosition)
VXP_HD M33 world_inv_inertia(Qt q, const M33& inv_local) {
    const M33 rm = quat_to_mat3(q);
    return mat3_mul(mat3_mul(rm, inv_local), mat3_transpose(rm));
}
VXP_HD float mat3_det(const M33& s) {
    return s.m[0] * (s.m[4] * s.m[8] - s.m[5] * s.m[7]) - s.m[1] * (s.m[3] * s.m[8] - s.m[5] * s.m[6]) +
           s.m[2] * (s.m[3] * s.m[7] - s.m[4] * s.m[6]);
}
VXP_HD M33 mat3_inverse(const M33& s) {  // Mat3.inverse (math.zig:482-507)
    const float det = mat3_det(s);
    M33 r;
    if (fabsf(det) < kEpsilon) {
        for (int i = 0; i < 9; ++i) r.m[i] = (i % 4 == 0) ? 1.f : 0.f;
        return r;
    }
    const float id = 1.0f / det;
    r.m[0] = (s.m[4] * s.m[8] - s.m[5] * s.m[7]) * id;
    r.m[1] = (s.m[2] * s.m[7] - s.m[1] * s.m[8]) * id;
    r.m[2] = (s.m[1] * s.m[5] - s.m[2] * s.m[4]) * id;
    r.m[3] = (s.m[5] * s.m[6] - s.m[3] * s.m[8]) * id;
    r.m[4] = (s.m[0] * s.m[8] - s.m[2] * s.m[6]) * id;
    r.m[5] = (s.m[2] * s.m[3] - s.m[0] * s.m[5]) * id;
    r.m[6] = (s.m[3] * s.m[7] - s.m[4] * s.m[6]) * id;
    r.m[7] = (s.m[1] * s.m[6] - s.m[0] * s.m[7]) * id;
    r.m[8] = (s.m[0] * s.m[4] - s.m[1] * s.m[3]) * id;
    return r;
}

// ---- transforms --------------------------------------------------------------
// Transform.transformPoint normalises the rotation on every call; callers that
// hold qn = qnormalize(q) pass it here.
VXP_HD F3 transform_point_n(F3 pos, Qt qn, F3 p) { return qrotate(qn, p) + pos; }
VXP_HD F3 transform_point(F3 pos, Qt q, F3 p) { return qrotate(qnormalize(q), p) + pos; }
// Transform.inverseTransformPoint: conjugate().rotate(w - pos), no forced normalise.
VXP_HD F3 inverse_transform_point(F3 pos, Qt q, F3 w) { return qrotate(qconj(q), w - pos); }

// ---- voxel bytes ---------------------------------------------------------------
constexpr uint8_t kEmpty = 0, kCorner = 1, kEdge = 2, kFace = 3, kInside = 4;
VXP_HD uint32_t vtype(uint32_t v) { return v & 7u; }
VXP_HD uint32_t vnormal(uint32_t v) { return v >> 3; }
// shouldCheckCollision (narrow_phase.zig:701-709).
VXP_HD bool type_filter(uint32_t ta, uint32_t tb) {
    if (ta == kEmpty || tb == kEmpty) return false;
    if (ta == kCorner || tb == kCorner) return true;
    return ta == kEdge && tb == kEdge;
}
// @divFloor(v, 8) and @mod(v, 8) on two's complement i32.
VXP_HD int32_t div_floor8(int32_t v) { return v >> 3; }
VXP_HD int32_t mod8(int32_t v) { return v & 7; }

// ContactPoint.computeFeatureId (narrow_phase.zig:384-392).
VXP_HD uint64_t feature_id(I3 a, I3 b) {
    return (uint64_t)((int64_t)a.x & 0xFFFF) | ((uint64_t)((int64_t)a.y & 0xFFFF) << 16) |
           ((uint64_t)((int64_t)a.z & 0xFFFF) << 32) | ((uint64_t)((int64_t)b.x & 0xF) << 48) |
           ((uint64_t)((int64_t)b.y & 0xF) << 52) | ((uint64_t)((int64_t)b.z & 0xF) << 56);
}
VXP_HD uint64_t pair_key(uint32_t a, uint32_t b) {
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ((uint64_t)lo << 32) | (uint64_t)hi;
}

}  // namespace vxp
