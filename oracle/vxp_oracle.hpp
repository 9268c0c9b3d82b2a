// vxp_oracle.hpp — CPU restatement of the reference's per-step hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the CUDA
// library under zig-voxel-physics_b200/csrc and the timed CPU baseline of
// bench.py.  Nothing in the product links it.
//
// It restates, operation for operation, the Zig sources of
// nitanmarcel/zig-voxel-physics (Zig 0.15.2, std only):
//   src/math.zig            Vec3/Quat/Mat3/Transform/AABB/OBB, integrateRotation
//   src/collision_voxel.zig VoxelType, NORMAL_LUT, classification, shouldCollide
//   src/collider.zig        CollisionBrick / VoxelCollider lookups and metadata
//   src/body.zig            BodyMotionState, getWorldInvInertia, updateSleepState,
//                           computeMassProperties
//   src/narrow_phase.zig    SAT, overlap region, detectVoxelCollisions,
//                           checkNeighborhood, generateContact, addContact,
//                           BrickPairCache, ContactManager, processPair
//   src/solver.zig          ContactSolver (TGS soft), BodyState
//   src/islands.zig         GraphColoring.build
//   src/system.zig          step / narrowPhase / solve / updateSleepStates
//
// Zig's default float mode is strict IEEE: no contraction, correctly rounded
// `/` and `@sqrt`.  Build with -ffp-contract=off and without fast-math so every
// expression below rounds exactly like the Zig code (left-to-right evaluation,
// one rounding per operator).
//
// Parity notes (where the reference leaves a result unpinned):
//   * std.AutoHashMap iteration order decides the reference's manifold order
//     (src/system.zig:687-702) and brick iteration order.  Here manifolds are
//     kept in pair order and bricks in the order they were supplied.
//   * @sin/@cos (src/math.zig:230-240) are evaluated by sin_f32/cos_f32 below:
//     a Cody-Waite reduction by pi/2 and Taylor series in double, rounded once
//     to float, i.e. the correctly rounded value except in double-rounding
//     corner cases (probability ~1e-8 per call).
//   * The solver sweeps manifolds colour-major (see ColourMode) so that a
//     parallel sweep over colour batches is the same sequence of operations.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

namespace vxo {

// ---------------------------------------------------------------------------
// sin / cos for f32 (Cody-Waite reduction + Taylor series, in double)
// ---------------------------------------------------------------------------
inline double taylor_sin(double r) {
    const double r2 = r * r;
    double p = 0x1.952c77030ad4ap-49;            // 1/17!
    p = -0x1.ae7f3e733b81fp-41 + r2 * p;         // -1/15!
    p = 0x1.6124613a86d09p-33 + r2 * p;          // 1/13!
    p = -0x1.ae64567f544e4p-26 + r2 * p;         // -1/11!
    p = 0x1.71de3a556c734p-19 + r2 * p;          // 1/9!
    p = -0x1.a01a01a01a01ap-13 + r2 * p;         // -1/7!
    p = 0x1.1111111111111p-7 + r2 * p;           // 1/5!
    p = -0x1.5555555555555p-3 + r2 * p;          // -1/3!
    return r + (r * r2) * p;
}
inline double taylor_cos(double r) {
    const double r2 = r * r;
    double p = 0x1.6827863b97d97p-53;            // 1/18!
    p = -0x1.ae7f3e733b81fp-45 + r2 * p;         // -1/16!
    p = 0x1.93974a8c07c9dp-37 + r2 * p;          // 1/14!
    p = -0x1.1eed8eff8d898p-29 + r2 * p;         // -1/12!
    p = 0x1.27e4fb7789f5cp-22 + r2 * p;          // 1/10!
    p = -0x1.a01a01a01a01ap-16 + r2 * p;         // -1/8!
    p = 0x1.6c16c16c16c17p-10 + r2 * p;          // 1/6!
    p = -0x1.5555555555555p-5 + r2 * p;          // -1/4!
    p = 0x1.0000000000000p-1 + r2 * p;           // -(-1/2!) folded below
    return 1.0 - r2 * p;
}
// Returns sin (which=0) or cos (which=1) of a float argument.
inline float sincos_f32(float xf, int which) {
    const double x = (double)xf;
    if (!(std::fabs(x) < 1.0e6)) {  // huge or non-finite: not on any solver path
        return which == 0 ? (float)std::sin(x) : (float)std::cos(x);
    }
    const double k = std::nearbyint(x * 0x1.45f306dc9c883p-1);  // x * 2/pi
    double r = x - k * 0x1.921fb54400000p+0;
    r = r - k * 0x1.0b4611a600000p-34;
    r = r - k * 0x1.3198a2e037073p-69;
    const int q = ((int)k + which) & 3;
    double v;
    switch (q) {
        case 0: v = taylor_sin(r); break;
        case 1: v = taylor_cos(r); break;
        case 2: v = -taylor_sin(r); break;
        default: v = -taylor_cos(r); break;
    }
    return (float)v;
}

template <class R> inline R vsin(R x);
template <class R> inline R vcos(R x);
template <> inline float vsin<float>(float x) { return sincos_f32(x, 0); }
template <> inline float vcos<float>(float x) { return sincos_f32(x, 1); }
template <> inline double vsin<double>(double x) { return std::sin(x); }
template <> inline double vcos<double>(double x) { return std::cos(x); }

// Zig @min/@max on floats are LLVM minnum/maxnum (== fmin/fmax).
template <class R> inline R fmx(R a, R b) { return std::fmax(a, b); }
template <class R> inline R fmn(R a, R b) { return std::fmin(a, b); }
// std.math.clamp(v, lo, hi) == @max(lo, @min(v, hi))
template <class R> inline R fclamp(R v, R lo, R hi) { return fmx(lo, fmn(v, hi)); }

// ---------------------------------------------------------------------------
// math.zig
// ---------------------------------------------------------------------------
template <class R> struct V3 {
    R x, y, z;
};
struct IV3 {
    int32_t x, y, z;
};
template <class R> struct Q {
    R x, y, z, w;
};
template <class R> struct M3 {
    R m[3][3];
};
template <class R> struct Xf {
    V3<R> p;
    Q<R> q;
};
template <class R> struct Aabb {
    V3<R> mn, mx;
};
template <class R> struct Obb {
    V3<R> c, h;
    Q<R> q;
};

template <class R> constexpr R kEps() { return (R)1e-6f; }  // math.zig:4 (f32 literal)

template <class R> inline V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R> inline V3<R> splat(R s) { return {s, s, s}; }
template <class R> inline V3<R> add(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> scale(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> neg(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R len2(V3<R> a) { return dot(a, a); }
template <class R> inline R len(V3<R> a) { return std::sqrt(len2(a)); }
template <class R> inline V3<R> normalize(V3<R> a) {  // math.zig:101-105
    const R l = len(a);
    if (l < kEps<R>()) return {0, 0, 0};
    return scale(a, (R)1 / l);
}
template <class R> inline V3<R> normalizeOrZero(V3<R> a) {  // math.zig:107-111
    const R l2 = len2(a);
    if (l2 < kEps<R>() * kEps<R>()) return {0, 0, 0};
    return scale(a, (R)1 / std::sqrt(l2));
}
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) { return {fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) { return {fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z)}; }
template <class R> inline V3<R> vclamp(V3<R> v, V3<R> lo, V3<R> hi) {
    return {fclamp(v.x, lo.x, hi.x), fclamp(v.y, lo.y, hi.y), fclamp(v.z, lo.z, hi.z)};
}
template <class R> inline bool finite3(V3<R> v) {
    return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z);
}

template <class R> inline Q<R> qident() { return {0, 0, 0, 1}; }
template <class R> inline Q<R> qmul(Q<R> s, Q<R> o) {  // math.zig:258-265
    return {s.w * o.x + s.x * o.w + s.y * o.z - s.z * o.y,
            s.w * o.y - s.x * o.z + s.y * o.w + s.z * o.x,
            s.w * o.z + s.x * o.y - s.y * o.x + s.z * o.w,
            s.w * o.w - s.x * o.x - s.y * o.y - s.z * o.z};
}
template <class R> inline Q<R> qconj(Q<R> q) { return {-q.x, -q.y, -q.z, q.w}; }
template <class R> inline Q<R> qnormalize(Q<R> q) {  // math.zig:298-308
    const R l = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (l < kEps<R>()) return qident<R>();
    const R inv = (R)1 / l;
    return {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
template <class R> inline V3<R> qrotate(Q<R> self, V3<R> v) {  // math.zig:267-275
    const R l2 = self.x * self.x + self.y * self.y + self.z * self.z + self.w * self.w;
    const Q<R> q = (l2 < (R)0.99f || l2 > (R)1.01f) ? qnormalize(self) : self;
    const V3<R> qv = {q.x, q.y, q.z};
    const V3<R> uv = cross(qv, v);
    const V3<R> uuv = cross(qv, uv);
    return add(add(v, scale(uv, (R)2 * q.w)), scale(uuv, (R)2));
}
template <class R> inline Q<R> fromAxisAngle(V3<R> axis, R angle) {  // math.zig:230-240
    const R half = angle * (R)0.5;
    const R s = vsin<R>(half);
    const V3<R> n = normalize(axis);
    return {n.x * s, n.y * s, n.z * s, vcos<R>(half)};
}
template <class R> inline M3<R> toMat3(Q<R> q) {  // math.zig:350-372
    const R x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    const R xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    const R yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    const R wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    M3<R> r;
    r.m[0][0] = (R)1 - (yy + zz); r.m[0][1] = xy + wz; r.m[0][2] = xz - wy;
    r.m[1][0] = xy - wz; r.m[1][1] = (R)1 - (xx + zz); r.m[1][2] = yz + wx;
    r.m[2][0] = xz + wy; r.m[2][1] = yz - wx; r.m[2][2] = (R)1 - (xx + yy);
    return r;
}
template <class R> inline M3<R> mzero() {
    M3<R> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = 0;
    return r;
}
template <class R> inline M3<R> midentity() {
    M3<R> r = mzero<R>();
    r.m[0][0] = r.m[1][1] = r.m[2][2] = 1;
    return r;
}
template <class R> inline V3<R> mulVec(const M3<R>& a, V3<R> v) {  // math.zig:446-452
    return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
            a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
template <class R> inline M3<R> mmul(const M3<R>& a, const M3<R>& b) {  // math.zig:454-464
    M3<R> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}
template <class R> inline M3<R> mtranspose(const M3<R>& a) {
    M3<R> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}
template <class R> inline R mdet(const M3<R>& s) {  // math.zig:476-480
    return s.m[0][0] * (s.m[1][1] * s.m[2][2] - s.m[1][2] * s.m[2][1]) -
           s.m[0][1] * (s.m[1][0] * s.m[2][2] - s.m[1][2] * s.m[2][0]) +
           s.m[0][2] * (s.m[1][0] * s.m[2][1] - s.m[1][1] * s.m[2][0]);
}
template <class R> inline M3<R> minverse(const M3<R>& s) {  // math.zig:482-507
    const R det = mdet(s);
    if (std::fabs(det) < kEps<R>()) return midentity<R>();
    const R id = (R)1 / det;
    M3<R> r;
    r.m[0][0] = (s.m[1][1] * s.m[2][2] - s.m[1][2] * s.m[2][1]) * id;
    r.m[0][1] = (s.m[0][2] * s.m[2][1] - s.m[0][1] * s.m[2][2]) * id;
    r.m[0][2] = (s.m[0][1] * s.m[1][2] - s.m[0][2] * s.m[1][1]) * id;
    r.m[1][0] = (s.m[1][2] * s.m[2][0] - s.m[1][0] * s.m[2][2]) * id;
    r.m[1][1] = (s.m[0][0] * s.m[2][2] - s.m[0][2] * s.m[2][0]) * id;
    r.m[1][2] = (s.m[0][2] * s.m[1][0] - s.m[0][0] * s.m[1][2]) * id;
    r.m[2][0] = (s.m[1][0] * s.m[2][1] - s.m[1][1] * s.m[2][0]) * id;
    r.m[2][1] = (s.m[0][1] * s.m[2][0] - s.m[0][0] * s.m[2][1]) * id;
    r.m[2][2] = (s.m[0][0] * s.m[1][1] - s.m[0][1] * s.m[1][0]) * id;
    return r;
}
template <class R> inline V3<R> transformPoint(const Xf<R>& t, V3<R> p) {  // math.zig:543-546
    return add(qrotate(qnormalize(t.q), p), t.p);
}
template <class R> inline V3<R> inverseTransformPoint(const Xf<R>& t, V3<R> w) {  // math.zig:552-554
    return qrotate(qconj(t.q), sub(w, t.p));
}
template <class R> inline Aabb<R> aabbEmpty() {
    const R inf = std::numeric_limits<R>::infinity();
    return {{inf, inf, inf}, {-inf, -inf, -inf}};
}
template <class R> inline Aabb<R> aabbMerge(const Aabb<R>& a, const Aabb<R>& b) {
    return {vmin(a.mn, b.mn), vmax(a.mx, b.mx)};
}
template <class R> inline void aabbVerts(const Aabb<R>& a, V3<R> out[8]) {  // math.zig:673-684
    out[0] = {a.mn.x, a.mn.y, a.mn.z};
    out[1] = {a.mx.x, a.mn.y, a.mn.z};
    out[2] = {a.mn.x, a.mx.y, a.mn.z};
    out[3] = {a.mx.x, a.mx.y, a.mn.z};
    out[4] = {a.mn.x, a.mn.y, a.mx.z};
    out[5] = {a.mx.x, a.mn.y, a.mx.z};
    out[6] = {a.mn.x, a.mx.y, a.mx.z};
    out[7] = {a.mx.x, a.mx.y, a.mx.z};
}
template <class R> inline Aabb<R> aabbTransform(const Aabb<R>& a, const Xf<R>& t) {  // math.zig:686-693
    V3<R> c[8];
    aabbVerts(a, c);
    Aabb<R> r = aabbEmpty<R>();
    for (int i = 0; i < 8; ++i) {
        const V3<R> p = transformPoint(t, c[i]);
        r.mn = vmin(r.mn, p);
        r.mx = vmax(r.mx, p);
    }
    return r;
}
template <class R> inline Obb<R> obbFromAabb(const Aabb<R>& a, const Xf<R>& t) {  // math.zig:715-721
    const V3<R> center = scale(add(a.mn, a.mx), (R)0.5);
    const V3<R> ext = scale(sub(a.mx, a.mn), (R)0.5);
    return {transformPoint(t, center), ext, t.q};
}
template <class R> inline void obbAxes(const Obb<R>& o, V3<R> ax[3]) {  // math.zig:723-729
    ax[0] = qrotate(o.q, V3<R>{1, 0, 0});
    ax[1] = qrotate(o.q, V3<R>{0, 1, 0});
    ax[2] = qrotate(o.q, V3<R>{0, 0, 1});
}
template <class R> inline void obbVerts(const Obb<R>& o, V3<R> v[8]) {  // math.zig:731-747
    V3<R> ax[3];
    obbAxes(o, ax);
    const V3<R> ex = scale(ax[0], o.h.x), ey = scale(ax[1], o.h.y), ez = scale(ax[2], o.h.z);
    v[0] = sub(sub(sub(o.c, ex), ey), ez);
    v[1] = sub(sub(add(o.c, ex), ey), ez);
    v[2] = sub(add(sub(o.c, ex), ey), ez);
    v[3] = sub(add(add(o.c, ex), ey), ez);
    v[4] = add(sub(sub(o.c, ex), ey), ez);
    v[5] = add(sub(add(o.c, ex), ey), ez);
    v[6] = add(add(sub(o.c, ex), ey), ez);
    v[7] = add(add(add(o.c, ex), ey), ez);
}
template <class R> inline Q<R> integrateRotation(Q<R> rot, V3<R> w, R dt) {  // math.zig:755-768
    const V3<R> omega = scale(w, dt);
    const R ol = len(omega);
    if (ol < kEps<R>()) return rot;
    const R half = ol * (R)0.5;
    const V3<R> axis = scale(omega, (R)1 / ol);
    const Q<R> delta = fromAxisAngle(axis, half * (R)2);
    return qnormalize(qmul(delta, rot));
}

// ---------------------------------------------------------------------------
// collision_voxel.zig
// ---------------------------------------------------------------------------
enum VType : uint8_t { T_EMPTY = 0, T_CORNER = 1, T_EDGE = 2, T_FACE = 3, T_INSIDE = 4 };

static const int kNormalLut[26][3] = {  // collision_voxel.zig:47-76
    {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},  {0, 0, 1},  {0, 0, -1},  {1, 1, 0},
    {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1},   {1, 0, -1}, {-1, 0, 1},  {-1, 0, -1},
    {0, 1, 1},  {0, 1, -1}, {0, -1, 1},  {0, -1, -1}, {1, 1, 1},  {1, 1, -1},  {1, -1, 1},
    {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};

inline uint8_t vtype(uint8_t v) { return v & 7u; }
inline uint8_t vnormal(uint8_t v) { return v >> 3; }
inline uint8_t make_voxel(uint8_t type, uint8_t normal) { return (uint8_t)((type & 7u) | (normal << 3)); }

template <class R> inline V3<R> getNormalVec3(uint8_t idx) {  // collision_voxel.zig:79-83
    if (idx >= 26) return {0, 0, 0};
    return normalize(V3<R>{(R)kNormalLut[idx][0], (R)kNormalLut[idx][1], (R)kNormalLut[idx][2]});
}
inline uint8_t findClosestNormalIndex(V3<float> d) {  // collision_voxel.zig:86-100
    uint8_t best = 0;
    float best_dot = -std::numeric_limits<float>::infinity();
    for (int i = 0; i < 26; ++i) {
        const float dd = dot(d, getNormalVec3<float>((uint8_t)i));
        if (dd > best_dot) {
            best_dot = dd;
            best = (uint8_t)i;
        }
    }
    return best;
}
inline uint8_t computeNormalIndex(uint8_t empty) {  // collision_voxel.zig:103-130
    if (__builtin_popcount(empty) == 0) return 0;
    int dx = 0, dy = 0, dz = 0;
    if (empty & 1) dx -= 1;
    if (empty & 2) dx += 1;
    if (empty & 4) dy -= 1;
    if (empty & 8) dy += 1;
    if (empty & 16) dz -= 1;
    if (empty & 32) dz += 1;
    for (int i = 0; i < 26; ++i)
        if (kNormalLut[i][0] == dx && kNormalLut[i][1] == dy && kNormalLut[i][2] == dz) return (uint8_t)i;
    return findClosestNormalIndex(V3<float>{(float)dx, (float)dy, (float)dz});
}
inline uint8_t classifyVoxel(bool solid, uint8_t empty) {  // collision_voxel.zig:194-210
    if (!solid) return 0;
    const int c = __builtin_popcount(empty);
    const uint8_t t = c == 0 ? T_INSIDE : c == 1 ? T_FACE : c == 2 ? T_EDGE : T_CORNER;
    return make_voxel(t, computeNormalIndex(empty));
}
inline uint8_t classifyFromNeighbors(bool solid, bool nx, bool px, bool ny, bool py, bool nz, bool pz) {
    if (!solid) return 0;  // collision_voxel.zig:213-235
    uint8_t m = 0;
    if (!nx) m |= 1;
    if (!px) m |= 2;
    if (!ny) m |= 4;
    if (!py) m |= 8;
    if (!nz) m |= 16;
    if (!pz) m |= 32;
    return classifyVoxel(solid, m);
}
inline bool shouldCheckCollision(uint8_t ta, uint8_t tb) {  // narrow_phase.zig:701-709
    if (ta == T_EMPTY || tb == T_EMPTY) return false;
    if (ta == T_CORNER || tb == T_CORNER) return true;
    if (ta == T_EDGE && tb == T_EDGE) return true;
    return false;
}

// ---------------------------------------------------------------------------
// collider.zig
// ---------------------------------------------------------------------------
inline uint64_t hashBrickPos(IV3 p) {  // collider.zig:187-192
    const uint64_t ux = (uint64_t)(int64_t)p.x, uy = (uint64_t)(int64_t)p.y, uz = (uint64_t)(int64_t)p.z;
    return ux ^ (uy * 0x517cc1b727220a95ull) ^ (uz * 0x9e3779b97f4a7c15ull);
}
inline int32_t divFloor8(int32_t v) { return v >= 0 ? v / 8 : -((-v + 7) / 8); }
inline int32_t mod8(int32_t v) { return v - divFloor8(v) * 8; }

struct Brick {
    IV3 pos;
    uint8_t vox[512];
    bool is_empty;
    uint16_t solid_count;
};

template <class R> struct Collider {
    R voxel_size = (R)0.1f;
    std::vector<Brick> bricks;                      // supplied order
    std::unordered_map<uint64_t, int32_t> by_hash;  // hashBrickPos -> brick
    IV3 min_bound{0, 0, 0}, max_bound{0, 0, 0};
    Aabb<R> local_aabb = aabbEmpty<R>();
    uint32_t solid_count = 0;

    uint8_t get(IV3 v) const {  // collider.zig:257-264
        const IV3 bp{divFloor8(v.x), divFloor8(v.y), divFloor8(v.z)};
        auto it = by_hash.find(hashBrickPos(bp));
        if (it == by_hash.end()) return 0;
        const Brick& b = bricks[(size_t)it->second];
        return b.vox[mod8(v.x) + 8 * mod8(v.y) + 64 * mod8(v.z)];
    }
    V3<R> voxelToLocal(IV3 v) const {  // collider.zig:213-220
        const R half = voxel_size * (R)0.5;
        return {(R)v.x * voxel_size + half, (R)v.y * voxel_size + half, (R)v.z * voxel_size + half};
    }
    IV3 localToVoxel(V3<R> p) const {  // collider.zig:223-229
        return {(int32_t)std::floor(p.x / voxel_size), (int32_t)std::floor(p.y / voxel_size),
                (int32_t)std::floor(p.z / voxel_size)};
    }
    bool isValidCoord(IV3 v) const {  // collider.zig:276-280
        return v.x >= min_bound.x && v.x < max_bound.x && v.y >= min_bound.y && v.y < max_bound.y &&
               v.z >= min_bound.z && v.z < max_bound.z;
    }
    // Returns false when two bricks share a hashBrickPos value.
    bool build(R vs, const IV3* pos, const uint8_t* vox, uint32_t n) {
        voxel_size = vs;
        bricks.resize(n);
        by_hash.clear();
        for (uint32_t i = 0; i < n; ++i) {
            bricks[i].pos = pos[i];
            std::memcpy(bricks[i].vox, vox + (size_t)i * 512, 512);
            if (!by_hash.emplace(hashBrickPos(pos[i]), (int32_t)i).second) return false;
        }
        recomputeMetadata();
        return true;
    }
    void recomputeMetadata() {  // collider.zig:283-333 (+ CollisionBrick 90-133)
        min_bound = {INT32_MAX, INT32_MAX, INT32_MAX};
        max_bound = {INT32_MIN, INT32_MIN, INT32_MIN};
        solid_count = 0;
        local_aabb = aabbEmpty<R>();
        for (Brick& b : bricks) {
            b.solid_count = 0;
            const R inf = std::numeric_limits<R>::infinity();
            V3<R> bmn = {inf, inf, inf}, bmx = {-inf, -inf, -inf};
            for (int i = 0; i < 512; ++i) {
                if (vtype(b.vox[i]) == T_EMPTY) continue;
                b.solid_count++;
                const int cx = i % 8, cy = (i / 8) % 8, cz = i / 64;
                const V3<R> lp = scale(V3<R>{(R)b.pos.x * (R)8 + (R)cx, (R)b.pos.y * (R)8 + (R)cy,
                                             (R)b.pos.z * (R)8 + (R)cz},
                                       voxel_size);
                bmn = vmin(bmn, lp);
                bmx = vmax(bmx, add(lp, splat(voxel_size)));
            }
            b.is_empty = b.solid_count == 0;
            if (b.is_empty) continue;
            solid_count += b.solid_count;
            for (int i = 0; i < 512; ++i) {
                if (vtype(b.vox[i]) == T_EMPTY) continue;
                const int32_t vx = b.pos.x * 8 + i % 8, vy = b.pos.y * 8 + (i / 8) % 8, vz = b.pos.z * 8 + i / 64;
                min_bound = {std::min(min_bound.x, vx), std::min(min_bound.y, vy), std::min(min_bound.z, vz)};
                max_bound = {std::max(max_bound.x, vx + 1), std::max(max_bound.y, vy + 1),
                             std::max(max_bound.z, vz + 1)};
            }
            local_aabb = aabbMerge(local_aabb, Aabb<R>{bmn, bmx});
        }
        if (solid_count == 0) {
            min_bound = {0, 0, 0};
            max_bound = {0, 0, 0};
        }
    }
    // setCollisionVoxel (collider.zig:267-273): getOrCreateBrick (232-239)
    // appends a zeroed brick when no brick has the position's hash.
    void set(IV3 v, uint8_t val) {
        const IV3 bp{divFloor8(v.x), divFloor8(v.y), divFloor8(v.z)};
        const uint64_t hb = hashBrickPos(bp);
        auto it = by_hash.find(hb);
        int32_t bi;
        if (it == by_hash.end()) {
            Brick b{};
            b.pos = bp;
            std::memset(b.vox, 0, sizeof(b.vox));
            bi = (int32_t)bricks.size();
            bricks.push_back(b);
            by_hash.emplace(hb, bi);
        } else {
            bi = it->second;
        }
        bricks[(size_t)bi].vox[mod8(v.x) + 8 * mod8(v.y) + 64 * mod8(v.z)] = val;
    }
    // An edit batch as a host caller writes it with the reference's calls.
    // mode 0: setCollisionVoxel(coords[i], values[i]) in list order.
    // mode 1: each voxel in list order becomes solid (values[i] != 0; an empty
    // voxel gets an inside byte, a solid one keeps its byte) or empty; then
    // every listed voxel and each of its six face neighbours that is solid is
    // set to classifyFromNeighbors (collision_voxel.zig:213-235) of the face
    // neighbours' occupancy.  Then recomputeMetadata.
    void edit(const int32_t* coords, const uint8_t* values, uint32_t n, int mode) {
        for (uint32_t i = 0; i < n; ++i) {
            const IV3 v{coords[i * 3], coords[i * 3 + 1], coords[i * 3 + 2]};
            if (mode == 0) set(v, values[i]);
            else if (!values[i]) set(v, 0);
            else set(v, vtype(get(v)) == T_EMPTY ? (uint8_t)T_INSIDE : get(v));
        }
        if (mode == 1) {
            const int32_t off[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
            auto solid = [&](IV3 u) { return vtype(get(u)) != T_EMPTY; };
            for (uint32_t i = 0; i < n; ++i)
                for (int k = 0; k < 7; ++k) {
                    const IV3 u{coords[i * 3] + off[k][0], coords[i * 3 + 1] + off[k][1], coords[i * 3 + 2] + off[k][2]};
                    if (!solid(u)) continue;
                    set(u, classifyFromNeighbors(true, solid({u.x - 1, u.y, u.z}), solid({u.x + 1, u.y, u.z}),
                                                 solid({u.x, u.y - 1, u.z}), solid({u.x, u.y + 1, u.z}),
                                                 solid({u.x, u.y, u.z - 1}), solid({u.x, u.y, u.z + 1})));
                }
        }
        recomputeMetadata();
    }
    V3<R> getCenterOfMass() const {  // collider.zig:376-403
        if (solid_count == 0) return {0, 0, 0};
        V3<R> sum = {0, 0, 0};
        uint32_t count = 0;
        for (const Brick& b : bricks) {
            if (b.is_empty) continue;
            for (int i = 0; i < 512; ++i) {
                if (vtype(b.vox[i]) == T_EMPTY) continue;
                const IV3 vp{b.pos.x * 8 + i % 8, b.pos.y * 8 + (i / 8) % 8, b.pos.z * 8 + i / 64};
                sum = add(sum, add(voxelToLocal(vp), splat(voxel_size * (R)0.5)));
                count++;
            }
        }
        return scale(sum, (R)1 / (R)count);
    }
};

// body.zig:462-519, bricks in supplied order.
template <class R> inline void computeMassProperties(const Collider<R>& c, R density, R* inv_mass, M3<R>* inv_inertia) {
    if (c.solid_count == 0) {
        *inv_mass = 0;
        *inv_inertia = mzero<R>();
        return;
    }
    const R vv = c.voxel_size * c.voxel_size * c.voxel_size;
    const R vm = vv * density;
    const R total = vm * (R)c.solid_count;
    const V3<R> com = c.getCenterOfMass();
    M3<R> I = mzero<R>();
    for (const Brick& b : c.bricks) {
        if (b.is_empty) continue;
        for (int i = 0; i < 512; ++i) {
            if (vtype(b.vox[i]) == T_EMPTY) continue;
            const IV3 vp{b.pos.x * 8 + i % 8, b.pos.y * 8 + (i / 8) % 8, b.pos.z * 8 + i / 64};
            const V3<R> pos = add(c.voxelToLocal(vp), splat(c.voxel_size * (R)0.5));
            const V3<R> r = sub(pos, com);
            const R r2 = dot(r, r);
            I.m[0][0] += vm * (r2 - r.x * r.x);
            I.m[1][1] += vm * (r2 - r.y * r.y);
            I.m[2][2] += vm * (r2 - r.z * r.z);
            I.m[0][1] -= vm * r.x * r.y;
            I.m[0][2] -= vm * r.x * r.z;
            I.m[1][2] -= vm * r.y * r.z;
        }
    }
    I.m[1][0] = I.m[0][1];
    I.m[2][0] = I.m[0][2];
    I.m[2][1] = I.m[1][2];
    *inv_mass = (R)1 / total;
    *inv_inertia = minverse(I);
}

// ---------------------------------------------------------------------------
// body.zig
// ---------------------------------------------------------------------------
enum BodyType : uint32_t { B_STATIC = 0, B_KINEMATIC = 1, B_DYNAMIC = 2 };

template <class R> struct Body {
    uint32_t id = 0;
    uint32_t type = B_DYNAMIC;
    int32_t collider = -1;
    bool sleeping = false;
    V3<R> pos{0, 0, 0};
    Q<R> rot{0, 0, 0, 1};
    V3<R> v{0, 0, 0}, w{0, 0, 0};
    R inv_mass = 1;
    M3<R> inv_I_local = midentity<R>();
    R friction = (R)0.5f, restitution = 0, lin_damp = (R)0.3f, ang_damp = (R)0.5f;
    R sleep_timer = 0;

    Xf<R> xf() const { return {pos, rot}; }
    M3<R> worldInvInertia() const {  // body.zig:386-392
        if (inv_mass == 0) return mzero<R>();
        const M3<R> rm = toMat3(rot);
        return mmul(mmul(rm, inv_I_local), mtranspose(rm));
    }
    void updateSleepState(R dt) {  // body.zig:415-427 (+ isNearlyAtRest 94-99, sleep 407-412)
        if (type != B_DYNAMIC) return;
        if (sleeping) return;
        if (len(v) < (R)0.1f && len(w) < (R)0.1f) {
            sleep_timer += dt;
            if (sleep_timer >= (R)0.5f) {
                sleeping = true;
                v = {0, 0, 0};
                w = {0, 0, 0};
            }
        } else {
            sleep_timer = 0;
        }
    }
};

// ---------------------------------------------------------------------------
// narrow_phase.zig
// ---------------------------------------------------------------------------
template <class R> struct Contact {  // narrow_phase.zig:336-393
    V3<R> point{0, 0, 0}, normal{0, 0, 0};
    R penetration = 0;
    V3<R> la{0, 0, 0}, lb{0, 0, 0};
    R normal_impulse = 0;
    R tangent_impulse[2] = {0, 0};
    R normal_mass = 0;
    R tangent_mass[2] = {0, 0};
    uint64_t feature_id = 0;
};

inline uint64_t computeFeatureId(IV3 a, IV3 b) {  // narrow_phase.zig:384-392
    const uint64_t ax = (uint64_t)((int64_t)a.x & 0xFFFF);
    const uint64_t ay = (uint64_t)(((int64_t)a.y & 0xFFFF) << 16);
    const uint64_t az = (uint64_t)(((int64_t)a.z & 0xFFFF) << 32);
    const uint64_t bx = (uint64_t)(((int64_t)b.x & 0xF) << 48);
    const uint64_t by = (uint64_t)(((int64_t)b.y & 0xF) << 52);
    const uint64_t bz = (uint64_t)(((int64_t)b.z & 0xF) << 56);
    return ax | ay | az | bx | by | bz;
}

template <class R> struct Manifold {  // narrow_phase.zig:416-502
    uint32_t a = 0, b = 0;
    Contact<R> c[4];
    uint32_t n = 0;
    R friction = (R)0.5f, restitution = 0;

    void addContact(const Contact<R>& k) {  // narrow_phase.zig:451-481
        for (uint32_t i = 0; i < n; ++i) {
            if (c[i].feature_id == k.feature_id) {
                const R ni = c[i].normal_impulse, t0 = c[i].tangent_impulse[0], t1 = c[i].tangent_impulse[1];
                c[i] = k;
                c[i].normal_impulse = ni;
                c[i].tangent_impulse[0] = t0;
                c[i].tangent_impulse[1] = t1;
                return;
            }
        }
        if (n < 4) {
            c[n++] = k;
            return;
        }
        R mp = k.penetration;
        int mi = -1;
        for (uint32_t i = 0; i < n; ++i) {
            if (c[i].penetration < mp) {
                mp = c[i].penetration;
                mi = (int)i;
            }
        }
        if (mi >= 0) c[mi] = k;
    }
};

inline uint64_t pairKey(uint32_t a, uint32_t b) {  // narrow_phase.zig:973-977
    const uint32_t lo = std::min(a, b), hi = std::max(a, b);
    return ((uint64_t)lo << 32) | (uint64_t)hi;
}

template <class R> inline void projectObb(const Obb<R>& o, V3<R> axis, R* mn, R* mx) {  // narrow_phase.zig:505-517
    V3<R> v[8];
    obbVerts(o, v);
    R lo = std::numeric_limits<R>::infinity(), hi = -std::numeric_limits<R>::infinity();
    for (int i = 0; i < 8; ++i) {
        const R p = dot(v[i], axis);
        lo = fmn(lo, p);
        hi = fmx(hi, p);
    }
    *mn = lo;
    *mx = hi;
}
template <class R> inline bool overlap1(R amn, R amx, R bmn, R bmx) { return !(amx < bmn || bmx < amn); }

template <class R> inline bool satEarlyOut(const Obb<R>& a, const Obb<R>& b) {  // narrow_phase.zig:532-569
    V3<R> aa[3], ab[3];
    obbAxes(a, aa);
    obbAxes(b, ab);
    R p0, p1, q0, q1;
    for (int i = 0; i < 3; ++i) {
        projectObb(a, aa[i], &p0, &p1);
        projectObb(b, aa[i], &q0, &q1);
        if (!overlap1(p0, p1, q0, q1)) return true;
    }
    for (int i = 0; i < 3; ++i) {
        projectObb(a, ab[i], &p0, &p1);
        projectObb(b, ab[i], &q0, &q1);
        if (!overlap1(p0, p1, q0, q1)) return true;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const V3<R> cr = cross(aa[i], ab[j]);
            const R l = len(cr);
            if (l < (R)0.001f) continue;
            const V3<R> ax = scale(cr, (R)1 / l);
            projectObb(a, ax, &p0, &p1);
            projectObb(b, ax, &q0, &q1);
            if (!overlap1(p0, p1, q0, q1)) return true;
        }
    return false;
}

// narrow_phase.zig:572-623 (test-only in the reference; kept for its known-answer tests)
template <class R> inline bool satWithPenetration(const Obb<R>& a, const Obb<R>& b, V3<R>* axis_out, R* depth) {
    R min_ov = std::numeric_limits<R>::infinity();
    V3<R> min_ax = {1, 0, 0};
    V3<R> aa[3], ab[3];
    obbAxes(a, aa);
    obbAxes(b, ab);
    auto test = [&](V3<R> axis) -> bool {
        const R l = len(axis);
        if (l < (R)0.001f) return true;
        const V3<R> n = scale(axis, (R)1 / l);
        R p0, p1, q0, q1;
        projectObb(a, n, &p0, &p1);
        projectObb(b, n, &q0, &q1);
        if (!overlap1(p0, p1, q0, q1)) return false;
        R ov;
        if (p1 < q0) ov = p1 - q0;
        else if (q1 < p0) ov = q1 - p0;
        else ov = fmn(p1 - q0, q1 - p0);
        if (ov < min_ov) {
            min_ov = ov;
            min_ax = dot(sub(b.c, a.c), n) < 0 ? neg(n) : n;
        }
        return true;
    };
    for (int i = 0; i < 3; ++i)
        if (!test(aa[i])) return false;
    for (int i = 0; i < 3; ++i)
        if (!test(ab[i])) return false;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (!test(cross(aa[i], ab[j]))) return false;
    *axis_out = min_ax;
    *depth = min_ov;
    return true;
}

struct Region {
    IV3 mn, mx;
    bool valid;
};

template <class R>
inline Region getOverlapRegion(const Xf<R>& ta, const Collider<R>& ca, const Xf<R>& tb, const Collider<R>& cb) {
    // narrow_phase.zig:644-698
    const Obb<R> ob = obbFromAabb(cb.local_aabb, tb);
    V3<R> vb[8];
    obbVerts(ob, vb);
    const Q<R> inv = qconj(ta.q);
    const R inf = std::numeric_limits<R>::infinity();
    V3<R> tmn = {inf, inf, inf}, tmx = {-inf, -inf, -inf};
    for (int i = 0; i < 8; ++i) {
        const V3<R> rel = qrotate(inv, sub(vb[i], ta.p));
        tmn = vmin(tmn, rel);
        tmx = vmax(tmx, rel);
    }
    const R vs = ca.voxel_size;
    tmn = sub(tmn, splat(vs));
    tmx = add(tmx, splat(vs));
    const V3<R> mnc = vclamp(tmn, ca.local_aabb.mn, ca.local_aabb.mx);
    const V3<R> mxc = vclamp(tmx, ca.local_aabb.mn, ca.local_aabb.mx);
    if (mnc.x >= mxc.x || mnc.y >= mxc.y || mnc.z >= mxc.z) return {{0, 0, 0}, {0, 0, 0}, false};
    const IV3 a = ca.localToVoxel(mnc), b = ca.localToVoxel(mxc);
    return {{std::max(a.x, ca.min_bound.x), std::max(a.y, ca.min_bound.y), std::max(a.z, ca.min_bound.z)},
            {std::min(b.x, ca.max_bound.x), std::min(b.y, ca.max_bound.y), std::min(b.z, ca.max_bound.z)},
            true};
}

// One voxel pair that passed the type filter (debug dump).
struct CandRec {
    uint32_t pair_index;
    IV3 a, b;
    uint32_t passed;
    float dist_sq;
};

template <class R>
inline Contact<R> generateContact(uint8_t va, IV3 ca, V3<R> wa, const Xf<R>& ta, uint8_t vb, IV3 cb, V3<R> wb,
                                  const Xf<R>& tb, V3<R> diff, R dist_sq, R vs) {  // narrow_phase.zig:860-922
    const R dist = std::sqrt(dist_sq);
    const V3<R> cp = scale(add(wa, wb), (R)0.5);
    R pen = vs - dist;
    V3<R> normal;
    const V3<R> na = qrotate(ta.q, getNormalVec3<R>(vnormal(va)));
    const V3<R> nb = qrotate(tb.q, getNormalVec3<R>(vnormal(vb)));
    if (vtype(va) == T_FACE) {
        normal = na;
    } else if (vtype(vb) == T_FACE) {
        normal = neg(nb);
    } else if (dist > (R)0.001f) {
        const V3<R> dn = scale(diff, (R)1 / dist);
        if (dot(dn, na) > (R)0.3f) normal = na;
        else if (dot(dn, neg(nb)) > (R)0.3f) normal = neg(nb);
        else normal = dn;
    } else {
        normal = na;
    }
    if (vtype(va) == T_INSIDE || vtype(vb) == T_INSIDE) pen = fmx(pen, vs);
    Contact<R> k;
    k.point = cp;
    k.normal = normal;
    k.penetration = pen;
    k.la = inverseTransformPoint(ta, cp);
    k.lb = inverseTransformPoint(tb, cp);
    k.feature_id = computeFeatureId(ca, cb);
    return k;
}

template <class R> struct DetectResult {
    Manifold<R> m;
    uint32_t voxels_checked = 0;
    bool has_collision = false;
    uint32_t candidates = 0;
};

// detectVoxelCollisions + checkNeighborhood (narrow_phase.zig:722-857).
template <class R>
inline DetectResult<R> detectVoxelCollisions(const Body<R>& ba, const Collider<R>& ca, const Body<R>& bb,
                                             const Collider<R>& cb, std::vector<CandRec>* dump, uint32_t pidx) {
    DetectResult<R> res;
    const Xf<R> ta = ba.xf(), tb = bb.xf();
    res.m.a = ba.id;
    res.m.b = bb.id;
    res.m.friction = std::sqrt(ba.friction * bb.friction);
    res.m.restitution = fmx(ba.restitution, bb.restitution);
    const Region reg = getOverlapRegion(ta, ca, tb, cb);
    if (!reg.valid) return res;
    const R vs = ca.voxel_size;
    const R cds = vs * vs * (R)1.0f * (R)1.0f;
    const R margin = (R)0.02f;
    const R spec = cds + margin * margin + (R)2 * std::sqrt(cds) * margin;
    for (int32_t z = reg.mn.z; z <= reg.mx.z; ++z)
        for (int32_t y = reg.mn.y; y <= reg.mx.y; ++y)
            for (int32_t x = reg.mn.x; x <= reg.mx.x; ++x) {
                const IV3 ia{x, y, z};
                const uint8_t va = ca.get(ia);
                if (vtype(va) == T_EMPTY) continue;
                const V3<R> wa = transformPoint(ta, ca.voxelToLocal(ia));
                const IV3 cbv = cb.localToVoxel(inverseTransformPoint(tb, wa));
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            const IV3 ib{cbv.x + dx, cbv.y + dy, cbv.z + dz};
                            if (!cb.isValidCoord(ib)) continue;
                            const uint8_t vb = cb.get(ib);
                            if (vtype(vb) == T_EMPTY) continue;
                            res.voxels_checked++;
                            if (!shouldCheckCollision(vtype(va), vtype(vb))) continue;
                            const V3<R> wb = transformPoint(tb, cb.voxelToLocal(ib));
                            const V3<R> diff = sub(wb, wa);
                            const R d2 = len2(diff);
                            const bool pass = d2 < spec;
                            if (dump) dump->push_back({pidx, ia, ib, pass ? 1u : 0u, (float)d2});
                            if (pass) {
                                res.candidates++;
                                res.m.addContact(generateContact(va, ia, wa, ta, vb, ib, wb, tb, diff, d2, vs));
                            }
                        }
            }
    res.has_collision = res.m.n > 0;
    return res;
}

// Brick-pair cache (narrow_phase.zig:65-333).
struct CacheKey {
    uint32_t a, b;
    IV3 ba, bb;
    uint64_t th;
    bool operator==(const CacheKey& o) const {
        return a == o.a && b == o.b && ba.x == o.ba.x && ba.y == o.ba.y && ba.z == o.ba.z && bb.x == o.bb.x &&
               bb.y == o.bb.y && bb.z == o.bb.z && th == o.th;
    }
    uint64_t hash() const {  // narrow_phase.zig:118-131
        uint64_t h = 0;
        h = h * 31 + (uint64_t)a;
        h = h * 31 + (uint64_t)b;
        h = h * 31 + (uint64_t)(uint32_t)ba.x;
        h = h * 31 + (uint64_t)(uint32_t)ba.y;
        h = h * 31 + (uint64_t)(uint32_t)ba.z;
        h = h * 31 + (uint64_t)(uint32_t)bb.x;
        h = h * 31 + (uint64_t)(uint32_t)bb.y;
        h = h * 31 + (uint64_t)(uint32_t)bb.z;
        h = h * 31 + th;
        return h;
    }
};
inline uint64_t computeTransformHash(V3<float> rp, Q<float> rr) {  // narrow_phase.zig:148-169
    const int32_t qx = (int32_t)(rp.x * 100.0f), qy = (int32_t)(rp.y * 100.0f), qz = (int32_t)(rp.z * 100.0f);
    const int16_t rw = (int16_t)fclamp(rr.w * 1000.0f, -32767.0f, 32767.0f);
    const int16_t rx = (int16_t)fclamp(rr.x * 1000.0f, -32767.0f, 32767.0f);
    const int16_t ry = (int16_t)fclamp(rr.y * 1000.0f, -32767.0f, 32767.0f);
    const int16_t rz = (int16_t)fclamp(rr.z * 1000.0f, -32767.0f, 32767.0f);
    uint64_t h = 0;
    h = h * 31 + (uint64_t)(uint32_t)qx;
    h = h * 31 + (uint64_t)(uint32_t)qy;
    h = h * 31 + (uint64_t)(uint32_t)qz;
    h = h * 31 + (uint64_t)(uint16_t)rw;
    h = h * 31 + (uint64_t)(uint16_t)rx;
    h = h * 31 + (uint64_t)(uint16_t)ry;
    h = h * 31 + (uint64_t)(uint16_t)rz;
    return h;
}
inline CacheKey makeCacheKey(uint32_t a, uint32_t b, IV3 ba, IV3 bb, V3<float> rp, Q<float> rr) {
    const bool af = a < b;  // narrow_phase.zig:99-115
    return {af ? a : b, af ? b : a, af ? ba : bb, af ? bb : ba, computeTransformHash(rp, rr)};
}

template <class R> struct CacheValue {
    Contact<R> c[4];
    uint8_t n = 0;
    bool has_collision = false;
    uint32_t voxels_checked = 0;
};

template <class R> struct BrickPairCache {
    struct Entry {
        CacheKey key;
        CacheValue<R> value;
        uint64_t last_used = 0;
        bool valid = false;
    };
    std::vector<Entry> e;
    uint64_t frame = 0;
    uint64_t hits = 0, misses = 0, evictions = 0, invalidations = 0;

    explicit BrickPairCache(size_t cap = 1024) : e(cap) {}
    void beginFrame() { frame++; }
    const CacheValue<R>* get(const CacheKey& k) {  // narrow_phase.zig:228-253
        const size_t cap = e.size();
        size_t idx = (size_t)(k.hash() % cap);
        const size_t maxp = std::min<size_t>(cap, 16);
        for (size_t p = 0; p < maxp; ++p) {
            Entry& en = e[idx];
            if (!en.valid) {
                misses++;
                return nullptr;
            }
            if (en.key == k) {
                en.last_used = frame;
                hits++;
                return &en.value;
            }
            idx = (idx + 1) % cap;
        }
        misses++;
        return nullptr;
    }
    void put(const CacheKey& k, const CacheValue<R>& v) {  // narrow_phase.zig:256-302
        const size_t cap = e.size();
        const size_t start = (size_t)(k.hash() % cap);
        size_t idx = start;
        const size_t maxp = std::min<size_t>(cap, 16);
        size_t oldest = start;
        uint64_t oldest_frame = UINT64_MAX;
        for (size_t p = 0; p < maxp; ++p) {
            Entry& en = e[idx];
            if (!en.valid) {
                en = Entry{k, v, frame, true};
                return;
            }
            if (en.key == k) {
                en.value = v;
                en.last_used = frame;
                return;
            }
            if (en.last_used < oldest_frame) {
                oldest_frame = en.last_used;
                oldest = idx;
            }
            idx = (idx + 1) % cap;
        }
        evictions++;
        e[oldest] = Entry{k, v, frame, true};
    }
    void invalidateBody(uint32_t id) {  // narrow_phase.zig:305-312
        for (Entry& en : e)
            if (en.valid && (en.key.a == id || en.key.b == id)) {
                en.valid = false;
                invalidations++;
            }
    }
};

// ContactManager (narrow_phase.zig:980-1069); manifolds kept in insertion order.
template <class R> struct ContactManager {
    std::vector<Manifold<R>> cur, prev;
    std::unordered_map<uint64_t, size_t> cur_idx, prev_idx;

    void beginFrame() {  // narrow_phase.zig:1003-1008
        std::swap(cur, prev);
        std::swap(cur_idx, prev_idx);
        cur.clear();
        cur_idx.clear();
    }
    const Manifold<R>* prevGet(uint64_t key) const {
        auto it = prev_idx.find(key);
        return it == prev_idx.end() ? nullptr : &prev[it->second];
    }
    void put(uint64_t key, const Manifold<R>& m) {
        auto it = cur_idx.find(key);
        if (it != cur_idx.end()) {
            cur[it->second] = m;
            return;
        }
        cur_idx.emplace(key, cur.size());
        cur.push_back(m);
    }
    Manifold<R>* getMut(uint32_t a, uint32_t b) {
        auto it = cur_idx.find(pairKey(a, b));
        return it == cur_idx.end() ? nullptr : &cur[it->second];
    }
    void addManifold(const Manifold<R>& m) {  // narrow_phase.zig:1011-1021, 1049-1059
        const uint64_t key = pairKey(m.a, m.b);
        const Manifold<R>* p = prevGet(key);
        if (p) {
            Manifold<R> nm = m;
            for (uint32_t i = 0; i < nm.n; ++i)
                for (uint32_t j = 0; j < p->n; ++j)
                    if (nm.c[i].feature_id == p->c[j].feature_id) {
                        nm.c[i].normal_impulse = p->c[j].normal_impulse;
                        nm.c[i].tangent_impulse[0] = p->c[j].tangent_impulse[0];
                        nm.c[i].tangent_impulse[1] = p->c[j].tangent_impulse[1];
                        break;
                    }
            put(key, nm);
        } else {
            put(key, m);
        }
    }
};

// ---------------------------------------------------------------------------
// solver.zig
// ---------------------------------------------------------------------------
template <class R> struct SolverConfig {  // solver.zig:75-119
    uint32_t substeps = 4, velocity_iterations = 1, position_iterations = 2;
    bool disable_rotation = false;
    R hertz = (R)30.0f, damping_ratio = (R)1.0f, position_correction_rate = (R)0.2f,
      max_position_correction = (R)0.04f, slop = (R)0.005f;
    bool warm_starting = true;
    R warm_start_scale = (R)0.8f;
    V3<R> gravity = {0, (R)-9.81f, 0};
    bool enable_friction = true, enable_restitution = true;
};

template <class R> struct SoftParams {
    R bias_rate, mass_coeff, impulse_coeff;
};
template <class R> inline SoftParams<R> computeSoftParams(R hertz, R zeta, R h) {  // solver.zig:57-72
    if (hertz <= 0) return {0, 1, 1};
    const R pi = (R)3.14159274101257324f;  // std.math.pi as f32
    const R omega = (R)2 * pi * hertz;
    const R a1 = (R)2 * zeta + omega * h;
    const R a2 = h * omega * a1;
    const R a3 = (R)1 / ((R)1 + a2);
    return {omega / a1, a2 * a3, a3};
}
template <class R> inline V3<R> computeOrthogonal(V3<R> v) {  // solver.zig:967-981
    if (std::fabs(v.x) < std::fabs(v.y)) {
        if (std::fabs(v.x) < std::fabs(v.z)) return normalizeOrZero(V3<R>{0, -v.z, v.y});
        return normalizeOrZero(V3<R>{-v.y, v.x, 0});
    }
    if (std::fabs(v.y) < std::fabs(v.z)) return normalizeOrZero(V3<R>{-v.z, 0, v.x});
    return normalizeOrZero(V3<R>{-v.y, v.x, 0});
}
template <class R> inline Q<R> integrateRotationSmall(Q<R> r, V3<R> d) {  // solver.zig:984-1005
    const Q<R> h = {d.x * (R)0.5, d.y * (R)0.5, d.z * (R)0.5, 0};
    const Q<R> dq = {h.w * r.x + h.x * r.w + h.y * r.z - h.z * r.y, h.w * r.y - h.x * r.z + h.y * r.w + h.z * r.x,
                     h.w * r.z + h.x * r.y - h.y * r.x + h.z * r.w, h.w * r.w - h.x * r.x - h.y * r.y - h.z * r.z};
    return qnormalize(Q<R>{r.x + dq.x, r.y + dq.y, r.z + dq.z, r.w + dq.w});
}

template <class R> struct BodyState {  // solver.zig:203-357
    V3<R> p;
    Q<R> q;
    V3<R> v, w;
    R inv_mass;
    M3<R> iiw;
    uint32_t type;
    bool sleeping;
    Body<R>* body;

    bool writable() const { return type == B_DYNAMIC && !sleeping; }
    V3<R> pointVel(V3<R> wp) const { return add(v, cross(w, sub(wp, p))); }
    void applyImpulseAtPoint(V3<R> imp, V3<R> r) {  // solver.zig:327-332
        if (type != B_DYNAMIC || sleeping) return;
        v = add(v, scale(imp, inv_mass));
        w = add(w, mulVec(iiw, cross(r, imp)));
    }
    void integratePosition(R dt, bool disable_rot) {  // solver.zig:341-356
        if (type == B_STATIC) return;
        if (sleeping) return;
        p = add(p, scale(v, dt));
        if (!disable_rot) q = integrateRotation(q, w, dt);
        if (type == B_DYNAMIC) {
            const M3<R> rm = toMat3(q);
            iiw = mmul(mmul(rm, body->inv_I_local), mtranspose(rm));
        }
    }
    void writeBack() {  // solver.zig:246-296
        if (type == B_STATIC) return;
        const bool qf = std::isfinite(q.x) && std::isfinite(q.y) && std::isfinite(q.z) && std::isfinite(q.w);
        if (!finite3(p) || !qf) {
            p = finite3(body->pos) ? body->pos : V3<R>{0, 2, 0};
            q = qident<R>();
            v = {0, 0, 0};
            w = {0, 0, 0};
        }
        if (!finite3(v)) v = {0, 0, 0};
        if (!finite3(w)) w = {0, 0, 0};
        const R ls2 = len2(v), as2 = len2(w);
        if (ls2 > (R)50 * (R)50) v = scale(v, (R)50 / std::sqrt(ls2));
        if (as2 > (R)30 * (R)30) w = scale(w, (R)30 / std::sqrt(as2));
        if (ls2 < (R)0.002f) v = {0, 0, 0};
        if (as2 < (R)0.002f) w = {0, 0, 0};
        q = qnormalize(q);
        body->pos = p;
        body->rot = q;
        body->v = v;
        body->w = w;
    }
};

template <class R> struct CPoint {  // solver.zig:122-168
    V3<R> point, normal, la, lb, ra, rb;
    R base_sep, normal_mass, tangent_mass[2];
    V3<R> t1, t2;
    R bias, ni, ti[2], init_vn, penetration;
};
template <class R> struct CManifold {  // solver.zig:171-200
    uint32_t ia, ib;
    R friction, restitution;
    uint32_t n;
    CPoint<R> pt[8];
    uint32_t colour = 0;
    uint32_t order = 0;  // position in the constraint list (addManifold order)
};

// Colour assignment modes for the sweep order.
enum ColourMode : uint32_t { COLOUR_PROJECT = 0, COLOUR_REFERENCE = 1, COLOUR_NONE = 2 };

// Priority used by the project colouring (Jones-Plassmann); higher first.
inline uint32_t jpPriority(uint32_t k) {
    uint32_t h = k * 0x9E3779B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
inline bool jpBefore(uint32_t i, uint32_t j) {  // true if i is coloured before j
    const uint32_t pi = jpPriority(i), pj = jpPriority(j);
    return pi != pj ? pi > pj : i < j;
}

template <class R> struct ContactSolver {
    SolverConfig<R> cfg;
    std::vector<BodyState<R>> bodies;
    std::unordered_map<uint32_t, uint32_t> id2idx;
    std::vector<CManifold<R>> cons;
    ContactManager<R>* manager = nullptr;
    uint32_t position_iterations_run = 0;
    R max_penetration = 0;
    uint32_t colours = 0;
    // Per-substep record (test hook): after each substep's relax sweep, every
    // body's position, rotation, linear and angular velocity as float, in
    // body order (13 floats per body).
    bool record_substeps = false;
    std::vector<float> substep_log;
    uint32_t substeps_logged = 0;

    void clear() {
        bodies.clear();
        id2idx.clear();
        cons.clear();
        manager = nullptr;
        position_iterations_run = 0;
        max_penetration = 0;
        colours = 0;
    }
    void addBody(Body<R>* b) {  // solver.zig:429-435, BodyState.fromBody 231-243
        if (id2idx.count(b->id)) return;
        id2idx[b->id] = (uint32_t)bodies.size();
        bodies.push_back({b->pos, b->rot, b->v, b->w, b->inv_mass, b->worldInvInertia(), b->type, b->sleeping, b});
    }
    void addManifold(const Manifold<R>& m) {  // solver.zig:449-491
        auto ia = id2idx.find(m.a), ib = id2idx.find(m.b);
        if (ia == id2idx.end() || ib == id2idx.end()) return;
        const BodyState<R>& sa = bodies[ia->second];
        const BodyState<R>& sb = bodies[ib->second];
        CManifold<R> cm{};
        cm.ia = ia->second;
        cm.ib = ib->second;
        cm.friction = m.friction;
        cm.restitution = m.restitution;
        cm.n = m.n;
        cm.order = (uint32_t)cons.size();
        for (uint32_t i = 0; i < m.n; ++i) {
            const Contact<R>& c = m.c[i];
            const V3<R> wa = add(qrotate(sa.q, c.la), sa.p);
            const V3<R> wb = add(qrotate(sb.q, c.lb), sb.p);
            const V3<R> ad = sub(wb, wa);
            CPoint<R>& p = cm.pt[i];
            p = CPoint<R>{};
            p.point = c.point;
            p.normal = c.normal;
            p.la = c.la;
            p.lb = c.lb;
            p.ra = sub(wa, sa.p);
            p.rb = sub(wb, sb.p);
            p.base_sep = -c.penetration - dot(ad, c.normal);
            p.ni = c.normal_impulse;
            p.ti[0] = c.tangent_impulse[0];
            p.ti[1] = c.tangent_impulse[1];
            p.penetration = c.penetration;
        }
        cons.push_back(cm);
    }

    // Project colouring: sequential greedy in Jones-Plassmann priority order
    // over writable bodies.  Returns the number of colours.
    uint32_t colourProject() {
        const uint32_t M = (uint32_t)cons.size();
        std::vector<uint32_t> order(M);
        for (uint32_t k = 0; k < M; ++k) order[k] = k;
        std::sort(order.begin(), order.end(), [](uint32_t i, uint32_t j) { return jpBefore(i, j); });
        std::vector<std::vector<uint32_t>> body_cons(bodies.size());
        for (uint32_t k = 0; k < M; ++k) {
            if (bodies[cons[k].ia].writable()) body_cons[cons[k].ia].push_back(k);
            if (bodies[cons[k].ib].writable() && cons[k].ib != cons[k].ia) body_cons[cons[k].ib].push_back(k);
        }
        std::vector<int32_t> col(M, -1);
        uint32_t ncol = 0;
        for (uint32_t k : order) {
            std::vector<bool> used(ncol + 1, false);
            for (uint32_t bi : {cons[k].ia, cons[k].ib}) {
                if (!bodies[bi].writable()) continue;
                for (uint32_t j : body_cons[bi])
                    if (col[j] >= 0) used[(size_t)col[j]] = true;
            }
            uint32_t c = 0;
            while (used[c]) ++c;
            col[k] = (int32_t)c;
            ncol = std::max(ncol, c + 1);
        }
        for (uint32_t k = 0; k < M; ++k) cons[k].colour = (uint32_t)col[k];
        return ncol;
    }

    void sortColourMajor() {
        std::stable_sort(cons.begin(), cons.end(),
                         [](const CManifold<R>& x, const CManifold<R>& y) { return x.colour < y.colour; });
    }

    void solve(R dt) {  // solver.zig:494-561
        if (dt <= 0) return;
        if (bodies.empty()) return;
        const bool has = !cons.empty();
        const R h = dt / (R)cfg.substeps;
        const SoftParams<R> soft = computeSoftParams(cfg.hertz, cfg.damping_ratio, h);
        substep_log.clear();
        substeps_logged = 0;
        for (uint32_t s = 0; s < cfg.substeps; ++s) {
            applyGravity(h);
            if (has) {
                prepare(soft, h);
                if (cfg.warm_starting && s == 0) warmStart();
                for (uint32_t it = 0; it < cfg.velocity_iterations; ++it) solveVelocity(soft, true);
            }
            for (auto& b : bodies) b.integratePosition(h, cfg.disable_rotation);
            if (has) solveVelocity(SoftParams<R>{0, 1, 1}, false);
            if (record_substeps) {
                for (const auto& b : bodies) {
                    const float r[13] = {(float)b.p.x, (float)b.p.y, (float)b.p.z, (float)b.q.x, (float)b.q.y,
                                         (float)b.q.z, (float)b.q.w, (float)b.v.x, (float)b.v.y, (float)b.v.z,
                                         (float)b.w.x, (float)b.w.y, (float)b.w.z};
                    substep_log.insert(substep_log.end(), r, r + 13);
                }
                ++substeps_logged;
            }
        }
        if (has) {
            for (uint32_t it = 0; it < cfg.position_iterations; ++it) {
                position_iterations_run++;
                if (solvePosition()) break;
            }
        }
        for (auto& b : bodies) b.writeBack();
        if (has) storeImpulses();
    }
    void applyGravity(R h) {  // solver.zig:564-605
        for (auto& s : bodies) {
            if (!(s.type == B_DYNAMIC && !s.sleeping)) continue;
            s.v = add(s.v, scale(cfg.gravity, h));
            R ld = s.body->lin_damp, ad = s.body->ang_damp;
            const R ls = len(s.v), as = len(s.w);
            if (ls < (R)0.5f) ld += (R)5.0f * ((R)1.0 - (ls / (R)0.5f));
            if (as < (R)0.5f) ad += (R)5.0f * ((R)1.0 - (as / (R)0.5f));
            const R ldec = fmx((R)0.0, (R)1.0 - ld * h), adec = fmx((R)0.0, (R)1.0 - ad * h);
            s.v = scale(s.v, ldec);
            s.w = scale(s.w, adec);
            const R ve = (R)0.001f;
            if (len2(s.v) < ve * ve) s.v = {0, 0, 0};
            if (len2(s.w) < ve * ve) s.w = {0, 0, 0};
        }
    }
    void prepare(const SoftParams<R>& soft, R h) {  // solver.zig:608-699
        const R hinv = h > kEps<R>() ? (R)1 / h : (R)0;
        for (auto& cm : cons) {
            const BodyState<R>& a = bodies[cm.ia];
            const BodyState<R>& b = bodies[cm.ib];
            for (uint32_t i = 0; i < cm.n; ++i) {
                CPoint<R>& cp = cm.pt[i];
                const V3<R> wa = add(qrotate(a.q, cp.la), a.p);
                const V3<R> wb = add(qrotate(b.q, cp.lb), b.p);
                cp.ra = sub(wa, a.p);
                cp.rb = sub(wb, b.p);
                cp.point = scale(add(wa, wb), (R)0.5);
                const V3<R> ad = sub(wb, wa);
                const R sep = cp.base_sep + dot(ad, cp.normal);
                const V3<R> rna = cross(cp.ra, cp.normal), rnb = cross(cp.rb, cp.normal);
                R k = a.inv_mass + b.inv_mass;
                k += dot(rna, mulVec(a.iiw, rna));
                k += dot(rnb, mulVec(b.iiw, rnb));
                cp.normal_mass = k > kEps<R>() ? (R)1 / k : (R)0;
                const V3<R> rv = sub(b.pointVel(cp.point), a.pointVel(cp.point));
                const R vn = dot(rv, cp.normal);
                cp.init_vn = vn;
                if (sep > (R)0) cp.bias = sep * hinv;
                else cp.bias = fmx(soft.bias_rate * sep, (R)-0.2);
                if (cfg.enable_restitution && vn < -(R)1.0f) cp.bias = fmx(cp.bias, -cm.restitution * vn);
                if (cfg.enable_friction) {
                    cp.t1 = computeOrthogonal(cp.normal);
                    cp.t2 = cross(cp.normal, cp.t1);
                    const V3<R> r1a = cross(cp.ra, cp.t1), r1b = cross(cp.rb, cp.t1);
                    R k1 = a.inv_mass + b.inv_mass;
                    k1 += dot(r1a, mulVec(a.iiw, r1a));
                    k1 += dot(r1b, mulVec(b.iiw, r1b));
                    cp.tangent_mass[0] = k1 > kEps<R>() ? (R)1 / k1 : (R)0;
                    const V3<R> r2a = cross(cp.ra, cp.t2), r2b = cross(cp.rb, cp.t2);
                    R k2 = a.inv_mass + b.inv_mass;
                    k2 += dot(r2a, mulVec(a.iiw, r2a));
                    k2 += dot(r2b, mulVec(b.iiw, r2b));
                    cp.tangent_mass[1] = k2 > kEps<R>() ? (R)1 / k2 : (R)0;
                }
            }
        }
    }
    void warmStart() {  // solver.zig:702-729
        const R sc = cfg.warm_start_scale;
        for (auto& cm : cons) {
            BodyState<R>& a = bodies[cm.ia];
            BodyState<R>& b = bodies[cm.ib];
            for (uint32_t i = 0; i < cm.n; ++i) {
                CPoint<R>& cp = cm.pt[i];
                const R sn = cp.ni * sc, s1 = cp.ti[0] * sc, s2 = cp.ti[1] * sc;
                const V3<R> imp = add(add(scale(cp.normal, sn), scale(cp.t1, s1)), scale(cp.t2, s2));
                a.applyImpulseAtPoint(neg(imp), cp.ra);
                b.applyImpulseAtPoint(imp, cp.rb);
                cp.ni = sn;
                cp.ti[0] = s1;
                cp.ti[1] = s2;
            }
        }
    }
    void solveVelocity(const SoftParams<R>& soft, bool use_bias) {  // solver.zig:732-838
        for (auto& cm : cons) {
            BodyState<R>& a = bodies[cm.ia];
            BodyState<R>& b = bodies[cm.ib];
            for (uint32_t i = 0; i < cm.n; ++i) {
                CPoint<R>& cp = cm.pt[i];
                const V3<R> rv = sub(b.pointVel(cp.point), a.pointVel(cp.point));
                const R vn = dot(rv, cp.normal);
                R imp;
                if (use_bias) imp = -soft.mass_coeff * cp.normal_mass * (vn + cp.bias) - soft.impulse_coeff * cp.ni;
                else imp = -cp.normal_mass * vn;
                const R nn = fmx(cp.ni + imp, (R)0);
                imp = nn - cp.ni;
                cp.ni = nn;
                const V3<R> P = scale(cp.normal, imp);
                a.applyImpulseAtPoint(neg(P), cp.ra);
                b.applyImpulseAtPoint(P, cp.rb);
                if (cfg.enable_friction && cm.friction > 0) {
                    const V3<R> rv1 = sub(b.pointVel(cp.point), a.pointVel(cp.point));
                    const R mf = cm.friction * cp.ni;
                    {
                        const R vt1 = dot(rv1, cp.t1);
                        R f1 = -cp.tangent_mass[0] * vt1;
                        const R o1 = cp.ti[0];
                        cp.ti[0] = fclamp(o1 + f1, -mf, mf);
                        f1 = cp.ti[0] - o1;
                        const V3<R> I1 = scale(cp.t1, f1);
                        a.applyImpulseAtPoint(neg(I1), cp.ra);
                        b.applyImpulseAtPoint(I1, cp.rb);
                    }
                    {
                        const V3<R> rv2 = sub(b.pointVel(cp.point), a.pointVel(cp.point));
                        const R vt2 = dot(rv2, cp.t2);
                        R f2 = -cp.tangent_mass[1] * vt2;
                        const R o2 = cp.ti[1];
                        cp.ti[1] = fclamp(o2 + f2, -mf, mf);
                        f2 = cp.ti[1] - o2;
                        const V3<R> I2 = scale(cp.t2, f2);
                        a.applyImpulseAtPoint(neg(I2), cp.ra);
                        b.applyImpulseAtPoint(I2, cp.rb);
                    }
                }
            }
        }
    }
    bool solvePosition() {  // solver.zig:860-923
        R min_sep = 0;
        for (auto& cm : cons) {
            BodyState<R>& a = bodies[cm.ia];
            BodyState<R>& b = bodies[cm.ib];
            if (a.type == B_STATIC && b.type == B_STATIC) continue;
            for (uint32_t i = 0; i < cm.n; ++i) {
                CPoint<R>& cp = cm.pt[i];
                const V3<R> wa = add(qrotate(a.q, cp.la), a.p);
                const V3<R> wb = add(qrotate(b.q, cp.lb), b.p);
                const V3<R> ad = sub(wb, wa);
                const R sep = cp.base_sep + dot(ad, cp.normal);
                min_sep = fmn(min_sep, sep);
                max_penetration = fmx(max_penetration, -sep);
                if (sep >= -cfg.slop) continue;
                const R corr = fmx(cfg.position_correction_rate * (sep + cfg.slop), -cfg.max_position_correction);
                const V3<R> ra = sub(wa, a.p), rb = sub(wb, b.p);
                const V3<R> rna = cross(ra, cp.normal), rnb = cross(rb, cp.normal);
                R k = a.inv_mass + b.inv_mass;
                k += dot(rna, mulVec(a.iiw, rna));
                k += dot(rnb, mulVec(b.iiw, rnb));
                if (k < kEps<R>()) continue;
                const V3<R> pi = scale(cp.normal, -corr / k);
                if (a.type == B_DYNAMIC && !a.sleeping) {
                    a.p = sub(a.p, scale(pi, a.inv_mass));
                    a.q = integrateRotationSmall(a.q, mulVec(a.iiw, cross(ra, neg(pi))));
                }
                if (b.type == B_DYNAMIC && !b.sleeping) {
                    b.p = add(b.p, scale(pi, b.inv_mass));
                    b.q = integrateRotationSmall(b.q, mulVec(b.iiw, cross(rb, pi)));
                }
            }
        }
        return min_sep >= (R)-3.0 * cfg.slop;
    }
    void storeImpulses() {  // solver.zig:933-958
        if (!manager) return;
        for (auto& cm : cons) {
            Manifold<R>* m = manager->getMut(bodies[cm.ia].body->id, bodies[cm.ib].body->id);
            if (!m) continue;
            const uint32_t n = std::min(cm.n, m->n);
            for (uint32_t i = 0; i < n; ++i) {
                m->c[i].normal_impulse = cm.pt[i].ni;
                m->c[i].tangent_impulse[0] = cm.pt[i].ti[0];
                m->c[i].tangent_impulse[1] = cm.pt[i].ti[1];
                m->c[i].normal_mass = cm.pt[i].normal_mass;
                m->c[i].tangent_mass[0] = cm.pt[i].tangent_mass[0];
                m->c[i].tangent_mass[1] = cm.pt[i].tangent_mass[1];
            }
        }
    }
};

// GraphColoring.build (islands.zig:668-736) over manifolds in list order.
// Returns per-manifold colours; *max_colour set.
template <class R>
inline std::vector<uint8_t> graphColouring(const std::vector<Manifold<R>>& ms, uint32_t* max_colour) {
    std::unordered_map<uint32_t, std::vector<uint32_t>> bm;
    for (uint32_t i = 0; i < ms.size(); ++i) {
        bm[ms[i].a].push_back(i);
        bm[ms[i].b].push_back(i);
    }
    std::vector<uint8_t> colours;
    colours.reserve(ms.size());
    uint32_t mc = 0;
    for (uint32_t i = 0; i < ms.size(); ++i) {
        bool used[256] = {false};
        for (uint32_t id : {ms[i].a, ms[i].b}) {
            auto it = bm.find(id);
            if (it == bm.end()) continue;
            for (uint32_t j : it->second)
                if (j < colours.size()) used[colours[j]] = true;
        }
        uint32_t c = 0;
        while (c < 255 && used[c]) ++c;
        colours.push_back((uint8_t)c);
        mc = std::max(mc, c);
    }
    *max_colour = mc;
    return colours;
}

// ---------------------------------------------------------------------------
// islands.zig: UnionFind (25-137) and IslandManager (194-495), as
// system.solve drives it (system.zig:705-760).  Only its statistics leave it:
// updateSleepStates reads copies of the bodies and writes none of them.
// ---------------------------------------------------------------------------
struct UnionFind {  // islands.zig:25-137
    std::vector<uint32_t> parent, rank;
    size_t count = 0, set_count = 0;
    explicit UnionFind(size_t n = 0) { resize(n); }
    void reset() {
        for (size_t i = 0; i < count; ++i) {
            parent[i] = (uint32_t)i;
            rank[i] = 0;
        }
        set_count = count;
    }
    void resize(size_t n) {
        if (n > parent.size()) {
            parent.resize(n);
            rank.resize(n);
        }
        count = n;
        reset();
    }
    uint32_t find(uint32_t x) {  // with path compression
        if (x >= count) return x;
        uint32_t root = x;
        while (parent[root] != root) root = parent[root];
        uint32_t cur = x;
        while (cur != root) {
            const uint32_t next = parent[cur];
            parent[cur] = root;
            cur = next;
        }
        return root;
    }
    void unite(uint32_t x, uint32_t y) {  // union by rank
        const uint32_t rx = find(x), ry = find(y);
        if (rx == ry) return;
        if (rank[rx] < rank[ry]) {
            parent[rx] = ry;
        } else if (rank[rx] > rank[ry]) {
            parent[ry] = rx;
        } else {
            parent[ry] = rx;
            rank[rx] += 1;
        }
        set_count -= 1;
    }
    bool connected(uint32_t x, uint32_t y) { return find(x) == find(y); }
};

template <class R> struct IslandManager {
    struct Island {
        std::vector<uint32_t> bodies, manifolds;
        uint32_t id = 0;
        bool is_sleeping = false;
        R sleep_timer = 0;
        bool needs_solving = true;
    };
    UnionFind uf;
    std::vector<Island> islands;
    std::unordered_map<uint32_t, uint32_t> body_to_island;
    uint64_t previous_graph_hash = 0;
    bool needs_rebuild = true;
    uint32_t rebuilds_skipped = 0, rebuilds_performed = 0;
    size_t total_islands = 0, active_islands = 0, sleeping_islands = 0, largest_island_size = 0, total_bodies = 0,
           total_contacts = 0;

    explicit IslandManager(size_t max_bodies = 1024) : uf(max_bodies) {}

    // computeGraphHash (islands.zig:277-296): every manifold is active
    static uint64_t graphHash(const std::vector<Manifold<R>>& ms) {
        uint64_t hash = 0;
        const uint64_t prime = 0x100000001b3ull;
        for (const auto& m : ms) {
            const uint32_t a = std::min(m.a, m.b), b = std::max(m.a, m.b);
            hash ^= ((uint64_t)a << 32) | (uint64_t)b;
            hash *= prime;
        }
        hash ^= (uint64_t)ms.size();
        hash *= prime;
        return hash;
    }
    void markDirty() { needs_rebuild = true; }  // islands.zig:299-302

    // buildIslandsWithBodyTypes (islands.zig:318-423); types[id] for ids
    // below types.size(), as the reference's body_types slice
    void build(const std::vector<Manifold<R>>& ms, size_t body_count, const std::vector<uint32_t>& types) {
        const uint64_t h = graphHash(ms);
        if (!needs_rebuild && h == previous_graph_hash && total_islands > 0) {
            ++rebuilds_skipped;
            return;
        }
        previous_graph_hash = h;
        needs_rebuild = false;
        ++rebuilds_performed;
        for (auto& isl : islands) isl = Island{};
        body_to_island.clear();
        total_islands = active_islands = sleeping_islands = largest_island_size = total_bodies = total_contacts = 0;
        if (ms.empty()) return;
        // the body ids the manifolds name; the reference walks a hash set, so
        // its island numbering follows hash order: no statistic depends on it
        std::vector<uint32_t> body_ids;
        for (const auto& m : ms) {
            body_ids.push_back(m.a);
            body_ids.push_back(m.b);
        }
        std::sort(body_ids.begin(), body_ids.end());
        body_ids.erase(std::unique(body_ids.begin(), body_ids.end()), body_ids.end());
        const uint32_t max_id = body_ids.back();
        const size_t required = std::max(body_count, (size_t)max_id + 1);
        if (required > uf.count) uf.resize(required);
        else uf.reset();
        for (const auto& m : ms) {
            const bool as = m.a < types.size() && types[m.a] == B_STATIC;
            const bool bs = m.b < types.size() && types[m.b] == B_STATIC;
            if (as || bs) continue;
            uf.unite(m.a, m.b);
        }
        total_contacts = ms.size();
        std::unordered_map<uint32_t, uint32_t> root_to_island;
        uint32_t count = 0;
        for (uint32_t id : body_ids) {
            const uint32_t root = uf.find(id);
            if (!root_to_island.count(root)) {
                root_to_island[root] = count;
                while (islands.size() <= count) islands.emplace_back();
                islands[count].id = root;
                ++count;
            }
            const uint32_t idx = root_to_island[root];
            body_to_island[id] = idx;
            auto& bl = islands[idx].bodies;
            if (std::find(bl.begin(), bl.end(), id) == bl.end()) bl.push_back(id);
        }
        for (uint32_t mi = 0; mi < ms.size(); ++mi) {
            auto it = root_to_island.find(uf.find(ms[mi].a));
            if (it != root_to_island.end()) islands[it->second].manifolds.push_back(mi);
        }
        total_islands = count;
        for (uint32_t k = 0; k < count; ++k) {
            const size_t size = islands[k].bodies.size();
            total_bodies += size;
            largest_island_size = std::max(largest_island_size, size);
            if (islands[k].is_sleeping) ++sleeping_islands;
            else ++active_islands;
        }
    }

    // updateSleepStates (islands.zig:426-472).  bodies: the body table, read
    // at index body id, as the reference reads its copies (islands.zig:437-440).
    void updateSleepStates(const std::vector<Body<R>>& bodies, R dt) {
        const R thr = (R)(0.1f * 0.1f);  // ISLAND_SLEEP_{LINEAR,ANGULAR}_THRESHOLD squared, in f32
        for (auto& isl : islands) {
            if (isl.bodies.empty()) continue;
            bool all_still = true;
            for (uint32_t id : isl.bodies) {
                if (id >= bodies.size()) continue;
                const Body<R>& b = bodies[id];
                if (b.type != B_DYNAMIC) continue;
                if (dot(b.v, b.v) > thr || dot(b.w, b.w) > thr) {
                    all_still = false;
                    break;
                }
            }
            if (all_still) {
                isl.sleep_timer += dt;
                if (isl.sleep_timer >= (R)0.5f) {  // ISLAND_SLEEP_TIME_THRESHOLD
                    isl.is_sleeping = true;
                    isl.needs_solving = false;
                }
            } else {
                isl.sleep_timer = 0;
                isl.is_sleeping = false;
                isl.needs_solving = true;
            }
        }
        sleeping_islands = active_islands = 0;
        for (size_t k = 0; k < total_islands; ++k) {
            if (islands[k].is_sleeping) ++sleeping_islands;
            else ++active_islands;
        }
    }
};

// ---------------------------------------------------------------------------
// system.zig: step / narrowPhase / solve / updateSleepStates
// ---------------------------------------------------------------------------
struct Stats {
    uint32_t pairs_in = 0, pairs_tested = 0, pairs_colliding = 0, voxels_checked = 0, contacts_generated = 0,
             pairs_skipped_sleeping = 0, manifolds_preserved = 0, cache_hits = 0, cache_misses = 0,
             cache_evictions = 0, manifolds = 0, constraints = 0, contact_points = 0, colours = 0,
             position_iterations_run = 0, step_skipped = 0;
    float max_penetration = 0;
    uint32_t candidates = 0;
    // PhysicsStats island fields (system.zig:119-122)
    uint32_t island_count = 0, active_islands = 0, sleeping_islands = 0, largest_island_size = 0;
};

struct WorldConfig {
    float gravity[3] = {0, -9.81f, 0};
    float fixed_timestep = 1.0f / 60.0f;
    bool enable_sleeping = true, enable_warm_starting = true;
    bool use_brick_sat = true, use_brick_pair_cache = true;
    uint32_t cache_size = 1024;
    bool reference_caps = false;
    uint32_t colouring = COLOUR_PROJECT;
    bool enable_islands = true;
};

template <class R> struct World {
    WorldConfig wcfg;
    SolverConfig<R> scfg;
    std::vector<Collider<R>> colliders;
    std::vector<Body<R>> bodies;
    std::unordered_map<uint32_t, uint32_t> id2idx;
    ContactManager<R> cm;
    BrickPairCache<R> cache;
    ContactSolver<R> solver;
    Stats stats;
    IslandManager<R> islands;
    bool dump = false;
    std::vector<CandRec> candidates;
    std::vector<uint32_t> last_colours;  // per constraint in addManifold order
    bool colouring_overflow = false;

    World(const WorldConfig& w, const SolverConfig<R>& s) : wcfg(w), scfg(s), cache(w.cache_size) {
        solver.cfg = s;
    }

    void reindex() {
        id2idx.clear();
        for (uint32_t i = 0; i < bodies.size(); ++i) id2idx[bodies[i].id] = i;
    }
    Body<R>* find(uint32_t id) {
        auto it = id2idx.find(id);
        return it == id2idx.end() ? nullptr : &bodies[it->second];
    }

    bool allDynamicSleeping() const {  // system.zig:558-567
        for (const auto& b : bodies)
            if (b.type == B_DYNAMIC && !b.sleeping) return false;
        return true;
    }

    void step(R dt, const std::vector<std::pair<uint32_t, uint32_t>>& pairs) {  // system.zig:537-555
        stats = Stats{};
        stats.pairs_in = (uint32_t)pairs.size();
        solver.substep_log.clear();
        solver.substeps_logged = 0;
        if (wcfg.enable_sleeping && allDynamicSleeping()) {
            stats.step_skipped = 1;
            return;
        }
        narrowPhase(pairs);
        solve(dt);
        if (wcfg.enable_sleeping)
            for (auto& b : bodies)
                if (b.type == B_DYNAMIC && !b.sleeping) b.updateSleepState(dt);
    }

    void processPair(const Body<R>& a, const Body<R>& b, uint32_t pidx) {  // narrow_phase.zig:1414-1525
        stats.pairs_tested++;
        if (a.sleeping && b.sleeping) {
            const Manifold<R>* pm = cm.prevGet(pairKey(a.id, b.id));
            if (pm) {
                stats.pairs_skipped_sleeping++;
                stats.manifolds_preserved++;
                stats.contacts_generated += pm->n;
                cm.put(pairKey(a.id, b.id), *pm);
                return;
            }
            stats.pairs_skipped_sleeping++;
            return;
        }
        if (a.collider < 0 || b.collider < 0) return;
        const Collider<R>& ca = colliders[(size_t)a.collider];
        const Collider<R>& cb = colliders[(size_t)b.collider];
        const Xf<R> ta = a.xf(), tb = b.xf();
        if (wcfg.use_brick_sat) {
            if (satEarlyOut(obbFromAabb(ca.local_aabb, ta), obbFromAabb(cb.local_aabb, tb))) return;
        }
        const bool use_cache = wcfg.use_brick_pair_cache &&
                               (a.type == B_STATIC || b.type == B_STATIC || a.sleeping || b.sleeping);
        std::vector<CandRec>* dp = dump ? &candidates : nullptr;
        if (use_cache) {
            const V3<R> rp = sub(tb.p, ta.p);
            const Q<R> rr = qmul(qconj(ta.q), tb.q);
            const CacheKey key = makeCacheKey(a.id, b.id, IV3{0, 0, 0}, IV3{0, 0, 0},
                                              V3<float>{(float)rp.x, (float)rp.y, (float)rp.z},
                                              Q<float>{(float)rr.x, (float)rr.y, (float)rr.z, (float)rr.w});
            const uint64_t ev0 = cache.evictions;
            if (const CacheValue<R>* cv = cache.get(key)) {
                stats.cache_hits++;
                if (cv->has_collision) {
                    Manifold<R> m;
                    m.a = a.id;
                    m.b = b.id;
                    m.friction = std::sqrt(a.friction * b.friction);
                    m.restitution = fmx(a.restitution, b.restitution);
                    for (uint32_t i = 0; i < cv->n; ++i) m.addContact(cv->c[i]);
                    stats.pairs_colliding++;
                    stats.contacts_generated += cv->n;
                    stats.voxels_checked += cv->voxels_checked;
                    cm.addManifold(m);
                }
                return;
            }
            stats.cache_misses++;
            DetectResult<R> r = detectVoxelCollisions(a, ca, b, cb, dp, pidx);
            stats.candidates += r.candidates;
            CacheValue<R> v;
            v.has_collision = r.has_collision;
            v.voxels_checked = r.voxels_checked;
            if (r.has_collision) {
                v.n = (uint8_t)std::min<uint32_t>(r.m.n, 4);
                for (uint32_t i = 0; i < v.n; ++i) v.c[i] = r.m.c[i];
            }
            cache.put(key, v);
            stats.cache_evictions += (uint32_t)(cache.evictions - ev0);
            stats.voxels_checked += r.voxels_checked;
            if (r.has_collision) {
                stats.pairs_colliding++;
                stats.contacts_generated += r.m.n;
                cm.addManifold(r.m);
            }
        } else {
            DetectResult<R> r = detectVoxelCollisions(a, ca, b, cb, dp, pidx);
            stats.candidates += r.candidates;
            stats.voxels_checked += r.voxels_checked;
            if (r.has_collision) {
                stats.pairs_colliding++;
                stats.contacts_generated += r.m.n;
                cm.addManifold(r.m);
            }
        }
    }

    // system.zig:586-655 (sequential path).  Manifolds are kept in pair order:
    // a carried both-sleeping manifold takes its pair's position.
    void narrowPhase(const std::vector<std::pair<uint32_t, uint32_t>>& pairs) {
        cm.beginFrame();
        cache.beginFrame();
        candidates.clear();
        uint32_t skipped = 0, kept = 0;
        for (uint32_t i = 0; i < pairs.size(); ++i) {
            Body<R>* a = find(pairs[i].first);
            Body<R>* b = find(pairs[i].second);
            const bool as = a ? a->sleeping : false, bs = b ? b->sleeping : false;
            if (as && bs) {
                skipped++;
                const uint64_t key = pairKey(pairs[i].first, pairs[i].second);
                if (const Manifold<R>* pm = cm.prevGet(key)) cm.put(key, *pm);
                continue;
            }
            if (wcfg.reference_caps && kept >= 512) continue;
            kept++;
            if (a && b) processPair(*a, *b, i);
        }
        stats.pairs_skipped_sleeping += skipped;
        stats.manifolds = (uint32_t)cm.cur.size();
    }

    void solve(R dt) {  // system.zig:670-783
        solver.clear();
        solver.cfg.gravity = {(R)wcfg.gravity[0], (R)wcfg.gravity[1], (R)wcfg.gravity[2]};
        for (auto& b : bodies) solver.addBody(&b);
        if (wcfg.enable_warm_starting) solver.manager = &cm;
        std::vector<uint32_t> ref_colour_of_cons;
        uint32_t ref_max = 0;
        std::vector<uint8_t> ref_colours;
        if (wcfg.colouring == COLOUR_REFERENCE) ref_colours = graphColouring(cm.cur, &ref_max);
        for (uint32_t mi = 0; mi < cm.cur.size(); ++mi) {
            const Manifold<R>& m = cm.cur[mi];
            Body<R>* a = find(m.a);
            Body<R>* b = find(m.b);
            const bool as = a ? a->sleeping : true, bs = b ? b->sleeping : true;
            if (as && bs) continue;
            solver.addManifold(m);
            if (wcfg.colouring == COLOUR_REFERENCE) ref_colour_of_cons.push_back(ref_colours[mi]);
        }
        stats.constraints = (uint32_t)solver.cons.size();
        if (wcfg.enable_islands) {  // system.zig:705-760
            uint32_t max_id = 0;
            for (const auto& b : bodies) max_id = std::max(max_id, b.id);
            std::vector<uint32_t> types((size_t)max_id + 1, B_STATIC);
            for (const auto& b : bodies) types[b.id] = b.type;
            islands.build(cm.cur, bodies.size(), types);
            islands.updateSleepStates(bodies, dt);
            stats.island_count = (uint32_t)islands.total_islands;
            stats.active_islands = (uint32_t)islands.active_islands;
            stats.sleeping_islands = (uint32_t)islands.sleeping_islands;
            stats.largest_island_size = (uint32_t)islands.largest_island_size;
        }
        uint32_t pts = 0;
        for (auto& c : solver.cons) pts += c.n;
        stats.contact_points = pts;
        colouring_overflow = false;
        if (wcfg.colouring == COLOUR_PROJECT) {
            stats.colours = solver.colourProject();
        } else if (wcfg.colouring == COLOUR_REFERENCE) {
            uint32_t mx = 0;
            for (uint32_t k = 0; k < solver.cons.size(); ++k) {
                solver.cons[k].colour = ref_colour_of_cons[k];
                mx = std::max(mx, ref_colour_of_cons[k] + 1);
            }
            colouring_overflow = ref_max >= 255;
            stats.colours = mx;
        } else {
            stats.colours = solver.cons.empty() ? 0 : 1;
        }
        last_colours.resize(solver.cons.size());
        for (uint32_t k = 0; k < solver.cons.size(); ++k) last_colours[k] = solver.cons[k].colour;
        if (wcfg.colouring != COLOUR_NONE) solver.sortColourMajor();
        solver.solve(dt);
        stats.position_iterations_run = solver.position_iterations_run;
        stats.max_penetration = (float)solver.max_penetration;
    }

    // Pair source: inflated world AABB overlap, not both static, sorted (a, b).
    std::vector<std::pair<uint32_t, uint32_t>> findPairs(R margin) const {
        std::vector<std::pair<uint32_t, uint32_t>> out;
        const size_t n = bodies.size();
        std::vector<Aabb<R>> bx(n);
        for (size_t i = 0; i < n; ++i) {
            const Body<R>& b = bodies[i];
            if (b.collider < 0) {
                bx[i] = {b.pos, b.pos};
            } else {
                bx[i] = aabbTransform(colliders[(size_t)b.collider].local_aabb, b.xf());
            }
            bx[i].mn = sub(bx[i].mn, splat(margin));
            bx[i].mx = add(bx[i].mx, splat(margin));
        }
        for (size_t i = 0; i < n; ++i)
            for (size_t j = i + 1; j < n; ++j) {
                if (bodies[i].type == B_STATIC && bodies[j].type == B_STATIC) continue;
                const Aabb<R>& p = bx[i];
                const Aabb<R>& q = bx[j];
                if (p.mn.x <= q.mx.x && p.mx.x >= q.mn.x && p.mn.y <= q.mx.y && p.mx.y >= q.mn.y &&
                    p.mn.z <= q.mx.z && p.mx.z >= q.mn.z) {
                    const uint32_t a = std::min(bodies[i].id, bodies[j].id), c = std::max(bodies[i].id, bodies[j].id);
                    out.push_back({a, c});
                }
            }
        std::sort(out.begin(), out.end());
        return out;
    }
};

}  // namespace vxo
