// host_math.h -- host-side single-precision vector helpers with the reference's formulas.
//
// Used where the host computes values the reference computes (builder rest lengths, collider
// world poses, the solve prologue), so the host result is the reference's bit for bit:
// dot is left to right, length = sqrt(dot), quaternion rotation v + 2*(w*(u x v) + u x (u x v)).
// The library is built with -ffp-contract=off so no fused multiply-add changes a rounding.
#ifndef PXB_HOST_MATH_H
#define PXB_HOST_MATH_H

#include <cmath>

namespace pxb {
namespace hm {

struct V3 {
    float x, y, z;
};
struct Q4 {
    float x, y, z, w;  // stored x, y, z, w like glm::quat
};

inline V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline V3 ld(const float* p) { return V3{p[0], p[1], p[2]}; }
inline Q4 ldq(const float* p) { return Q4{p[0], p[1], p[2], p[3]}; }
inline void st(float* p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

inline V3 qrot(Q4 q, V3 v) {
    const V3 u{q.x, q.y, q.z};
    const V3 uv = cross(u, v);
    const V3 uuv = cross(u, uv);
    return add(v, mul(add(mul(uv, q.w), uuv), 2.0f));
}
inline Q4 qmul(Q4 p, Q4 q) {
    return Q4{p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y,
              p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z,
              p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x,
              p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z};
}
// Columns of the rotation matrix (glm::mat3_cast), i.e. OBB::axes (obb.h:31-36).
inline void axes(Q4 q, V3& ax, V3& ay, V3& az) {
    const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const float xz = q.x * q.z, xy = q.x * q.y, yz = q.y * q.z;
    const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    ax = V3{1.0f - 2.0f * (yy + zz), 2.0f * (xy + wz), 2.0f * (xz - wy)};
    ay = V3{2.0f * (xy - wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + wx)};
    az = V3{2.0f * (xz + wy), 2.0f * (yz - wx), 1.0f - 2.0f * (xx + yy)};
}
// util::safe_normalize (math.h:46-50).
inline V3 safe_normalize(V3 v) {
    const float l2 = dot(v, v);
    if (l2 < 1e-6f * 1e-6f) return V3{0.0f, 0.0f, 0.0f};
    return mul(v, 1.0f / std::sqrt(l2));
}
// First tangent of util::orthonormal_basis (math.h:62-68).
inline V3 orthonormal_t1(V3 n) {
    const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    return V3{1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x};
}

}  // namespace hm
}  // namespace pxb

#endif  // PXB_HOST_MATH_H
