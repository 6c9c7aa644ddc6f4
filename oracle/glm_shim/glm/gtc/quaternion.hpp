// glm-subset shim, quaternion part: TEST INFRASTRUCTURE ONLY (see ../glm.hpp).
// Unit-quaternion algebra written from the Hamilton product and the standard rotation formulas.
#ifndef PXB_GLM_SHIM_QUATERNION_HPP
#define PXB_GLM_SHIM_QUATERNION_HPP

#include <cfloat>
#include <cmath>

#include "../glm.hpp"

namespace glm {

struct quat {
    // Storage order x, y, z, w; the 4-scalar constructor takes (w, x, y, z) as glm's does.
    float x = 0.0f, y = 0.0f, z = 0.0f, w = 1.0f;
    constexpr quat() = default;
    constexpr quat(float w_, float x_, float y_, float z_) : x(x_), y(y_), z(z_), w(w_) {}
    constexpr quat(float w_, const vec3& v) : x(v.x), y(v.y), z(v.z), w(w_) {}
};

inline quat operator*(const quat& p, const quat& q) {
    return quat(p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z,
                p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y,
                p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z,
                p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x);
}
// Rotation of v by unit q:  v + 2*(w*(u x v) + u x (u x v)),  u = (x, y, z).
inline vec3 operator*(const quat& q, const vec3& v) {
    const vec3 u(q.x, q.y, q.z);
    const vec3 uv = cross(u, v);
    const vec3 uuv = cross(u, uv);
    return v + ((uv * q.w) + uuv) * 2.0f;
}
inline quat operator*(const quat& q, float s) { return quat(q.w * s, q.x * s, q.y * s, q.z * s); }
inline quat operator*(float s, const quat& q) { return q * s; }
inline quat operator/(const quat& q, float s) { return quat(q.w / s, q.x / s, q.y / s, q.z / s); }
inline quat operator+(const quat& a, const quat& b) {
    return quat(a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z);
}
inline quat operator-(const quat& q) { return quat(-q.w, -q.x, -q.y, -q.z); }
inline bool operator==(const quat& a, const quat& b) {
    return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}

inline float dot(const quat& a, const quat& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
inline quat conjugate(const quat& q) { return quat(q.w, -q.x, -q.y, -q.z); }
inline quat inverse(const quat& q) { return conjugate(q) / dot(q, q); }
inline float length(const quat& q) { return std::sqrt(dot(q, q)); }
inline quat normalize(const quat& q) {
    const float len = length(q);
    if (len <= 0.0f) return quat(1.0f, 0.0f, 0.0f, 0.0f);
    const float inv = 1.0f / len;
    return quat(q.w * inv, q.x * inv, q.y * inv, q.z * inv);
}

// Rotation matrix of a unit quaternion (columns are the rotated basis vectors).
inline mat3 mat3_cast(const quat& q) {
    const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const float xz = q.x * q.z, xy = q.x * q.y, yz = q.y * q.z;
    const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    return mat3(1.0f - 2.0f * (yy + zz), 2.0f * (xy + wz), 2.0f * (xz - wy),
                2.0f * (xy - wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + wx),
                2.0f * (xz + wy), 2.0f * (yz - wx), 1.0f - 2.0f * (xx + yy));
}
inline mat4 mat4_cast(const quat& q) { return mat4(mat3_cast(q)); }

// Quaternion for a rotation of `angle` radians about unit `axis`.
inline quat angleAxis(float angle, const vec3& axis) {
    const float half = angle * 0.5f;
    const float s = std::sin(half);
    return quat(std::cos(half), axis * s);
}

// Spherical linear interpolation along the shorter arc, falling back to a component-wise lerp
// when the two rotations are within FLT_EPSILON of each other (sin(theta) -> 0).
inline quat slerp(const quat& a, const quat& b_in, float t) {
    quat b = b_in;
    float cos_theta = dot(a, b);
    if (cos_theta < 0.0f) {
        b = -b;
        cos_theta = -cos_theta;
    }
    if (cos_theta > 1.0f - FLT_EPSILON) {
        return quat(mix(a.w, b.w, t), mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t));
    }
    const float theta = std::acos(cos_theta);
    return (std::sin((1.0f - t) * theta) * a + std::sin(t * theta) * b) / std::sin(theta);
}

}  // namespace glm

#endif  // PXB_GLM_SHIM_QUATERNION_HPP
