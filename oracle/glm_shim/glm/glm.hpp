// glm-subset shim: TEST INFRASTRUCTURE ONLY.
//
// The reference library (physxcoopa) does its vector arithmetic through glm (OpenGL
// Mathematics, a third-party header library whose version the reference tree does not pin;
// it reaches the reference through libcoopa, which is absent here). This file re-implements the
// small part of glm's public API that the reference's cloth/hair closure uses, written from the
// GLSL specification's definitions and the quaternion algebra, so that those reference headers
// compile UNMODIFIED into oracle/_ref (see oracle/Makefile).
//
// Semantics follow the GLSL / glm documented definitions:
//   dot(a,b)      = a.x*b.x + a.y*b.y + a.z*b.z      (left to right)
//   length(v)     = sqrt(dot(v,v))
//   normalize(v)  = v * (1 / sqrt(dot(v,v)))         (glm's inversesqrt form)
//   mix(x,y,a)    = x*(1-a) + y*a                    (GLSL definition)
//   clamp(x,l,h)  = min(max(x,l),h)
// Bitwise agreement with any particular glm release is NOT claimed (parity against real glm is
// unpinned); the reference's own tests pin results to tolerances only.
#ifndef PXB_GLM_SHIM_GLM_HPP
#define PXB_GLM_SHIM_GLM_HPP

#include <cmath>
#include <cstdint>
#include <type_traits>

namespace glm {

struct vec4;

struct vec2 {
    float x = 0.0f, y = 0.0f;
    constexpr vec2() = default;
    template <typename S, typename = std::enable_if_t<std::is_arithmetic_v<S>>>
    explicit constexpr vec2(S s) : x(static_cast<float>(s)), y(static_cast<float>(s)) {}
    template <typename A, typename B>
    constexpr vec2(A a, B b) : x(static_cast<float>(a)), y(static_cast<float>(b)) {}
    float& operator[](int i) { return i == 0 ? x : y; }
    const float& operator[](int i) const { return i == 0 ? x : y; }
};
inline vec2 operator+(vec2 a, vec2 b) { return {a.x + b.x, a.y + b.y}; }
inline vec2 operator-(vec2 a, vec2 b) { return {a.x - b.x, a.y - b.y}; }
inline vec2 operator*(vec2 a, float s) { return {a.x * s, a.y * s}; }
inline vec2 operator*(float s, vec2 a) { return {s * a.x, s * a.y}; }
inline vec2 operator-(vec2 a) { return {-a.x, -a.y}; }
inline bool operator==(vec2 a, vec2 b) { return a.x == b.x && a.y == b.y; }
inline float dot(vec2 a, vec2 b) { return a.x * b.x + a.y * b.y; }

struct vec3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    constexpr vec3() = default;
    template <typename S, typename = std::enable_if_t<std::is_arithmetic_v<S>>>
    explicit constexpr vec3(S s)
        : x(static_cast<float>(s)), y(static_cast<float>(s)), z(static_cast<float>(s)) {}
    template <typename A, typename B, typename C>
    constexpr vec3(A a, B b, C c)
        : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)) {}
    explicit vec3(const vec4& v);
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    vec3& operator-=(const vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    vec3& operator*=(const vec3& o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
    vec3& operator/=(const vec3& o) { x /= o.x; y /= o.y; z /= o.z; return *this; }
    vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};
inline vec3 operator+(const vec3& a, const vec3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(const vec3& a, const vec3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator*(const vec3& a, const vec3& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3 operator/(const vec3& a, const vec3& b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline vec3 operator*(const vec3& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline vec3 operator*(float s, const vec3& a) { return {s * a.x, s * a.y, s * a.z}; }
inline vec3 operator/(const vec3& a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline vec3 operator/(float s, const vec3& a) { return {s / a.x, s / a.y, s / a.z}; }
inline vec3 operator+(const vec3& a, float s) { return {a.x + s, a.y + s, a.z + s}; }
inline vec3 operator-(const vec3& a, float s) { return {a.x - s, a.y - s, a.z - s}; }
inline vec3 operator-(const vec3& a) { return {-a.x, -a.y, -a.z}; }
inline bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator!=(const vec3& a, const vec3& b) { return !(a == b); }

struct vec4 {
    float x = 0.0f, y = 0.0f, z = 0.0f, w = 0.0f;
    constexpr vec4() = default;
    template <typename S, typename = std::enable_if_t<std::is_arithmetic_v<S>>>
    explicit constexpr vec4(S s)
        : x(static_cast<float>(s)), y(static_cast<float>(s)), z(static_cast<float>(s)),
          w(static_cast<float>(s)) {}
    template <typename A, typename B, typename C, typename D>
    constexpr vec4(A a, B b, C c, D d)
        : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)),
          w(static_cast<float>(d)) {}
    vec4(const vec3& v, float s) : x(v.x), y(v.y), z(v.z), w(s) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
inline vec3::vec3(const vec4& v) : x(v.x), y(v.y), z(v.z) {}
inline vec4 operator+(const vec4& a, const vec4& b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline vec4 operator*(const vec4& a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }

struct ivec3 {
    int32_t x = 0, y = 0, z = 0;
    constexpr ivec3() = default;
    constexpr ivec3(int32_t a, int32_t b, int32_t c) : x(a), y(b), z(c) {}
};

struct uvec2 {
    uint32_t x = 0, y = 0;
    constexpr uvec2() = default;
    constexpr uvec2(uint32_t a, uint32_t b) : x(a), y(b) {}
};

// Column-major 3x3 matrix: c[i] is column i, as in GLSL.
struct mat3 {
    vec3 c[3];
    mat3() : c{vec3(1, 0, 0), vec3(0, 1, 0), vec3(0, 0, 1)} {}
    explicit mat3(float d) : c{vec3(d, 0, 0), vec3(0, d, 0), vec3(0, 0, d)} {}
    mat3(const vec3& a, const vec3& b, const vec3& d) : c{a, b, d} {}
    mat3(float x0, float y0, float z0, float x1, float y1, float z1, float x2, float y2, float z2)
        : c{vec3(x0, y0, z0), vec3(x1, y1, z1), vec3(x2, y2, z2)} {}
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};
inline vec3 operator*(const mat3& m, const vec3& v) {
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}
inline mat3 operator*(const mat3& a, const mat3& b) { return {a * b.c[0], a * b.c[1], a * b.c[2]}; }
inline mat3 operator*(const mat3& m, float s) { return {m.c[0] * s, m.c[1] * s, m.c[2] * s}; }
inline mat3 operator+(const mat3& a, const mat3& b) { return {a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]}; }
inline mat3 transpose(const mat3& m) {
    return mat3(m.c[0].x, m.c[1].x, m.c[2].x, m.c[0].y, m.c[1].y, m.c[2].y, m.c[0].z, m.c[1].z,
                m.c[2].z);
}

// Column-major 4x4 matrix.
struct mat4 {
    vec4 c[4];
    mat4() : c{vec4(1, 0, 0, 0), vec4(0, 1, 0, 0), vec4(0, 0, 1, 0), vec4(0, 0, 0, 1)} {}
    explicit mat4(float d) : c{vec4(d, 0, 0, 0), vec4(0, d, 0, 0), vec4(0, 0, d, 0), vec4(0, 0, 0, d)} {}
    explicit mat4(const mat3& m)
        : c{vec4(m.c[0], 0.0f), vec4(m.c[1], 0.0f), vec4(m.c[2], 0.0f), vec4(0, 0, 0, 1)} {}
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};
inline vec4 operator*(const mat4& m, const vec4& v) {
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w;
}

// --- scalar helpers ---------------------------------------------------------------------------
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }

// --- vec3 functions ---------------------------------------------------------------------------
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline float length(const vec2& v) { return std::sqrt(dot(v, v)); }
inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline vec3 min(const vec3& a, const vec3& b) { return {min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)}; }
inline vec3 max(const vec3& a, const vec3& b) { return {max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)}; }
inline vec3 clamp(const vec3& x, const vec3& lo, const vec3& hi) { return min(max(x, lo), hi); }
inline vec3 clamp(const vec3& x, float lo, float hi) { return clamp(x, vec3(lo), vec3(hi)); }
inline vec3 mix(const vec3& x, const vec3& y, float a) { return x * (1.0f - a) + y * a; }

// 4x4 inverse by cofactor expansion (column-major storage; m[c][r]).
inline mat4 inverse(const mat4& m) {
    float a[16];
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) a[col * 4 + row] = m.c[col][row];
    float inv[16];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] +
             a[9] * a[7] * a[14] + a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] -
             a[8] * a[7] * a[14] - a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] +
             a[8] * a[7] * a[13] + a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] -
              a[8] * a[6] * a[13] - a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] -
             a[9] * a[3] * a[14] - a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] +
             a[8] * a[3] * a[14] + a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] -
             a[8] * a[3] * a[13] - a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] +
              a[8] * a[2] * a[13] + a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] +
             a[5] * a[3] * a[14] + a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] -
             a[4] * a[3] * a[14] - a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] +
              a[4] * a[3] * a[13] + a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] -
              a[4] * a[2] * a[13] - a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] -
             a[5] * a[3] * a[10] - a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] +
             a[4] * a[3] * a[10] + a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] -
              a[4] * a[3] * a[9] - a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] +
              a[4] * a[2] * a[9] + a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    const float det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    const float s = 1.0f / det;
    mat4 out;
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) out.c[col][row] = inv[col * 4 + row] * s;
    return out;
}

}  // namespace glm

#endif  // PXB_GLM_SHIM_GLM_HPP
