// Minimal stand-in for the parts of the glm vector-math library that
// libFluid's hot-path sources use (vec2/vec3 arithmetic, dot, length,
// normalize, isnan, any; vec4 and the r/g/b/a colour names for the image
// types of the tone mapper). Test infrastructure only: it lets the oracle build
// compile the reference solver sources unmodified.
//
// Arithmetic follows glm's scalar (non-SIMD) code path:
//   - component-wise + - * / in float, one IEEE rounding per operation;
//   - dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z  (left to right);
//   - length(v) = sqrt(dot(v, v)) with the float sqrt;
//   - normalize(v) = v * (1 / sqrt(dot(v, v))).
// The oracle is compiled with -ffp-contract=off so no FMA is formed.
#pragma once

// The real header pulls these in transitively; the reference sources rely on it.
#include <cassert>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>

namespace glm {

    struct bvec2 {
        bool x, y;
    };
    struct bvec3 {
        bool x, y, z;
    };

    struct vec2 {
        float x, y;
        vec2() = default;
        constexpr explicit vec2(float s) : x(s), y(s) {}
        constexpr vec2(float a, float b) : x(a), y(b) {}
        float& operator[](std::size_t i) { return i == 0 ? x : y; }
        const float& operator[](std::size_t i) const { return i == 0 ? x : y; }
        vec2& operator+=(const vec2& o) { x = x + o.x; y = y + o.y; return *this; }
        vec2& operator-=(const vec2& o) { x = x - o.x; y = y - o.y; return *this; }
        vec2& operator*=(float s) { x = x * s; y = y * s; return *this; }
        vec2& operator/=(float s) { x = x / s; y = y / s; return *this; }
    };

    struct vec3 {
        // r, g, b name the same components (glm's colour aliases)
        union { float x, r; };
        union { float y, g; };
        union { float z, b; };
        vec3() = default;
        constexpr explicit vec3(float s) : x(s), y(s), z(s) {}
        constexpr vec3(float a0, float a1, float a2) : x(a0), y(a1), z(a2) {}
        float& operator[](std::size_t i) { return i == 0 ? x : (i == 1 ? y : z); }
        const float& operator[](std::size_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
        vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
        vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
        vec3& operator*=(float s) { x = x * s; y = y * s; z = z * s; return *this; }
        vec3& operator/=(float s) { x = x / s; y = y / s; z = z / s; return *this; }
    };

    struct vec4 {
        union { float x, r; };
        union { float y, g; };
        union { float z, b; };
        union { float w, a; };
        vec4() = default;
        constexpr explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
        constexpr vec4(float a0, float a1, float a2, float a3) : x(a0), y(a1), z(a2), w(a3) {}
        constexpr vec4(const vec3& v, float a3) : x(v.x), y(v.y), z(v.z), w(a3) {}
    };

    // ---- vec2 ----
    inline vec2 operator+(const vec2& a, const vec2& b) { return vec2(a.x + b.x, a.y + b.y); }
    inline vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
    inline vec2 operator*(const vec2& a, const vec2& b) { return vec2(a.x * b.x, a.y * b.y); }
    inline vec2 operator/(const vec2& a, const vec2& b) { return vec2(a.x / b.x, a.y / b.y); }
    inline vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }
    inline vec2 operator*(float s, const vec2& a) { return vec2(s * a.x, s * a.y); }
    inline vec2 operator/(const vec2& a, float s) { return vec2(a.x / s, a.y / s); }
    inline vec2 operator/(float s, const vec2& a) { return vec2(s / a.x, s / a.y); }
    inline vec2 operator+(const vec2& a, float s) { return vec2(a.x + s, a.y + s); }
    inline vec2 operator-(const vec2& a, float s) { return vec2(a.x - s, a.y - s); }
    inline vec2 operator-(const vec2& a) { return vec2(-a.x, -a.y); }
    inline bool operator==(const vec2& a, const vec2& b) { return a.x == b.x && a.y == b.y; }
    inline bool operator!=(const vec2& a, const vec2& b) { return !(a == b); }

    // ---- vec3 ----
    inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
    inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
    inline vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
    inline vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
    inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
    inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
    inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
    inline vec3 operator/(float s, const vec3& a) { return vec3(s / a.x, s / a.y, s / a.z); }
    inline vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
    inline vec3 operator-(const vec3& a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
    inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
    inline bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
    inline bool operator!=(const vec3& a, const vec3& b) { return !(a == b); }

    inline float dot(const vec2& a, const vec2& b) {
        vec2 t = a * b;
        return t.x + t.y;
    }
    inline float dot(const vec3& a, const vec3& b) {
        vec3 t = a * b;
        return (t.x + t.y) + t.z;
    }
    inline float length(const vec2& v) { return std::sqrt(dot(v, v)); }
    inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
    inline vec2 normalize(const vec2& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
    inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
    inline bvec2 isnan(const vec2& v) { return {std::isnan(v.x), std::isnan(v.y)}; }
    inline bvec3 isnan(const vec3& v) { return {std::isnan(v.x), std::isnan(v.y), std::isnan(v.z)}; }
    inline bool any(const bvec2& b) { return b.x || b.y; }
    inline bool any(const bvec3& b) { return b.x || b.y || b.z; }

} // namespace glm
