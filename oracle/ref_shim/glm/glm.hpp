/*
 * glm.hpp -- TEST INFRASTRUCTURE ONLY: a minimal stand-in for the parts of
 * glm (OpenGL Mathematics, github.com/g-truc/glm; the reference pulls it from
 * vcpkg, unpinned) that the reference headers compiled by oracle/Makefile's
 * `ref` target use.  glm itself is not installed here.  Written for this
 * repository from glm's documented semantics, with glm's evaluation orders
 * where they decide the bits:
 *   dot(a, b)      = (a.x*b.x + a.y*b.y) + a.z*b.z  (component products first)
 *   normalize(v)   = v * inversesqrt(dot(v, v)),  inversesqrt(x) = 1 / sqrt(x)
 *   min(x, y)      = (y < x) ? y : x,   max(x, y) = (x < y) ? y : x
 *   clamp(x, a, b) = min(max(x, a), b)
 *   abs(x)         = x >= 0 ? x : -x
 *   pow, sqrt, tan = the C library's float functions
 * Component-wise vector operators evaluate x, then y, then z.
 */
#pragma once

#include <cmath>
#include <cstdint>

namespace glm {

struct vec2 {
    float x, y;
    constexpr vec2() : x(0.0f), y(0.0f) {}
    explicit constexpr vec2(float s) : x(s), y(s) {}
    constexpr vec2(float a, float b) : x(a), y(b) {}
};

struct vec3 {
    float x, y, z;
    constexpr vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    explicit constexpr vec3(float s) : x(s), y(s), z(s) {}
    constexpr vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};

struct vec4 {
    float x, y, z, w;
    constexpr vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
    explicit constexpr vec4(float s) : x(s), y(s), z(s), w(s) {}
    constexpr vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};

struct uvec2 {
    uint32_t x, y;
    constexpr uvec2() : x(0u), y(0u) {}
    explicit constexpr uvec2(uint32_t s) : x(s), y(s) {}
    constexpr uvec2(uint32_t a, uint32_t b) : x(a), y(b) {}
};

// column-major 4x4 matrix; only held as data by the headers compiled here
struct mat4 {
    vec4 col[4];
    constexpr mat4() : col{vec4(1, 0, 0, 0), vec4(0, 1, 0, 0), vec4(0, 0, 1, 0), vec4(0, 0, 0, 1)} {}
};

constexpr vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
constexpr vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
constexpr vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
constexpr vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
constexpr vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
constexpr vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
constexpr vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
constexpr vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
constexpr vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
constexpr bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

constexpr vec2 operator+(const vec2& a, const vec2& b) { return vec2(a.x + b.x, a.y + b.y); }
constexpr vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
constexpr vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }

constexpr uvec2 operator+(const uvec2& a, const uvec2& b) { return uvec2(a.x + b.x, a.y + b.y); }
constexpr bool operator==(const uvec2& a, const uvec2& b) { return a.x == b.x && a.y == b.y; }
constexpr bool operator!=(const uvec2& a, const uvec2& b) { return !(a == b); }

constexpr float dot(const vec3& a, const vec3& b) {
    const vec3 t = a * b;
    return (t.x + t.y) + t.z;
}
constexpr float sqrt(float x) { return std::sqrt(x); }
constexpr float inversesqrt(float x) { return 1.0f / std::sqrt(x); }
constexpr vec3 normalize(const vec3& v) { return v * inversesqrt(dot(v, v)); }
constexpr float length(const vec3& v) { return std::sqrt(dot(v, v)); }
constexpr float abs(float x) { return x >= 0.0f ? x : -x; }
constexpr bool isnan(float x) { return std::isnan(x); }
constexpr bool isinf(float x) { return std::isinf(x); }
constexpr float min(float x, float y) { return (y < x) ? y : x; }
constexpr float max(float x, float y) { return (x < y) ? y : x; }
constexpr float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
constexpr float pow(float b, float e) { return std::pow(b, e); }
constexpr float tan(float x) { return std::tan(x); }
constexpr float radians(float deg) { return deg * 0.01745329251994329576923690768489f; }

}  // namespace glm
