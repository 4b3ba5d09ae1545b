// glsl_shim.hpp — the small subset of GLSL 4.30 that the reference's compute
// shaders use, as C++ types and functions, so that the shader sources under
// resources/shaders/compute/ compile as C++ (after the mechanical rewrite in
// oracle/glsl/translate.py) and run on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  Arithmetic is single precision like GLSL
// `float`; signed overflow wraps (built with -fwrapv) like GLSL `int`.
// `texture()` on a sampler3D is exact trilinear filtering with
// clamp-to-edge addressing (the GL_LINEAR + CLAMP_TO_EDGE state set in
// src/opengl/Texture3D.cpp:25-32, without the hardware's fixed-point weights).
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>

namespace glsl {

typedef std::uint32_t uint;

struct vec2 { float x, y; };
struct vec3 { float x, y, z; };
struct ivec2 { int x, y; };
struct ivec3 { int x, y, z; };
struct uvec2 { uint x, y; };
struct uvec3 { uint x, y, z; };

#if defined(__GNUC__)
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wpedantic"
#endif
union vec4 {
    struct { float x, y, z, w; };
    struct { float r, g, b, a; };
    vec3 xyz;
};
#if defined(__GNUC__)
#pragma GCC diagnostic pop
#endif

// ---- constructors (GLSL `vec3(...)` is rewritten to `make_vec3(...)`) -----
inline vec3 make_vec3(float s) { return vec3{s, s, s}; }
inline vec3 make_vec3(float a, float b, float c) { return vec3{a, b, c}; }
inline vec3 make_vec3(ivec3 v) { return vec3{(float)v.x, (float)v.y, (float)v.z}; }
inline vec4 make_vec4(float s) { vec4 r; r.x = r.y = r.z = r.w = s; return r; }
inline vec4 make_vec4(vec3 v, float w) { vec4 r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = w; return r; }
inline vec4 make_vec4(float a, float b, float c, float d) { vec4 r; r.x = a; r.y = b; r.z = c; r.w = d; return r; }
inline ivec3 make_ivec3(vec3 v) { return ivec3{(int)v.x, (int)v.y, (int)v.z}; }
inline ivec3 make_ivec3(int a, int b, int c) { return ivec3{a, b, c}; }
inline ivec2 make_ivec2(int a, int b) { return ivec2{a, b}; }
inline uvec2 make_uvec2(uint a, uint b) { return uvec2{a, b}; }

// ---- vec3 arithmetic ------------------------------------------------------
inline vec3 operator+(vec3 a, vec3 b) { return vec3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(vec3 a, vec3 b) { return vec3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator-(vec3 a) { return vec3{-a.x, -a.y, -a.z}; }
inline vec3 operator*(vec3 a, float s) { return vec3{a.x * s, a.y * s, a.z * s}; }
inline vec3 operator*(float s, vec3 a) { return vec3{s * a.x, s * a.y, s * a.z}; }
inline vec3 operator*(vec3 a, vec3 b) { return vec3{a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3 operator/(vec3 a, float s) { return vec3{a.x / s, a.y / s, a.z / s}; }
inline vec3 operator/(vec3 a, vec3 b) { return vec3{a.x / b.x, a.y / b.y, a.z / b.z}; }
inline vec3 operator+(vec3 a, float s) { return vec3{a.x + s, a.y + s, a.z + s}; }
inline vec3& operator+=(vec3& a, vec3 b) { a = a + b; return a; }
inline vec3& operator-=(vec3& a, vec3 b) { a = a - b; return a; }
inline vec3& operator*=(vec3& a, float s) { a = a * s; return a; }
inline ivec3 operator+(ivec3 a, ivec3 b) { return ivec3{a.x + b.x, a.y + b.y, a.z + b.z}; }

// ---- built-in functions ---------------------------------------------------
inline float dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(vec3 a) { return std::sqrt(dot(a, a)); }
inline vec3 normalize(vec3 a) { return a / length(a); }
inline vec3 cross(vec3 a, vec3 b) { return vec3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline vec3 floor(vec3 a) { return vec3{std::floor(a.x), std::floor(a.y), std::floor(a.z)}; }
inline float floor(float a) { return std::floor(a); }
inline float sqrt(float a) { return std::sqrt(a); }
inline float abs(float a) { return std::fabs(a); }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float round(float a) { return std::nearbyint(a); }
inline float max(float a, float b) { return std::max(a, b); }
inline float min(float a, float b) { return std::min(a, b); }
inline uint max(uint a, uint b) { return std::max(a, b); }
inline uint min(uint a, uint b) { return std::min(a, b); }
inline float clamp(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
inline uint clamp(uint x, uint lo, uint hi) { return std::min(std::max(x, lo), hi); }
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline uint bitCount(uint v) { return (uint)__builtin_popcount(v); }

inline uint atomicAdd(uint& mem, uint v) { return __atomic_fetch_add(&mem, v, __ATOMIC_RELAXED); }
inline uint atomicOr(uint& mem, uint v) { return __atomic_fetch_or(&mem, v, __ATOMIC_RELAXED); }

// ---- sampler3D: R32F volume in GL order (x fastest) -------------------------
struct sampler3D {
    const float* texels = nullptr;
    int w = 0, h = 0, d = 0;
};

inline float texel(const sampler3D& s, int x, int y, int z)
{
    x = std::min(std::max(x, 0), s.w - 1);
    y = std::min(std::max(y, 0), s.h - 1);
    z = std::min(std::max(z, 0), s.d - 1);
    return s.texels[(long)x + (long)s.w * ((long)y + (long)s.h * z)];
}

// GL_LINEAR: u = tc*size - 0.5, weights from the fractional part, texel
// indices clamped to the edge.
inline vec4 texture(const sampler3D& s, vec3 tc)
{
    const float u = tc.x * (float)s.w - 0.5f;
    const float v = tc.y * (float)s.h - 0.5f;
    const float q = tc.z * (float)s.d - 0.5f;
    const float fu = std::floor(u), fv = std::floor(v), fq = std::floor(q);
    const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fq;
    const float a = u - fu, b = v - fv, c = q - fq;
    float cz[2][2];
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy) {
            const float t0 = texel(s, i0 + dx, j0 + dy, k0);
            const float t1 = texel(s, i0 + dx, j0 + dy, k0 + 1);
            cz[dx][dy] = t0 + (t1 - t0) * c;
        }
    const float c0 = cz[0][0] + (cz[0][1] - cz[0][0]) * b;
    const float c1 = cz[1][0] + (cz[1][1] - cz[1][0]) * b;
    return make_vec4(c0 + (c1 - c0) * a);
}

}  // namespace glsl
