/*
 * wgsl_prelude.h -- the WGSL types and builtins that the reference's compute
 * shaders use, as C++ (for the mechanical translation in oracle/_ref/).
 *
 * TEST INFRASTRUCTURE ONLY.  Semantics follow the WGSL specification for the
 * operations these shaders use: f32 IEEE arithmetic (compile with
 * -ffp-contract=off), u32(f32) truncation for in-range values,
 * countLeadingZeros(0) = 32, select(f, t, c) = c ? t : f, component-wise vec2
 * arithmetic, and inverseSqrt(x) = 1/sqrt(x) (WGSL allows 2 ULP; the oracle
 * uses the same correctly rounded form).  Atomics are plain read-modify-write:
 * the harness runs one invocation at a time.
 */
#pragma once

#include <array>
#include <cmath>
#include <cstdint>

namespace wgsl {

using u32 = uint32_t;
using i32 = int32_t;
using f32 = float;

struct vec2f {
    f32 x = 0.0f, y = 0.0f;
    vec2f() = default;
    explicit vec2f(f32 s) : x(s), y(s) {}
    vec2f(f32 a, f32 b) : x(a), y(b) {}
    vec2f& operator+=(const vec2f& o) { x = x + o.x; y = y + o.y; return *this; }
};
inline vec2f operator+(vec2f a, vec2f b) { return vec2f(a.x + b.x, a.y + b.y); }
inline vec2f operator-(vec2f a, vec2f b) { return vec2f(a.x - b.x, a.y - b.y); }
inline vec2f operator*(vec2f a, vec2f b) { return vec2f(a.x * b.x, a.y * b.y); }
inline vec2f operator/(vec2f a, vec2f b) { return vec2f(a.x / b.x, a.y / b.y); }
inline vec2f operator*(vec2f a, f32 s) { return vec2f(a.x * s, a.y * s); }
inline vec2f operator*(f32 s, vec2f a) { return vec2f(s * a.x, s * a.y); }
inline vec2f operator/(vec2f a, f32 s) { return vec2f(a.x / s, a.y / s); }

struct vec3u {
    u32 x = 0, y = 0, z = 0;
};

inline u32 countLeadingZeros(u32 v) { return v ? (u32)__builtin_clz(v) : 32u; }
template <typename T>
inline T select(T f, T t, bool c) { return c ? t : f; }
inline i32 min(i32 a, i32 b) { return a < b ? a : b; }
inline i32 max(i32 a, i32 b) { return a > b ? a : b; }
inline u32 min(u32 a, u32 b) { return a < b ? a : b; }
inline u32 max(u32 a, u32 b) { return a > b ? a : b; }
inline f32 min(f32 a, f32 b) { return std::fmin(a, b); }
inline f32 max(f32 a, f32 b) { return std::fmax(a, b); }
inline vec2f min(vec2f a, vec2f b) { return vec2f(min(a.x, b.x), min(a.y, b.y)); }
inline vec2f max(vec2f a, vec2f b) { return vec2f(max(a.x, b.x), max(a.y, b.y)); }
inline f32 clamp(f32 v, f32 lo, f32 hi) { return min(max(v, lo), hi); }
inline vec2f clamp(vec2f v, vec2f lo, vec2f hi) { return vec2f(clamp(v.x, lo.x, hi.x), clamp(v.y, lo.y, hi.y)); }
inline f32 dot(vec2f a, vec2f b) { return a.x * b.x + a.y * b.y; }
inline f32 sqrt(f32 v) { return std::sqrt(v); }
inline f32 inverseSqrt(f32 v) { return 1.0f / std::sqrt(v); }
inline u32 atomicAdd(u32* p, u32 v) { u32 old = *p; *p = old + v; return old; }

// ---- the render shaders' types and builtins (density.wgsl, tone_map.wgsl) ----
struct vec3f {
    f32 x = 0.0f, y = 0.0f, z = 0.0f;
    vec3f() = default;
    vec3f(f32 a, f32 b, f32 c) : x(a), y(b), z(c) {}
};
inline vec3f operator+(vec3f a, vec3f b) { return vec3f(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3f operator*(vec3f a, f32 s) { return vec3f(a.x * s, a.y * s, a.z * s); }
struct vec4f {
    f32 x = 0.0f, y = 0.0f, z = 0.0f, w = 0.0f;
    vec4f() = default;
    vec4f(f32 a, f32 b, f32 c, f32 d) : x(a), y(b), z(c), w(d) {}
    vec4f(vec2f a, f32 c, f32 d) : x(a.x), y(a.y), z(c), w(d) {}
    vec4f(vec3f a, f32 d) : x(a.x), y(a.y), z(a.z), w(d) {}
};
inline f32 length(vec2f v) { return std::sqrt(dot(v, v)); }
inline f32 exp(f32 v) { return std::exp(v); }
inline f32 pow(f32 a, f32 b) { return std::pow(a, b); }
// mix(e1, e2, t) = e1 * (1 - t) + e2 * t
inline vec3f mix(vec3f a, vec3f b, f32 t) { return a * (1.0f - t) + b * t; }
// A texture and a sampler: the harness sets the value a sample returns (the
// tone map samples its density texture at texel centres, i.e. a texel).
struct texture_2d {};
struct sampler {};
inline f32 g_texel = 0.0f;
inline vec4f textureSample(texture_2d, sampler, vec2f) { return vec4f(g_texel, 0.0f, 0.0f, 1.0f); }
// `discard` in a fragment shader: the harness reads this flag.
inline bool g_discarded = false;
inline void atomicStore(u32* p, u32 v) { *p = v; }

}  // namespace wgsl
