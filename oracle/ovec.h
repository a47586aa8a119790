// Oracle (test infrastructure only): f32 vector arithmetic with the exact
// operation order of the reference's math layer.
//
// The reference (Rust crate `interflect` 0.1.3) does all vector math through
// `glam 0.33.6` (Cargo.lock:102-104), which is not vendored. Its scalar `Vec3`
// semantics are restated here from glam's published source:
//   dot       = (x*x' + y*y') + z*z'        (left to right, no FMA)
//   length    = sqrt(dot(v, v))
//   normalize = v * (1 / length(v))          (length_recip, then a multiply)
//   cross     = (y*z' - y'*z, z*x' - z'*x, x*y' - x'*y)
//   v / s     = per-component division
//   min / max = per-component Rust f32::min / f32::max (NaN-ignoring)
//   clamp     = max(lo).min(hi)
//   lerp      = a * (1 - s) + b * s
// rustc never contracts a*b+c into an FMA, so this file must be compiled with
// -ffp-contract=off and without -ffast-math. Every literal is an f32 literal.
//
// The scalar helpers below restate Rust's f32 semantics that differ from C:
// `f32::clamp`, `signum`, and the saturating float-to-int `as` casts.
#pragma once

#include <cmath>
#include <cstdint>
#include <climits>

namespace orc {

// Rust `f32::clamp` (core/src/num/f32.rs): compare-and-replace, NaN passes through.
static inline float clampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// Rust `f32::max` / `f32::min`: IEEE maxNum / minNum (the non-NaN operand wins).
static inline float fmaxr(float a, float b) { return std::fmax(a, b); }
static inline float fminr(float a, float b) { return std::fmin(a, b); }
// Rust `f32::signum`: NaN stays NaN, otherwise +-1 carrying the sign bit.
static inline float signumr(float x) {
    if (std::isnan(x)) return x;
    return std::copysign(1.0f, x);
}
// Rust `f32 as i32`: truncation toward zero, saturating, NaN -> 0.
static inline int32_t as_i32(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
// Rust `f32 as u32`.
static inline uint32_t as_u32(float x) {
    if (std::isnan(x) || x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return UINT32_MAX;
    return (uint32_t)x;
}
// Rust `f32 as usize` (64-bit target).
static inline uint64_t as_usize(float x) {
    if (std::isnan(x) || x <= 0.0f) return 0u;
    if (x >= 18446744073709551616.0f) return UINT64_MAX;
    return (uint64_t)x;
}
// Rust `f32 as u8`.
static inline uint8_t as_u8(float x) {
    if (std::isnan(x) || x <= 0.0f) return 0u;
    if (x >= 255.0f) return 255u;
    return (uint8_t)x;
}
static inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// std::f32::consts
static const float PI_F = 3.14159265358979323846f;
static const float TAU_F = 6.28318530717958647692f;

struct V3 {
    float x, y, z;
    V3() : x(0.0f), y(0.0f), z(0.0f) {}
    V3(float a, float b, float c) : x(a), y(b), z(c) {}
    static V3 splat(float s) { return V3(s, s, s); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

static inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator*(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 operator/(V3 a, V3 b) { return V3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline V3 operator*(V3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator/(V3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }

static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length_squared(V3 a) { return dot(a, a); }
static inline float length(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 normalize(V3 a) { return a * (1.0f / length(a)); }
static inline V3 cross(V3 a, V3 b) {
    return V3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline V3 vabs(V3 a) { return V3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
static inline V3 vmax(V3 a, V3 b) { return V3(fmaxr(a.x, b.x), fmaxr(a.y, b.y), fmaxr(a.z, b.z)); }
static inline V3 vmin(V3 a, V3 b) { return V3(fminr(a.x, b.x), fminr(a.y, b.y), fminr(a.z, b.z)); }
static inline V3 vclamp(V3 a, V3 lo, V3 hi) { return vmin(vmax(a, lo), hi); }
static inline float max_element(V3 a) { return fmaxr(a.x, fmaxr(a.y, a.z)); }
static inline float min_element(V3 a) { return fminr(a.x, fminr(a.y, a.z)); }
static inline V3 lerp(V3 a, V3 b, float s) { return a * (1.0f - s) + b * s; }
static inline bool any_lt(V3 a, V3 b) { return a.x < b.x || a.y < b.y || a.z < b.z; }
static inline bool any_gt(V3 a, V3 b) { return a.x > b.x || a.y > b.y || a.z > b.z; }

}  // namespace orc
