// nan_math.cuh -- device math of the path-integration kernels.
//
// The translation units that include this file are compiled with
// --fmad=false: every a*b+c below is an unfused multiply and add unless it is
// written as __fmaf_rn (the reference's explicit mad()). sqrtf and '/' are
// IEEE (no fast-math). With these rules the kernels evaluate the reference's
// Slang expressions (common.slang, scene.slang) in a fixed order:
//   dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z, vector sums left to right,
//   normalize(v) = v * (1/sqrt(dot(v,v))), lerp(a,b,s) = a + s*(b-a),
//   sin/cos from nan_sincos(), exp from nan_exp(), log2 from nan_log2() (own
//   Cody-Waite reductions and series, no libdevice).
#pragma once

#include <cstdint>

namespace nbd {

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ f3 abs3(f3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__device__ __forceinline__ float len3(f3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ f3 normalize3(f3 a) { return a * (1.0f / sqrtf(dot3(a, a))); }
__device__ __forceinline__ float maxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sat(float a) { return minf(maxf(a, 0.0f), 1.0f); }
__device__ __forceinline__ f3 ld3(const float* p) { return {__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvPi = 0.31830988618379067154f;

// sin and cos of a float angle: Cody-Waite reduction by pi/2 (two-part
// constant, fused) and the Taylor polynomials of sin (degree 9) and cos
// (degree 10) on |r| <= pi/4, evaluated by Horner's rule with fused steps.
__device__ __forceinline__ void nan_sincos(float a, float* s, float* c) {
    const float kf = rintf(a * 0.636619772367581343f);
    const int k = (int)kf;
    float r = __fmaf_rn(-kf, 1.57079637050628662109375f, a);
    r = __fmaf_rn(-kf, -4.37113900018624283e-8f, r);
    const float r2 = r * r;
    float ps = __fmaf_rn(r2, 2.75573192239858907e-6f, -1.98412698412698413e-4f);
    ps = __fmaf_rn(r2, ps, 8.33333333333333333e-3f);
    ps = __fmaf_rn(r2, ps, -1.66666666666666667e-1f);
    const float sn = __fmaf_rn(r * r2, ps, r);
    float pc = __fmaf_rn(r2, -2.75573192239858907e-7f, 2.48015873015873016e-5f);
    pc = __fmaf_rn(r2, pc, -1.38888888888888889e-3f);
    pc = __fmaf_rn(r2, pc, 4.16666666666666667e-2f);
    pc = __fmaf_rn(r2, pc, -0.5f);
    const float cs = __fmaf_rn(r2, pc, 1.0f);
    switch (k & 3) {
        case 0: *s = sn; *c = cs; break;
        case 1: *s = cs; *c = -sn; break;
        case 2: *s = -sn; *c = -cs; break;
        default: *s = -cs; *c = sn; break;
    }
}

// e^x: Cody-Waite reduction x = k ln2 + r with |r| <= ln2/2 (ln2 split in a
// 16-bit head and a tail, fused steps), e^r by its Taylor series to degree 7
// (truncation below 6e-9 relative) in Horner form, then 2^k applied as two
// exact power-of-two factors. Below -87.3 the result is 0, above 88.7 inf.
__device__ __forceinline__ float nan_exp(float x) {
    if (x != x) return x;
    if (x > 88.7f) return __int_as_float(0x7f800000);
    if (x < -87.3f) return 0.0f;
    const float kf = rintf(x * 1.44269504088896341f);
    const int k = (int)kf;
    float r = __fmaf_rn(-kf, 0.693145751953125f, x);
    r = __fmaf_rn(-kf, 1.428606820309417232e-6f, r);
    float p = __fmaf_rn(r, 1.98412698412698413e-4f, 1.38888888888888889e-3f);
    p = __fmaf_rn(r, p, 8.33333333333333333e-3f);
    p = __fmaf_rn(r, p, 4.16666666666666667e-2f);
    p = __fmaf_rn(r, p, 1.66666666666666667e-1f);
    p = __fmaf_rn(r, p, 0.5f);
    p = __fmaf_rn(r, p, 1.0f);
    p = __fmaf_rn(r, p, 1.0f);
    const int k1 = k >> 1, k2 = k - k1;
    return (p * __int_as_float((k1 + 127) << 23)) * __int_as_float((k2 + 127) << 23);
}

// log2(x): x = m 2^e with m in [sqrt(1/2), sqrt(2)], ln m = 2 atanh(s),
// s = (m-1)/(m+1), |s| <= 0.1716, by the odd series to s^11 (truncation below
// 1e-10), then e + ln m * log2(e). Subnormals are scaled by 2^23 first.
__device__ __forceinline__ float nan_log2(float x) {
    if (x != x || x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (x > 3.40282347e38f) return x;
    int e = 0;
    if (x < 1.17549435e-38f) {
        x = x * 8388608.0f;
        e = -23;
    }
    const uint32_t bits = __float_as_uint(x);
    e += (int)((bits >> 23) & 0xffu) - 127;
    float m = __uint_as_float((bits & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = __fmaf_rn(s2, 9.09090909090909091e-2f, 1.11111111111111111e-1f);
    p = __fmaf_rn(s2, p, 1.42857142857142857e-1f);
    p = __fmaf_rn(s2, p, 2.0e-1f);
    p = __fmaf_rn(s2, p, 3.33333333333333333e-1f);
    p = __fmaf_rn(s2, p, 1.0f);
    const float ln_m = (2.0f * s) * p;
    return (float)e + ln_m * 1.44269504088896341f;
}

// LCG of common.slang:164-210.
struct Rng {
    uint32_t state;
    __device__ __forceinline__ Rng(uint32_t x, uint32_t y, uint32_t sample_index)
        : state((x * 100591u) ^ (y * 102191u) ^ (sample_index * 103643u)) {}
    __device__ __forceinline__ float next_1d() {
        state = 1664525u * state + 1013904223u;
        return (float)(state >> 8) * 0x1p-24f;
    }
};

// Tangent frame of common.slang:139-162.
struct Frame {
    f3 n, t, b;
    __device__ __forceinline__ Frame() {}
    __device__ __forceinline__ explicit Frame(f3 nn) {
        n = nn;
        t = normalize3(cross3(nn, mk3(-nn.z, nn.x, -nn.y)));
        b = cross3(nn, t);
    }
    __device__ __forceinline__ f3 to_global(f3 w) const { return (w.x * t + w.y * b) + w.z * n; }
    __device__ __forceinline__ f3 to_local(f3 w) const { return mk3(dot3(t, w), dot3(b, w), dot3(n, w)); }
};

// common.slang:54-68; returns direction, writes pdf.
__device__ __forceinline__ f3 cosine_sample_hemisphere(float ex, float ey, float* pdf) {
    const float phi = (2.0f * kPi) * ex;
    const float cos_theta = sqrtf(ey);
    const float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
    float s, c;
    nan_sincos(phi, &s, &c);
    *pdf = cos_theta * (1.0f / kPi);
    return mk3(sin_theta * c, sin_theta * s, cos_theta);
}

// common.slang:452-470 (direction only; the pdf is unused on the path).
__device__ __forceinline__ f3 sample_cone_direction(f3 axis, float cos_half, float ux, float uy) {
    const float cos_theta = 1.0f - ux * (1.0f - cos_half);
    const float sin_theta = sqrtf(maxf(0.0f, 1.0f - cos_theta * cos_theta));
    const float phi = kTwoPi * uy;
    float s, c;
    nan_sincos(phi, &s, &c);
    return Frame(axis).to_global(mk3(c * sin_theta, s * sin_theta, cos_theta));
}

// common.slang:475-490 with HLSL reflect(i, n) = i - 2*dot(n, i)*n.
__device__ __forceinline__ f3 adjust_shading_normal(f3 sn, f3 gn, f3 d) {
    const f3 r = d - (2.0f * dot3(sn, d)) * sn;
    const float k = dot3(r, gn);
    if (k < 0.0f) return normalize3(normalize3(r - k * gn) - d);
    return sn;
}

// atan2 and asin of float arguments, from the mathematics: for
// t = min(|x|, |y|) / max(|x|, |y|) in [0, 1], two half-angle steps
// t -> t / (1 + sqrt(1 + t^2)) (atan t = 2 atan of the result) bring t below
// tan(pi/16) ~ 0.2, where the odd Taylor series of atan to t^15 (truncation
// below 1e-12) is summed by Horner's rule with fused steps; the octant and
// quadrant come from the signs. The oracle runs the same operations (C fmaf
// is correctly rounded too), so GPU and oracle agree bit for bit.
// asin x = atan2(x, sqrt(1 - x^2)).
__device__ __forceinline__ float nan_atan01(float t) {
    t = t / (1.0f + sqrtf(1.0f + t * t));
    t = t / (1.0f + sqrtf(1.0f + t * t));
    const float s = t * t;
    float p = -6.66666666666666667e-2f;
    p = __fmaf_rn(p, s, 7.69230769230769231e-2f);
    p = __fmaf_rn(p, s, -9.09090909090909091e-2f);
    p = __fmaf_rn(p, s, 1.11111111111111111e-1f);
    p = __fmaf_rn(p, s, -1.42857142857142857e-1f);
    p = __fmaf_rn(p, s, 2.0e-1f);
    p = __fmaf_rn(p, s, -3.33333333333333333e-1f);
    return 4.0f * __fmaf_rn(t * s, p, t);
}

__device__ __forceinline__ float nan_atan2(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    float a = mx > 0.0f ? nan_atan01(mn / mx) : 0.0f;
    if (ay > ax) a = 1.57079632679489662f - a;
    if (x < 0.0f) a = 3.14159265358979324f - a;
    return y < 0.0f ? -a : a;
}

__device__ __forceinline__ float nan_asin(float x) { return nan_atan2(x, sqrtf(fmaxf(0.0f, 1.0f - x * x))); }

}  // namespace nbd
