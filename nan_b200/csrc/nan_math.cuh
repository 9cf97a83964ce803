// nan_math.cuh -- device math of the path-integration kernels.
//
// The translation units that include this file are compiled with
// --fmad=false: every a*b+c below is an unfused multiply and add unless it is
// written as __fmaf_rn (the reference's explicit mad()). sqrtf and '/' are
// IEEE (no fast-math). With these rules the kernels evaluate the reference's
// Slang expressions (common.slang, scene.slang) in a fixed order:
//   dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z, vector sums left to right,
//   normalize(v) = v * (1/sqrt(dot(v,v))), lerp(a,b,s) = a + s*(b-a),
//   sin/cos from nan_sincos() (own Cody-Waite + Taylor, no libdevice).
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

}  // namespace nbd
