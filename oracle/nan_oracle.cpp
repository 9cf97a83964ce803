// nan_oracle.cpp -- CPU restatement of the reference's path integration.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product): see
// nan_oracle.h. Citations are path:line inside the reference project.
//
// Arithmetic convention of the float "spec" mode (the Slang source leaves
// fusion and a few intrinsics to the driver; this fixes one reading of it):
//   * a*b+c written in Slang is an unfused multiply then add; only Slang's
//     explicit mad() is a fused multiply-add (fmaf);
//   * dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z; vector sums are left to right;
//   * normalize(v) = v * (1/sqrt(dot(v,v))), rsqrt(x) = 1/sqrt(x), both with
//     correctly rounded sqrt and division;
//   * lerp(a,b,s) = a + s*(b - a);
//   * sin/cos come from own_sincos() below (Cody-Waite reduction by pi/2 and
//     the Taylor polynomials of sin/cos), not from a math library, so the
//     CPU and GPU produce the same bits;
//   * floor(log2(x)) in the RGB9E5 pack is the exact binary exponent (frexp).
// Intersection is the watertight ray/triangle test of Woop, Benthin and Wald
// (JCGT 2013) against world-space triangles, with the closest hit chosen by
// (t, flat triangle index) so ties on shared edges resolve the same way in
// any traversal order.

#include "nan_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <array>
#include <cstring>
#include <limits>
#include <map>
#include <queue>
#include <set>
#include <tuple>
#include <unordered_map>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_error;

// ---------------------------------------------------------------------------
// Scalar operations per precision.
// ---------------------------------------------------------------------------

// sin/cos of a float angle by Cody-Waite reduction (two-part pi/2) and the
// degree-9 / degree-10 Taylor polynomials on |r| <= pi/4 (truncation error
// below 3e-9, under half an ulp of the result).
void own_sincos(float a, float* s, float* c) {
    const float two_over_pi = 0.636619772367581343f;
    const float pio2_hi = 1.57079637050628662109375f;
    const float pio2_lo = -4.37113900018624283e-8f;
    float kf = std::rint(a * two_over_pi);
    int k = (int)kf;
    float r = std::fmaf(-kf, pio2_hi, a);
    r = std::fmaf(-kf, pio2_lo, r);
    float r2 = r * r;
    float ps = std::fmaf(r2, 2.75573192239858907e-6f, -1.98412698412698413e-4f);
    ps = std::fmaf(r2, ps, 8.33333333333333333e-3f);
    ps = std::fmaf(r2, ps, -1.66666666666666667e-1f);
    float sn = std::fmaf(r * r2, ps, r);
    float pc = std::fmaf(r2, -2.75573192239858907e-7f, 2.48015873015873016e-5f);
    pc = std::fmaf(r2, pc, -1.38888888888888889e-3f);
    pc = std::fmaf(r2, pc, 4.16666666666666667e-2f);
    pc = std::fmaf(r2, pc, -0.5f);
    float cs = std::fmaf(r2, pc, 1.0f);
    switch (k & 3) {
        case 0: *s = sn; *c = cs; break;
        case 1: *s = cs; *c = -sn; break;
        case 2: *s = -sn; *c = -cs; break;
        default: *s = -cs; *c = sn; break;
    }
}

static float bits_float(uint32_t b) {
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

static uint32_t float_bits(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

// e^x by Cody-Waite reduction x = k ln2 + r (ln2 split in a 16-bit head and a
// tail), the Taylor series of e^r to degree 7 in Horner form, and 2^k as two
// exact power-of-two factors; 0 below -87.3, inf above 88.7.
float spec_exp(float x) {
    if (x != x) return x;
    if (x > 88.7f) return bits_float(0x7f800000u);
    if (x < -87.3f) return 0.0f;
    float kf = std::rint(x * 1.44269504088896341f);
    int k = (int)kf;
    float r = std::fmaf(-kf, 0.693145751953125f, x);
    r = std::fmaf(-kf, 1.428606820309417232e-6f, r);
    float p = std::fmaf(r, 1.98412698412698413e-4f, 1.38888888888888889e-3f);
    p = std::fmaf(r, p, 8.33333333333333333e-3f);
    p = std::fmaf(r, p, 4.16666666666666667e-2f);
    p = std::fmaf(r, p, 1.66666666666666667e-1f);
    p = std::fmaf(r, p, 0.5f);
    p = std::fmaf(r, p, 1.0f);
    p = std::fmaf(r, p, 1.0f);
    int k1 = k >> 1, k2 = k - k1;
    return (p * bits_float((uint32_t)(k1 + 127) << 23)) * bits_float((uint32_t)(k2 + 127) << 23);
}

// log2 x: x = m 2^e, m in [sqrt(1/2), sqrt(2)], ln m = 2 atanh((m-1)/(m+1)) by
// its odd series to s^11; subnormals scaled by 2^23 first.
float spec_log2(float x) {
    if (x != x || x < 0.0f) return bits_float(0x7fc00000u);
    if (x == 0.0f) return bits_float(0xff800000u);
    if (x > 3.40282347e38f) return x;
    int e = 0;
    if (x < 1.17549435e-38f) {
        x = x * 8388608.0f;
        e = -23;
    }
    uint32_t bits = float_bits(x);
    e += (int)((bits >> 23) & 0xffu) - 127;
    float m = bits_float((bits & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    float sv = (m - 1.0f) / (m + 1.0f);
    float s2 = sv * sv;
    float p = std::fmaf(s2, 9.09090909090909091e-2f, 1.11111111111111111e-1f);
    p = std::fmaf(s2, p, 1.42857142857142857e-1f);
    p = std::fmaf(s2, p, 2.0e-1f);
    p = std::fmaf(s2, p, 3.33333333333333333e-1f);
    p = std::fmaf(s2, p, 1.0f);
    float ln_m = (2.0f * sv) * p;
    return (float)e + ln_m * 1.44269504088896341f;
}

// atan2 / asin of floats: two half-angle steps t -> t / (1 + sqrt(1 + t^2))
// on t = min / max in [0, 1], the odd Taylor series of atan to t^15 by
// Horner's rule with fused steps, octant and quadrant from the signs; asin x
// = atan2(x, sqrt(1 - x^2)). The same operations as the kernels (nan_math.cuh).
float own_atan01(float t) {
    t = t / (1.0f + std::sqrt(1.0f + t * t));
    t = t / (1.0f + std::sqrt(1.0f + t * t));
    const float s = t * t;
    float p = -6.66666666666666667e-2f;
    p = std::fmaf(p, s, 7.69230769230769231e-2f);
    p = std::fmaf(p, s, -9.09090909090909091e-2f);
    p = std::fmaf(p, s, 1.11111111111111111e-1f);
    p = std::fmaf(p, s, -1.42857142857142857e-1f);
    p = std::fmaf(p, s, 2.0e-1f);
    p = std::fmaf(p, s, -3.33333333333333333e-1f);
    return 4.0f * std::fmaf(t * s, p, t);
}

float own_atan2(float y, float x) {
    const float ax = std::fabs(x), ay = std::fabs(y);
    const float mx = std::fmax(ax, ay), mn = std::fmin(ax, ay);
    float a = mx > 0.0f ? own_atan01(mn / mx) : 0.0f;
    if (ay > ax) a = 1.57079632679489662f - a;
    if (x < 0.0f) a = 3.14159265358979324f - a;
    return y < 0.0f ? -a : a;
}

float own_asin(float x) { return own_atan2(x, std::sqrt(std::fmax(0.0f, 1.0f - x * x))); }

template <class T> struct Ops;
template <> struct Ops<float> {
    static float fma(float a, float b, float c) { return std::fmaf(a, b, c); }
    static float sqrt(float a) { return std::sqrt(a); }
    static void sincos(float a, float* s, float* c) { own_sincos(a, s, c); }
    static float atan2(float y, float x) { return own_atan2(y, x); }
    static float asin(float x) { return own_asin(x); }
};
template <> struct Ops<double> {
    static double fma(double a, double b, double c) { return std::fma(a, b, c); }
    static double sqrt(double a) { return std::sqrt(a); }
    static double atan2(double y, double x) { return std::atan2(y, x); }
    static double asin(double x) { return std::asin(std::fmax(-1.0, std::fmin(1.0, x))); }
    static void sincos(double a, double* s, double* c) {
        *s = std::sin(a);
        *c = std::cos(a);
    }
};

template <class T> struct V3 {
    T x, y, z;
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> V3<T> vabs(V3<T> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
template <class T> T length(V3<T> a) { return Ops<T>::sqrt(dot(a, a)); }
template <class T> V3<T> normalize(V3<T> a) { return a * (T(1) / Ops<T>::sqrt(dot(a, a))); }
template <class T> T vmax(T a, T b) { return a > b ? a : b; }  // HLSL max for non-NaN
template <class T> T vmin(T a, T b) { return a < b ? a : b; }
template <class T> T saturate(T a) { return vmin(vmax(a, T(0)), T(1)); }

template <class T> struct Consts;
template <> struct Consts<float> {
    static constexpr float PI = 3.14159265358979323846f;
    static constexpr float TWO_PI = 6.28318530717958647692f;
    static constexpr float INV_PI = 0.31830988618379067154f;
};
template <> struct Consts<double> {
    static constexpr double PI = 3.14159265358979323846;
    static constexpr double TWO_PI = 6.28318530717958647692;
    static constexpr double INV_PI = 0.31830988618379067154;
};

// ---------------------------------------------------------------------------
// RNG: common.slang:164-210 (LCG, not PCG).
// ---------------------------------------------------------------------------
struct Rng {
    uint32_t state;
    Rng(uint32_t x, uint32_t y, uint32_t sample_index)
        : state((x * 100591u) ^ (y * 102191u) ^ (sample_index * 103643u)) {}
    uint32_t next() {
        state = 1664525u * state + 1013904223u;
        return state;
    }
    float next_1d() { return (float)(next() >> 8) * 0x1p-24f; }
};

// ---------------------------------------------------------------------------
// Sampling and frames: common.slang:54-68, 139-162, 452-470, 475-490.
// ---------------------------------------------------------------------------
template <class T> struct Frame {
    V3<T> n, t, b;
    explicit Frame(V3<T> nn) {  // common.slang:145-151 (Spencer & Jones eq. 3)
        n = nn;
        t = normalize(cross(nn, mk<T>(-nn.z, nn.x, -nn.y)));
        b = cross(nn, t);
    }
    V3<T> to_local(V3<T> w) const { return {dot(t, w), dot(b, w), dot(n, w)}; }
    V3<T> to_global(V3<T> w) const { return (w.x * t + w.y * b) + w.z * n; }
};

// common.slang:54-68
template <class T> void cosine_sample_hemisphere(T ex, T ey, V3<T>* h, T* pdf) {
    T phi = T(2) * Consts<T>::PI * ex;
    T cos_theta = Ops<T>::sqrt(ey);
    T sin_theta = Ops<T>::sqrt(T(1) - cos_theta * cos_theta);
    T s, c;
    Ops<T>::sincos(phi, &s, &c);
    *h = mk<T>(sin_theta * c, sin_theta * s, cos_theta);
    *pdf = cos_theta * (T(1) / Consts<T>::PI);
}

// common.slang:452-470
template <class T> V3<T> sample_cone_direction(V3<T> axis, T cos_half, T ux, T uy) {
    T cos_theta = T(1) - ux * (T(1) - cos_half);
    T sin_theta = Ops<T>::sqrt(vmax(T(0), T(1) - cos_theta * cos_theta));
    T phi = Consts<T>::TWO_PI * uy;
    T s, c;
    Ops<T>::sincos(phi, &s, &c);
    V3<T> local = mk<T>(c * sin_theta, s * sin_theta, cos_theta);
    return Frame<T>(axis).to_global(local);
}

// HLSL reflect(i, n) = i - 2*dot(n, i)*n
template <class T> V3<T> reflect(V3<T> i, V3<T> n) { return i - (T(2) * dot(n, i)) * n; }

// common.slang:475-490
template <class T> V3<T> adjust_shading_normal(V3<T> sn, V3<T> gn, V3<T> d) {
    V3<T> r = reflect(d, sn);
    T k = dot(r, gn);
    if (k < T(0)) return normalize(normalize(r - k * gn) - d);
    return sn;
}

// ---------------------------------------------------------------------------
// RGB9E5: mesh_colors.slang:218-253.
// ---------------------------------------------------------------------------
uint32_t pack_rgb9e5(float r, float g, float b) {
    const float kMax = 65408.0f;
    float v[3] = {std::isnan(r) ? 0.0f : r, std::isnan(g) ? 0.0f : g, std::isnan(b) ? 0.0f : b};
    for (float& x : v) x = std::min(std::max(x, 0.0f), kMax);
    float m = std::max(v[0], std::max(v[1], v[2]));
    if (m < 0x1p-25f) return 0;
    int e2 = 0;
    std::frexp(m, &e2);  // m = f * 2^e2, f in [0.5, 1): floor(log2 m) = e2 - 1
    int exponent = std::max(-15, e2);
    uint32_t shared = (uint32_t)(exponent + 15);
    float scale = std::ldexp(1.0f, (int)shared - 24);
    uint32_t mant[3];
    for (int i = 0; i < 3; ++i) mant[i] = (uint32_t)std::floor(v[i] / scale + 0.5f);
    if (std::max(mant[0], std::max(mant[1], mant[2])) == 512u && shared < 31u) {
        shared += 1;
        scale *= 2.0f;
        for (int i = 0; i < 3; ++i) mant[i] = (uint32_t)std::floor(v[i] / scale + 0.5f);
    }
    for (int i = 0; i < 3; ++i) mant[i] = std::min(mant[i], 511u);
    return mant[0] | (mant[1] << 9) | (mant[2] << 18) | (shared << 27);
}

void unpack_rgb9e5(uint32_t p, float* out) {
    float scale = std::ldexp(1.0f, (int)(p >> 27) - 24);
    out[0] = (float)(p & 0x1ffu) * scale;
    out[1] = (float)((p >> 9) & 0x1ffu) * scale;
    out[2] = (float)((p >> 18) & 0x1ffu) * scale;
}

// IEEE binary32 -> binary16, round to nearest even (f32tof16 in
// surface_probes.slang:84-96).
uint16_t f32_to_f16(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // >= 65520 rounds to inf
    if (ax < 0x38800000u) {  // below the smallest normal half: subnormal or zero
        if (ax < 0x33000000u) return (uint16_t)sign;  // < 2^-25 rounds to zero
        uint32_t e = ax >> 23;
        uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        uint32_t shift = 126u - e;  // value = m * 2^(e-150); half subnormal unit 2^-24
        uint32_t q = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (q & 1u))) q += 1;
        return (uint16_t)(sign | q);
    }
    uint32_t e = (ax >> 23) - 112u;  // rebias 127 -> 15
    uint32_t m = ax & 0x7fffffu;
    uint32_t q = (e << 10) | (m >> 13);
    uint32_t rem = m & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q += 1;  // carry may bump the exponent
    return (uint16_t)(sign | q);
}

float f16_to_f32(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1fu;
    uint32_t m = h & 0x3ffu;
    uint32_t bits;
    if (e == 0) {
        if (m == 0) {
            bits = sign;
        } else {
            float v = (float)m * 0x1p-24f;
            std::memcpy(&bits, &v, 4);
            bits |= sign;
        }
    } else if (e == 31) {
        bits = sign | 0x7f800000u | (m << 13);
    } else {
        bits = sign | ((e + 112u) << 23) | (m << 13);
    }
    float out;
    std::memcpy(&out, &bits, 4);
    return out;
}

// ---------------------------------------------------------------------------
// Hemi-oct mapping: surface_probes.slang:134-167.
// ---------------------------------------------------------------------------
void hemi_oct_encode(float dx, float dy, float dz, float* u, float* v) {
    V3<float> h = mk<float>(dx, dy, vmax(dz, 0.0f));
    float l2 = dot(h, h);
    if (l2 <= 1e-12f) {
        *u = 0.5f;
        *v = 0.5f;
        return;
    }
    h = h * (1.0f / std::sqrt(l2));
    float inv_l1 = 1.0f / vmax((std::fabs(h.x) + std::fabs(h.y)) + h.z, 1e-6f);
    float ox = h.x * inv_l1, oy = h.y * inv_l1;
    float sx = ox + oy, sy = ox - oy;
    *u = saturate(sx * 0.5f + 0.5f);
    *v = saturate(sy * 0.5f + 0.5f);
}

// Inverse of the encode above (the decode the reference's round-trip test
// uses): rotate back by 45 degrees and unfold the L1 diamond.
void hemi_oct_decode(float u, float v, float* out) {
    double sx = 2.0 * u - 1.0, sy = 2.0 * v - 1.0;
    double ox = 0.5 * (sx + sy), oy = 0.5 * (sx - sy);
    double oz = 1.0 - std::fabs(ox) - std::fabs(oy);
    if (oz < 0.0) oz = 0.0;
    double len = std::sqrt(ox * ox + oy * oy + oz * oz);
    out[0] = (float)(ox / len);
    out[1] = (float)(oy / len);
    out[2] = (float)(oz / len);
}

uint32_t radial_texel_index(float u, float v) {  // surface_probes.slang:157-167
    uint32_t x = std::min((uint32_t)(saturate(u) * 4.0f), 3u);
    uint32_t y = std::min((uint32_t)(saturate(v) * 4.0f), 3u);
    return y * 4u + x;
}

// surface_probe_path_tracer.slang:95-109
float radial_texel_cosine_probability(uint32_t texel) {
    uint32_t cx = texel % 4u, cy = texel / 4u;
    bool hb = cx == 0u || cx == 3u;
    bool vb = cy == 0u || cy == 3u;
    if (hb && vb) return 0.02221812f;
    if (hb || vb) return 0.06578385f;
    return 0.09621418f;
}

// ---------------------------------------------------------------------------
// Mesh Colors lattice: mesh_colors.slang:37-65, 272-363.
// ---------------------------------------------------------------------------
struct FaceInfo { uint32_t address, resolution; };
struct InstInfo { uint32_t face_offset, face_count, texel_offset, texel_count; };

uint32_t patch_texel_count(uint32_t r) { return (r + 1u) * (r + 2u) / 2u; }

uint32_t mc_address(uint32_t i, uint32_t j, const InstInfo& inst, const FaceInfo& f) {
    uint32_t row = i * (f.resolution + 1u) - i * (i - 1u) / 2u;
    return inst.texel_offset + f.address + row + j;
}

void address_to_ij(uint32_t address, uint32_t r, uint32_t* oi, uint32_t* oj) {
    uint32_t left = 0, right = r;
    while (left < right) {
        uint32_t mid = (left + right + 1u) / 2u;
        uint32_t ma = mid * (r + 1u) - mid * (mid - 1u) / 2u;
        if (ma <= address) left = mid; else right = mid - 1u;
    }
    uint32_t cum = left * (r + 1u) - left * (left - 1u) / 2u;
    *oi = left;
    *oj = address - cum;
}

bool find_face(const uint32_t* face_infos, const InstInfo& inst, uint32_t texel,
               FaceInfo* out, uint32_t* prim) {
    out->address = 0;
    out->resolution = 1;
    *prim = 0;
    int left = (int)inst.face_offset;
    int right = (int)(inst.face_offset + inst.face_count) - 1;
    while (left <= right) {
        int mid = (left + right) / 2;
        out->address = face_infos[2 * mid];
        out->resolution = face_infos[2 * mid + 1];
        int local = (int)texel - (int)out->address;
        int count = (int)patch_texel_count(out->resolution);
        if (local < 0) right = mid - 1;
        else if (local >= count) left = mid + 1;
        else {
            *prim = (uint32_t)mid - inst.face_offset;
            return true;
        }
    }
    return false;
}

float frac(float x) { return x - std::floor(x); }

uint32_t nearest_texel(float b0, float b1, float b2, const InstInfo& inst, const FaceInfo& f) {
    float rf = (float)f.resolution;
    float s0 = saturate(b0) * rf, s1 = saturate(b1) * rf, s2 = saturate(b2) * rf;
    uint32_t i = (uint32_t)s0, j = (uint32_t)s1;
    i = std::min(i, f.resolution);
    j = std::min(j, f.resolution - i);
    float w0 = frac(s0), w1 = frac(s1), w2 = frac(s2);
    bool upper = std::fabs(((w0 + w1) + w2) - 2.0f) <= 1e-3f;
    if (upper) { w0 = 1.0f - w0; w1 = 1.0f - w1; w2 = 1.0f - w2; }
    if ((w0 + w1) + w2 <= 1e-6f || i >= f.resolution || j >= f.resolution - i)
        return mc_address(i, j, inst, f);
    float largest = vmax(w0, vmax(w1, w2));
    if (upper) {
        if (std::fabs(largest - w0) < 1e-3f) return mc_address(i, j + 1u, inst, f);
        if (std::fabs(largest - w1) < 1e-3f) return mc_address(i + 1u, j, inst, f);
        return mc_address(i + 1u, j + 1u, inst, f);
    }
    if (std::fabs(largest - w0) < 1e-3f) return mc_address(i + 1u, j, inst, f);
    if (std::fabs(largest - w1) < 1e-3f) return mc_address(i, j + 1u, inst, f);
    return mc_address(i, j, inst, f);
}

// ---------------------------------------------------------------------------
// Scene: flattened world-space triangles + binned-SAH BVH (8 bins, the
// tinybvh BVH::Build heuristic: centroid bins, half-area SAH, C_trav = C_int
// = 1, split only while cheaper than a leaf).
// ---------------------------------------------------------------------------
struct Box {
    float lo[3], hi[3];
    void reset() {
        for (int a = 0; a < 3; ++a) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    float half_area() const {
        float e0 = hi[0] - lo[0], e1 = hi[1] - lo[1], e2 = hi[2] - lo[2];
        if (e0 < 0 || e1 < 0 || e2 < 0) return 0.0f;
        return e0 * e1 + e1 * e2 + e2 * e0;
    }
};

struct BvhNode {
    Box box;
    uint32_t left_first;  // first child index (interior) or first prim (leaf)
    uint32_t count;       // 0 for interior
};

struct Scene {
    std::vector<float> vertices;
    std::vector<uint32_t> indices, mesh_descs, instance_descs;
    std::vector<float> transforms, inv_transposes, materials;
    std::vector<uint32_t> flat_instance, flat_prim, instance_first_flat;
    std::vector<float> world_f;   // [T][9] float world triangles
    std::vector<double> world_d;  // [T][9] double world triangles
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> prim_order;
    std::vector<float> lights;  // area lights f32[L][16] (oracle_scene_set_area_lights)
    float light_power = 0.0f;
    float pad = 0.0f;
    uint32_t tri_count() const { return (uint32_t)flat_instance.size(); }
};

// mul(M, float4(p, 1)).xyz, unfused left to right.
template <class T> V3<T> xform_point(const float* m, V3<T> p) {
    return {((T(m[0]) * p.x + T(m[1]) * p.y) + T(m[2]) * p.z) + T(m[3]),
            ((T(m[4]) * p.x + T(m[5]) * p.y) + T(m[6]) * p.z) + T(m[7]),
            ((T(m[8]) * p.x + T(m[9]) * p.y) + T(m[10]) * p.z) + T(m[11])};
}

void build_bvh(Scene& s) {
    uint32_t n = s.tri_count();
    std::vector<Box> boxes(n);
    std::vector<float> cent(3 * (size_t)n);
    Box root;
    root.reset();
    float max_abs = 0.0f;
    for (uint32_t t = 0; t < n; ++t) {
        boxes[t].reset();
        for (int k = 0; k < 3; ++k) {
            const float* p = &s.world_f[9 * (size_t)t + 3 * k];
            boxes[t].grow(p);
            for (int a = 0; a < 3; ++a) max_abs = std::max(max_abs, std::fabs(p[a]));
        }
        for (int a = 0; a < 3; ++a) cent[3 * (size_t)t + a] = (boxes[t].lo[a] + boxes[t].hi[a]) * 0.5f;
        root.grow(boxes[t]);
    }
    s.pad = max_abs * 1e-5f + 1e-20f;
    s.prim_order.resize(n);
    for (uint32_t i = 0; i < n; ++i) s.prim_order[i] = i;
    s.nodes.clear();
    s.nodes.reserve(2 * (size_t)n + 1);
    BvhNode r;
    r.box = root;
    r.left_first = 0;
    r.count = n;
    s.nodes.push_back(r);
    std::vector<uint32_t> stack{0};
    const int B = 8;
    while (!stack.empty()) {
        uint32_t ni = stack.back();
        stack.pop_back();
        BvhNode node = s.nodes[ni];
        float sa = node.box.half_area();
        if (node.count <= 1 || sa <= 0.0f) continue;
        Box cb;
        cb.reset();
        for (uint32_t i = 0; i < node.count; ++i) cb.grow(&cent[3 * (size_t)s.prim_order[node.left_first + i]]);
        float best_cost = INFINITY;
        int best_axis = -1, best_pos = 0;
        float best_scale = 0.0f, best_min = 0.0f;
        for (int a = 0; a < 3; ++a) {
            float ext = cb.hi[a] - cb.lo[a];
            if (!(ext > 0.0f)) continue;
            float scale = (float)B / ext;
            Box bins[B];
            uint32_t cnt[B] = {0};
            for (int b = 0; b < B; ++b) bins[b].reset();
            for (uint32_t i = 0; i < node.count; ++i) {
                uint32_t p = s.prim_order[node.left_first + i];
                int bi = (int)((cent[3 * (size_t)p + a] - cb.lo[a]) * scale);
                bi = std::min(std::max(bi, 0), B - 1);
                bins[bi].grow(boxes[p]);
                cnt[bi]++;
            }
            float left_area[B - 1], right_area[B - 1];
            uint32_t left_n[B - 1], right_n[B - 1];
            Box lb, rb;
            lb.reset();
            rb.reset();
            uint32_t ln = 0, rn = 0;
            for (int i = 0; i < B - 1; ++i) {
                lb.grow(bins[i]);
                ln += cnt[i];
                left_area[i] = lb.half_area();
                left_n[i] = ln;
                rb.grow(bins[B - 1 - i]);
                rn += cnt[B - 1 - i];
                right_area[B - 2 - i] = rb.half_area();
                right_n[B - 2 - i] = rn;
            }
            for (int i = 0; i < B - 1; ++i) {
                if (left_n[i] == 0 || right_n[i] == 0) continue;
                float c = left_area[i] * (float)left_n[i] + right_area[i] * (float)right_n[i];
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_pos = i;
                    best_scale = scale;
                    best_min = cb.lo[a];
                }
            }
        }
        if (best_axis < 0) continue;
        float split_cost = 1.0f + best_cost / sa;
        if (split_cost >= (float)node.count) continue;
        uint32_t i = node.left_first, j = node.left_first + node.count;
        while (i < j) {
            uint32_t p = s.prim_order[i];
            int bi = (int)((cent[3 * (size_t)p + best_axis] - best_min) * best_scale);
            bi = std::min(std::max(bi, 0), B - 1);
            if (bi <= best_pos) ++i;
            else std::swap(s.prim_order[i], s.prim_order[--j]);
        }
        uint32_t left_count = i - node.left_first;
        if (left_count == 0 || left_count == node.count) continue;
        uint32_t c0 = (uint32_t)s.nodes.size();
        BvhNode L, R;
        L.left_first = node.left_first;
        L.count = left_count;
        R.left_first = i;
        R.count = node.count - left_count;
        L.box.reset();
        R.box.reset();
        for (uint32_t k = 0; k < L.count; ++k) L.box.grow(boxes[s.prim_order[L.left_first + k]]);
        for (uint32_t k = 0; k < R.count; ++k) R.box.grow(boxes[s.prim_order[R.left_first + k]]);
        s.nodes.push_back(L);
        s.nodes.push_back(R);
        s.nodes[ni].left_first = c0;
        s.nodes[ni].count = 0;
        stack.push_back(c0);
        stack.push_back(c0 + 1);
    }
}

// ---------------------------------------------------------------------------
// Watertight ray/triangle test (Woop, Benthin, Wald 2013).
// ---------------------------------------------------------------------------
template <class T> struct RayPre {
    V3<T> o, d;
    T tmin, tmax;
    int kx, ky, kz;
    T sx, sy, sz;
};

template <class T> RayPre<T> make_ray(V3<T> o, V3<T> d, T tmin, T tmax) {
    RayPre<T> r;
    r.o = o;
    r.d = d;
    r.tmin = tmin;
    r.tmax = tmax;
    T a[3] = {std::fabs(d.x), std::fabs(d.y), std::fabs(d.z)};
    int kz = 0;
    if (a[1] > a[kz]) kz = 1;
    if (a[2] > a[kz]) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (d[kz] < T(0)) std::swap(kx, ky);
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.sx = d[kx] / d[kz];
    r.sy = d[ky] / d[kz];
    r.sz = T(1) / d[kz];
    return r;
}

// Returns true with t, b1 (weight of v1), b2 (weight of v2) when the ray
// crosses the triangle's interior or edges (no culling); range not checked.
template <class T> bool tri_intersect(const RayPre<T>& r, const T* v, T* t_out, T* b1, T* b2) {
    V3<T> A = mk<T>(v[0], v[1], v[2]) - r.o;
    V3<T> B = mk<T>(v[3], v[4], v[5]) - r.o;
    V3<T> C = mk<T>(v[6], v[7], v[8]) - r.o;
    T ax = A[r.kx] - r.sx * A[r.kz];
    T ay = A[r.ky] - r.sy * A[r.kz];
    T bx = B[r.kx] - r.sx * B[r.kz];
    T by = B[r.ky] - r.sy * B[r.kz];
    T cx = C[r.kx] - r.sx * C[r.kz];
    T cy = C[r.ky] - r.sy * C[r.kz];
    T U = cx * by - cy * bx;
    T V = ax * cy - ay * cx;
    T W = bx * ay - by * ax;
    if (sizeof(T) == 4 && (U == T(0) || V == T(0) || W == T(0))) {
        U = (T)((double)cx * (double)by - (double)cy * (double)bx);
        V = (T)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (T)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < T(0) || V < T(0) || W < T(0)) && (U > T(0) || V > T(0) || W > T(0))) return false;
    T det = (U + V) + W;
    if (det == T(0)) return false;
    T az = r.sz * A[r.kz];
    T bz = r.sz * B[r.kz];
    T cz = r.sz * C[r.kz];
    T tt = (U * az + V * bz) + W * cz;
    *t_out = tt / det;
    *b1 = V / det;
    *b2 = W / det;
    return true;
}

struct HitRec {
    bool valid = false;
    uint32_t flat = 0xffffffffu;
    double t = 0.0;
    double b1 = 0.0, b2 = 0.0;
};

// Conservative slab test in double precision against the padded box.
bool box_hit(const Box& b, float pad, const double* o, const double* id, double tmin, double tmax,
             double* tenter) {
    double t0 = tmin, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        double lo = (double)b.lo[a] - pad, hi = (double)b.hi[a] + pad;
        double ta = (lo - o[a]) * id[a];
        double tb = (hi - o[a]) * id[a];
        if (std::isnan(ta) || std::isnan(tb)) { ta = -INFINITY; tb = INFINITY; }
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
    }
    *tenter = t0;
    return t0 <= t1;
}

template <class T> const T* tri_ptr(const Scene& s, uint32_t flat);
template <> const float* tri_ptr<float>(const Scene& s, uint32_t flat) { return &s.world_f[9 * (size_t)flat]; }
template <> const double* tri_ptr<double>(const Scene& s, uint32_t flat) { return &s.world_d[9 * (size_t)flat]; }

// mode: 0 BVH, otherwise brute force. any: stop at the first hit in range.
template <class T>
HitRec trace(const Scene& s, const RayPre<T>& r, bool any, bool use_bvh, OracleRayCounts* cnt) {
    HitRec best;
    T best_t = r.tmax;
    uint32_t best_key = 0xffffffffu;
    T best_b1 = 0, best_b2 = 0;
    auto test = [&](uint32_t flat) -> bool {
        if (cnt) cnt->triangle_tests++;
        T t, b1, b2;
        if (!tri_intersect<T>(r, tri_ptr<T>(s, flat), &t, &b1, &b2)) return false;
        if (!(t >= r.tmin)) return false;
        if (any) {
            if (t <= r.tmax) {
                best.valid = true;
                best.flat = flat;
                best.t = (double)t;
                return true;
            }
            return false;
        }
        if (t < best_t || (t == best_t && flat < best_key)) {
            best.valid = true;
            best_t = t;
            best_key = flat;
            best_b1 = b1;
            best_b2 = b2;
        }
        return false;
    };
    if (!use_bvh) {
        for (uint32_t f = 0; f < s.tri_count(); ++f)
            if (test(f)) return best;
    } else {
        double o[3] = {(double)r.o.x, (double)r.o.y, (double)r.o.z};
        double id[3] = {1.0 / (double)r.d.x, 1.0 / (double)r.d.y, 1.0 / (double)r.d.z};
        uint32_t stack[128];
        int sp = 0;
        double te;
        if (cnt) cnt->node_fetches++;
        if (box_hit(s.nodes[0].box, s.pad, o, id, (double)r.tmin, (double)r.tmax, &te)) stack[sp++] = 0;
        while (sp > 0) {
            const BvhNode& n = s.nodes[stack[--sp]];
            if (n.count > 0) {
                for (uint32_t k = 0; k < n.count; ++k)
                    if (test(s.prim_order[n.left_first + k])) return best;
                continue;
            }
            double limit = any ? (double)r.tmax : (double)best_t;
            double t0, t1;
            if (cnt) cnt->node_fetches += 2;
            bool h0 = box_hit(s.nodes[n.left_first].box, s.pad, o, id, (double)r.tmin, limit, &t0);
            bool h1 = box_hit(s.nodes[n.left_first + 1].box, s.pad, o, id, (double)r.tmin, limit, &t1);
            uint32_t c0 = n.left_first, c1 = n.left_first + 1;
            if (h0 && h1) {
                if (t1 < t0) { std::swap(c0, c1); }
                stack[sp++] = c1;  // far
                stack[sp++] = c0;  // near (popped first)
            } else if (h0) {
                stack[sp++] = c0;
            } else if (h1) {
                stack[sp++] = c1;
            }
            if (sp > 126) { g_error = "oracle BVH stack overflow"; return best; }
        }
    }
    if (!any && best.valid) {
        best.flat = best_key;
        best.t = (double)best_t;
        best.b1 = (double)best_b1;
        best.b2 = (double)best_b2;
    }
    return best;
}

// ---------------------------------------------------------------------------
// Shading: scene.slang:178-406.
// ---------------------------------------------------------------------------
struct Lighting {
    OracleLighting p;
};

template <class T> struct Shading {
    V3<T> position, origin_front, origin_back;
    T offset;
    V3<T> view_direction, face_normal, diffuse, emissive;
    Frame<T> shading_frame{mk<T>(0, 0, 1)};
    bool back_side = false;  // double-sided material seen from its back
};

template <class T> V3<T> load3(const float* p) { return mk<T>(T(p[0]), T(p[1]), T(p[2])); }

struct TriRefs {
    const float* v0;
    const float* v1;
    const float* v2;
    const float* m;
    const float* it;
    const float* mat;
    uint32_t flags;
};

TriRefs tri_refs(const Scene& s, uint32_t inst, uint32_t prim) {
    const uint32_t* idesc = &s.instance_descs[4 * (size_t)inst];
    const uint32_t* mdesc = &s.mesh_descs[4 * (size_t)idesc[0]];
    uint32_t base = mdesc[3] + prim * 3u;
    TriRefs r;
    r.v0 = &s.vertices[8 * (size_t)(mdesc[2] + s.indices[base + 0])];
    r.v1 = &s.vertices[8 * (size_t)(mdesc[2] + s.indices[base + 1])];
    r.v2 = &s.vertices[8 * (size_t)(mdesc[2] + s.indices[base + 2])];
    r.m = &s.transforms[16 * (size_t)idesc[2]];
    r.it = &s.inv_transposes[16 * (size_t)idesc[2]];
    r.mat = &s.materials[8 * (size_t)idesc[1]];
    r.flags = idesc[3];
    return r;
}

// scene.slang:178-269
template <class T>
void triangle_spawn(V3<T> v0, V3<T> v1, V3<T> v2, T bx, T by, const float* m, const float* it,
                    V3<T>* pos, V3<T>* nrm, T* off) {
    const T c0 = T(5.9604644775390625e-8f);
    const T c1 = T(1.7881397695873602e-7f);
    const T c2 = T(1.1920931797249068e-7f);
    V3<T> e1 = v1 - v0, e2 = v2 - v0;
    V3<T> op = {v0.x + Ops<T>::fma(bx, e1.x, by * e2.x), v0.y + Ops<T>::fma(bx, e1.y, by * e2.y),
                v0.z + Ops<T>::fma(bx, e1.z, by * e2.z)};
    V3<T> on = cross(e1, e2);
    V3<T> wp;
    wp.x = T(m[3]) + Ops<T>::fma(T(m[0]), op.x, Ops<T>::fma(T(m[1]), op.y, T(m[2]) * op.z));
    wp.y = T(m[7]) + Ops<T>::fma(T(m[4]), op.x, Ops<T>::fma(T(m[5]), op.y, T(m[6]) * op.z));
    wp.z = T(m[11]) + Ops<T>::fma(T(m[8]), op.x, Ops<T>::fma(T(m[9]), op.y, T(m[10]) * op.z));
    V3<T> wnu = {(T(it[0]) * on.x + T(it[1]) * on.y) + T(it[2]) * on.z,
                 (T(it[4]) * on.x + T(it[5]) * on.y) + T(it[6]) * on.z,
                 (T(it[8]) * on.x + T(it[9]) * on.y) + T(it[10]) * on.z};
    T ws = T(1) / Ops<T>::sqrt(vmax(dot(wnu, wnu), T(1e-30f)));
    V3<T> wn = wnu * ws;
    V3<T> ext3 = (vabs(e1) + vabs(e2)) + vabs(vabs(e1) - vabs(e2));
    T ext = vmax(vmax(ext3.x, ext3.y), ext3.z);
    V3<T> av0 = vabs(v0);
    V3<T> oe = {c0 * av0.x + c1 * ext, c0 * av0.y + c1 * ext, c0 * av0.z + c1 * ext};
    V3<T> aop = vabs(op);
    V3<T> we;
    we.x = c1 * dot(vabs(mk<T>(T(m[0]), T(m[1]), T(m[2]))), aop) + c2 * std::fabs(T(m[3]));
    we.y = c1 * dot(vabs(mk<T>(T(m[4]), T(m[5]), T(m[6]))), aop) + c2 * std::fabs(T(m[7]));
    we.z = c1 * dot(vabs(mk<T>(T(m[8]), T(m[9]), T(m[10]))), aop) + c2 * std::fabs(T(m[11]));
    V3<T> awp = vabs(wp);
    T te[3];
    for (int c = 0; c < 3; ++c) {
        // dot(abs(float4(it[0][c], it[1][c], it[2][c], it[3][c])), float4(|wp|, 1))
        te[c] = ((std::fabs(T(it[c])) * awp.x + std::fabs(T(it[4 + c])) * awp.y) +
                 std::fabs(T(it[8 + c])) * awp.z) +
                std::fabs(T(it[12 + c])) * T(1);
    }
    oe = oe + mk<T>(c2 * te[0], c2 * te[1], c2 * te[2]);
    T oo = dot(oe, vabs(on));
    T wo = dot(we, vabs(wn));
    wo = Ops<T>::fma(ws, oo, wo);
    *pos = wp;
    *nrm = wn;
    *off = wo;
}

// scene.slang:271-406 (opaque, untextured subset)
template <class T>
Shading<T> shading_data(const Scene& s, uint32_t inst, uint32_t prim, T bx, T by, V3<T> view) {
    TriRefs r = tri_refs(s, inst, prim);
    T b0 = (T(1) - bx) - by;
    V3<T> pos, fn;
    T off;
    triangle_spawn<T>(load3<T>(r.v0), load3<T>(r.v1), load3<T>(r.v2), bx, by, r.m, r.it, &pos, &fn, &off);
    V3<T> n0 = load3<T>(r.v0 + 3), n1 = load3<T>(r.v1 + 3), n2 = load3<T>(r.v2 + 3);
    V3<T> ni = (b0 * n0 + bx * n1) + by * n2;
    const float* it = r.it;
    V3<T> gnu = {((T(it[0]) * ni.x + T(it[1]) * ni.y) + T(it[2]) * ni.z) + T(it[3]) * T(0),
                 ((T(it[4]) * ni.x + T(it[5]) * ni.y) + T(it[6]) * ni.z) + T(it[7]) * T(0),
                 ((T(it[8]) * ni.x + T(it[9]) * ni.y) + T(it[10]) * ni.z) + T(it[11]) * T(0)};
    V3<T> gn = normalize(gnu);
    V3<T> sn = gn;
    uint32_t mflags;
    std::memcpy(&mflags, &r.mat[3], 4);
    bool double_sided = (mflags & 1u) != 0;
    bool front = dot(fn, view) > T(0);
    T sign = (double_sided && !front) ? T(-1) : T(1);
    fn = fn * sign;
    gn = gn * sign;
    sn = sn * sign;
    sn = adjust_shading_normal(sn, fn, -view);
    Shading<T> sd;
    sd.position = pos;
    sd.origin_front = pos + off * fn;
    sd.origin_back = pos - off * fn;
    sd.offset = off;
    sd.view_direction = view;
    sd.face_normal = fn;
    sd.shading_frame = Frame<T>(sn);
    sd.diffuse = load3<T>(r.mat);
    sd.emissive = load3<T>(r.mat + 4);
    sd.back_side = double_sided && !front;
    return sd;
}

// texture_space_path_tracer.slang:39-55
template <class T> V3<T> world_flat_normal(const Scene& s, uint32_t inst, uint32_t prim) {
    TriRefs r = tri_refs(s, inst, prim);
    V3<T> p0 = load3<T>(r.v0), p1 = load3<T>(r.v1), p2 = load3<T>(r.v2);
    V3<T> n = normalize(cross(p1 - p0, p2 - p0));  // common.slang:101-111
    if (r.flags & 1u) n = -n;
    const float* it = r.it;
    V3<T> w = {(T(it[0]) * n.x + T(it[1]) * n.y) + T(it[2]) * n.z,
               (T(it[4]) * n.x + T(it[5]) * n.y) + T(it[6]) * n.z,
               (T(it[8]) * n.x + T(it[9]) * n.y) + T(it[10]) * n.z};
    return normalize(w);
}

// ---------------------------------------------------------------------------
// Lights: scene.slang:940-990 (sun NEE), the sky as a constant or the
// sky-view LUT (sample_sky_lut, scene.slang:469-518), sun disk
// (scene.slang:408-465).
// ---------------------------------------------------------------------------
template <class T> struct LightCtx {
    V3<T> sun_dir, outer, trans, illum, sky;
    T cos_half, t_max;
    bool sun_disk, area_nee;
    const float* lut;
    int lut_w, lut_h;
    V3<T> up;
    T horizon;
    explicit LightCtx(const OracleLighting& p) {
        sun_dir = mk<T>(T(p.sun_direction[0]), T(p.sun_direction[1]), T(p.sun_direction[2]));
        V3<T> color = mk<T>(T(p.sun_color[0]), T(p.sun_color[1]), T(p.sun_color[2]));
        outer = color * T(p.sun_intensity);
        trans = mk<T>(T(p.sun_transmittance[0]), T(p.sun_transmittance[1]), T(p.sun_transmittance[2]));
        illum = outer * trans;
        sky = mk<T>(T(p.sky_radiance[0]), T(p.sky_radiance[1]), T(p.sky_radiance[2]));
        cos_half = T(p.sun_cos_half_angle);
        t_max = T(p.ray_t_max);
        sun_disk = (p.flags & 1u) != 0;
        area_nee = (p.flags & 2u) != 0;
        lut = p.sky_view_lut;
        lut_w = (int)p.sky_view_width;
        lut_h = (int)p.sky_view_height;
        up = mk<T>(T(p.sky_view_up[0]), T(p.sky_view_up[1]), T(p.sky_view_up[2]));
        horizon = T(p.sky_view_horizon_angle);
    }

    V3<T> texel(int x, int y) const {
        x %= lut_w;
        y %= lut_h;
        if (x < 0) x += lut_w;
        if (y < 0) y += lut_h;
        const float* e = lut + 4 * ((size_t)y * lut_w + x);
        return mk<T>(T(e[0]), T(e[1]), T(e[2]));
    }

    // sample_sky_lut, scene.slang:469-518 (a direction with no azimuth takes
    // u = 1/2; the bilinear fetch wraps, as the default sampler does).
    V3<T> sky_at(V3<T> d) const {
        if (!lut) return sky;
        const T half_pi = T(1.57079632679489662), two_pi = T(2) * T(3.14159265358979324);
        const T altitude = std::fmin(std::fmax(Ops<T>::asin(dot(d, up)), -half_pi + T(1e-2)), half_pi - T(1e-2));
        T azimuth = T(0);
        if (!(std::fabs(altitude) > half_pi - T(1e-4))) {
            const V3<T> right = cross(sun_dir, up);
            const V3<T> forward = cross(up, right);
            const V3<T> proj = normalize(d - up * dot(d, up));
            azimuth = Ops<T>::atan2(dot(proj, right), dot(proj, forward));
        }
        const T adj = (altitude + horizon) / half_pi;
        const T v = adj < T(0) ? T(0.5) * (T(1) - Ops<T>::sqrt(std::fmin(std::fmax(-adj, T(0)), T(1))))
                               : T(0.5) * (T(1) + Ops<T>::sqrt(std::fmin(std::fmax(adj, T(0)), T(1))));
        T u = azimuth / two_pi + T(0.5);
        if (!(u >= T(0) && u <= T(1))) u = T(0.5);
        const T fx = u * T(lut_w) - T(0.5), fy = v * T(lut_h) - T(0.5);
        const T x0 = std::floor(fx), y0 = std::floor(fy);
        const T tx = fx - x0, ty = fy - y0;
        const V3<T> a = texel((int)x0, (int)y0), b = texel((int)x0 + 1, (int)y0);
        const V3<T> c = texel((int)x0, (int)y0 + 1), e = texel((int)x0 + 1, (int)y0 + 1);
        const V3<T> top = mk<T>(a.x + tx * (b.x - a.x), a.y + tx * (b.y - a.y), a.z + tx * (b.z - a.z));
        const V3<T> bot = mk<T>(c.x + tx * (e.x - c.x), c.y + tx * (e.y - c.y), c.z + tx * (e.z - c.z));
        const V3<T> rgb = mk<T>(top.x + ty * (bot.x - top.x), top.y + ty * (bot.y - top.y), top.z + ty * (bot.z - top.z));
        return rgb * outer;
    }
};

template <class T> struct Tracer {
    const Scene& s;
    LightCtx<T> L;
    bool use_bvh;
    OracleRayCounts cnt{};
    Tracer(const Scene& sc, const OracleLighting& p) : s(sc), L(p), use_bvh(true) {}

    HitRec closest(V3<T> o, V3<T> d, T tmin, T tmax) {
        cnt.extend_rays++;
        RayPre<T> r = make_ray<T>(o, d, tmin, tmax);
        return trace<T>(s, r, false, use_bvh, &cnt);
    }
    T visibility(V3<T> o, V3<T> d) {
        cnt.shadow_rays++;
        RayPre<T> r = make_ray<T>(o, d, T(0), L.t_max);
        return trace<T>(s, r, true, use_bvh, &cnt).valid ? T(0) : T(1);
    }
    // scene.slang:954-990 (use_visibility_override == 0)
    V3<T> sun_nee(const Shading<T>& sd, T ux, T uy) {
        V3<T> l = sample_cone_direction<T>(L.sun_dir, L.cos_half, ux, uy);
        T vis = visibility(sd.origin_front, l);
        T ndl = vmax(T(0), dot(sd.shading_frame.n, l));
        V3<T> f = sd.diffuse * Consts<T>::INV_PI;
        return ((vis * f) * L.illum) * ndl;
    }
    // Area-light NEE of the screen tracer (an option beyond the reference):
    // triangle by area * luminance, uniform point, power-heuristic MIS weight
    // against the cosine BSDF pdf; emitters count from both sides.
    V3<T> area_nee(const Shading<T>& sd, T usel, T u0, T u1) {
        const size_t n = s.lights.size() / 16;
        if (n == 0) return mk<T>(0, 0, 0);
        size_t lo = 0, hi = n - 1;
        while (lo < hi) {
            size_t mid = (lo + hi) >> 1;
            if (usel < T(s.lights[16 * mid + 3])) hi = mid; else lo = mid + 1;
        }
        const float* r = &s.lights[16 * lo];
        T su = Ops<T>::sqrt(u0);
        T wa = su * (T(1) - u1), wb = su * u1;
        V3<T> p = mk<T>((T(r[0]) + T(r[4]) * wa) + T(r[8]) * wb, (T(r[1]) + T(r[5]) * wa) + T(r[9]) * wb,
                        (T(r[2]) + T(r[6]) * wa) + T(r[10]) * wb);
        V3<T> v = p - sd.origin_front;
        T d2 = dot(v, v);
        if (!(d2 > T(0))) return mk<T>(0, 0, 0);
        T dist = Ops<T>::sqrt(d2);
        V3<T> l = v * (T(1) / dist);
        T cx = dot(sd.shading_frame.n, l);
        if (!(cx > T(0))) return mk<T>(0, 0, 0);
        V3<T> nl = normalize(cross(mk<T>(T(r[4]), T(r[5]), T(r[6])), mk<T>(T(r[8]), T(r[9]), T(r[10]))));
        T cl = std::fabs(dot(nl, l));
        if (!(cl > T(1e-6f))) return mk<T>(0, 0, 0);
        T pl = ((T(r[11]) / T(s.light_power)) * d2) / cl;
        T pb = cx * Consts<T>::INV_PI;
        T w = (pl * pl) / (pl * pl + pb * pb);
        V3<T> f = sd.diffuse * Consts<T>::INV_PI;
        V3<T> c = (f * mk<T>(T(r[12]), T(r[13]), T(r[14]))) * ((cx / pl) * w);
        cnt.shadow_rays++;
        RayPre<T> ray = make_ray<T>(sd.origin_front, l, T(0), dist * T(0.999f));
        return trace<T>(s, ray, true, use_bvh, &cnt).valid ? mk<T>(0, 0, 0) : c;
    }
    T area_mis_weight(V3<T> emissive, V3<T> fn, V3<T> dir, T t, T pdf_bsdf) {
        T lum = (T(0.2126f) * emissive.x + T(0.7152f) * emissive.y) + T(0.0722f) * emissive.z;
        if (!(lum > T(0)) || s.lights.empty()) return T(1);
        T cl = std::fabs(dot(normalize(fn), dir));
        if (!(cl > T(1e-6f))) return T(0);
        T pl = ((lum / T(s.light_power)) * (t * t)) / cl;
        return (pdf_bsdf * pdf_bsdf) / (pdf_bsdf * pdf_bsdf + pl * pl);
    }
    // scene.slang:940-952
    V3<T> sun_irradiance(const Shading<T>& sd, T ux, T uy) {
        V3<T> l = sample_cone_direction<T>(L.sun_dir, L.cos_half, ux, uy);
        T vis = visibility(sd.origin_front, l);
        T ndl = vmax(T(0), dot(sd.shading_frame.n, l));
        return (vis * L.illum) * ndl;
    }
    // scene.slang:408-465
    V3<T> sun_disk(V3<T> dir) {
        V3<T> vp = mk<T>(T(0), T(6.360f + 0.0002f), T(0));
        V3<T> oc = vp;  // center at origin
        T a = dot(dir, dir);
        T b = T(2) * dot(oc, dir);
        T gr = T(6.360f);
        T c = dot(oc, oc) - gr * gr;
        T disc = b * b - T(4) * a * c;
        if (disc >= T(0)) {
            T sq = Ops<T>::sqrt(disc);
            T t0 = (-b - sq) / (T(2) * a);
            T t1 = (-b + sq) / (T(2) * a);
            if (t0 > T(0) || t1 > T(0)) return mk<T>(0, 0, 0);
        }
        T vdl = dot(dir, L.sun_dir);
        if (vdl > L.cos_half) {
            T solid = T(2) * Consts<T>::PI * (T(1) - L.cos_half);
            V3<T> lum = L.outer / solid;
            T soft = saturate(T(2) * (vdl - L.cos_half) / (T(1) - L.cos_half));
            return (L.trans * lum) * soft;
        }
        return mk<T>(0, 0, 0);
    }
};

// ---------------------------------------------------------------------------
// Screen path tracer: path_tracer.slang:40-130, camera.slang:201-236.
// ---------------------------------------------------------------------------
template <class T>
void screen_pixel(Tracer<T>& tr, const OracleLighting& lp, const OracleCamera& cam, uint32_t w,
                  uint32_t h, uint32_t frame, uint32_t max_vertices, uint32_t px, uint32_t py,
                  float* out) {
    Rng rng(px, py, frame * 1u + 0u);
    rng.next_1d();
    rng.next_1d();  // the unused jitter draw (path_tracer.slang:121)
    // camera.slang:223-236
    T pxf = (T((float)px) + T(0.5)) / T((float)w);
    T pyf = (T((float)py) + T(0.5)) / T((float)h);
    pxf = pxf + (-T(cam.jitter_x));
    pyf = pyf + T(cam.jitter_y);
    T nx = T(2) * pxf + T(-1);
    T ny = T(-2) * pyf + T(1);
    V3<T> U = load3<T>(cam.image_u), Vv = load3<T>(cam.image_v), W = load3<T>(cam.image_w);
    V3<T> dir = normalize((nx * U + ny * Vv) + W);
    T inv_cos = T(1) / dot(normalize(W), dir);
    T tmin = T(cam.near_clip) * inv_cos;
    T tmax = T(cam.far_clip) * inv_cos;
    V3<T> o = load3<T>(cam.position);
    V3<T> thp = mk<T>(1, 1, 1), Lr = mk<T>(0, 0, 0);
    T prev_pdf = T(1);
    (void)lp;
    for (uint32_t vi = 0; vi < max_vertices; ++vi) {
        HitRec hit = tr.closest(o, dir, tmin, tmax);
        if (!hit.valid) {
            V3<T> sky = tr.L.sky_at(dir);
            if (vi == 0 && tr.L.sun_disk) sky = sky + tr.sun_disk(dir);
            Lr = Lr + thp * sky;
            break;
        }
        uint32_t inst = tr.s.flat_instance[hit.flat], prim = tr.s.flat_prim[hit.flat];
        Shading<T> sd = shading_data<T>(tr.s, inst, prim, T(hit.b1), T(hit.b2), -dir);
        if (tr.L.area_nee && vi > 0)
            Lr = Lr + thp * (sd.emissive * tr.area_mis_weight(sd.emissive, sd.face_normal, dir, T(hit.t), prev_pdf));
        else
            Lr = Lr + thp * sd.emissive;
        T u0 = T(rng.next_1d()), u1 = T(rng.next_1d());
        V3<T> nee = tr.sun_nee(sd, u0, u1);
        Lr = Lr + thp * nee;
        // light reached from vertex vi lies on vertex vi + 1: sampled only where
        // that vertex exists, so both strategies cover the same path lengths
        if (tr.L.area_nee && vi + 1 < max_vertices) {
            T us = T(rng.next_1d()), a0 = T(rng.next_1d()), a1 = T(rng.next_1d());
            V3<T> an = tr.area_nee(sd, us, a0, a1);
            Lr = Lr + thp * an;
        }
        T e0 = T(rng.next_1d()), e1 = T(rng.next_1d());
        V3<T> wo;
        T pdf;
        cosine_sample_hemisphere<T>(e0, e1, &wo, &pdf);
        pdf = vmax(pdf, T(1e-6f));
        prev_pdf = pdf;
        V3<T> f = sd.diffuse * Consts<T>::INV_PI;
        thp = thp * ((f * std::fabs(wo.z)) / pdf);
        o = sd.origin_front;
        dir = sd.shading_frame.to_global(wo);
        tmin = T(0);
        tmax = tr.L.t_max;
    }
    out[0] = (float)Lr.x;
    out[1] = (float)Lr.y;
    out[2] = (float)Lr.z;
    out[3] = 1.0f;
}

// ---------------------------------------------------------------------------
// Texture-space tracer: texture_space_path_tracer.slang:57-216.
// ---------------------------------------------------------------------------
template <class T>
V3<T> ts_trace_radiance(Tracer<T>& tr, V3<T> o, V3<T> d, Rng& rng, uint32_t max_bounces) {
    V3<T> thp = mk<T>(1, 1, 1), rad = mk<T>(0, 0, 0);
    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        HitRec hit = tr.closest(o, d, T(0), tr.L.t_max);
        if (!hit.valid) {
            rad = rad + thp * tr.L.sky_at(d);
            return rad;
        }
        uint32_t inst = tr.s.flat_instance[hit.flat], prim = tr.s.flat_prim[hit.flat];
        Shading<T> sd = shading_data<T>(tr.s, inst, prim, T(hit.b1), T(hit.b2), -d);
        rad = rad + thp * sd.emissive;
        T u0 = T(rng.next_1d()), u1 = T(rng.next_1d());
        rad = rad + thp * tr.sun_nee(sd, u0, u1);
        T e0 = T(rng.next_1d()), e1 = T(rng.next_1d());
        V3<T> sdir;
        T pdf;
        cosine_sample_hemisphere<T>(e0, e1, &sdir, &pdf);
        if (pdf <= T(1e-6f)) return rad;
        V3<T> f = sd.diffuse * Consts<T>::INV_PI;
        thp = thp * ((f * std::fabs(sdir.z)) / pdf);
        o = sd.origin_front;
        d = sd.shading_frame.to_global(sdir);
    }
    return rad;
}

template <class T>
V3<T> ts_estimate(Tracer<T>& tr, uint32_t inst, uint32_t prim, T bx, T by, V3<T> view, uint32_t n,
                  Rng& rng, uint32_t max_bounces, bool direct = true) {
    Shading<T> sd = shading_data<T>(tr.s, inst, prim, bx, by, view);
    V3<T> irr = mk<T>(0, 0, 0);
    for (uint32_t k = 0; k < n; ++k) {
        T u0 = T(rng.next_1d()), u1 = T(rng.next_1d());
        V3<T> si = direct ? tr.sun_irradiance(sd, u0, u1) : mk<T>(0, 0, 0);
        T e0 = T(rng.next_1d()), e1 = T(rng.next_1d());
        V3<T> dir;
        T pdf;
        cosine_sample_hemisphere<T>(e0, e1, &dir, &pdf);
        if (pdf > T(1e-6f)) {
            V3<T> rad = ts_trace_radiance<T>(tr, sd.origin_front, sd.shading_frame.to_global(dir), rng,
                                             max_bounces);
            si = si + ((rad * std::fabs(dir.z)) / pdf);
        }
        irr = irr + si;
    }
    return irr / T((float)n);
}

// texture_space_path_tracer.slang:119-138 (float storage in the slot)
void store_running_mean(uint8_t* slots, uint32_t texel, const float* sample, bool reset) {
    uint32_t* w = reinterpret_cast<uint32_t*>(slots + 16 * (size_t)texel);
    uint32_t prev = reset ? 0u : w[3];
    float pv[3] = {0, 0, 0};
    if (prev != 0) std::memcpy(pv, w, 12);
    uint32_t next = std::min(prev + 1u, 65535u);
    float weight = 1.0f / (float)(prev + 1u);
    float acc[3];
    for (int c = 0; c < 3; ++c) acc[c] = pv[c] + weight * (sample[c] - pv[c]);
    std::memcpy(w, acc, 12);
    w[3] = next;
}

// ---------------------------------------------------------------------------
// Surface-probe baker: surface_probe_path_tracer.slang:47-315.
// ---------------------------------------------------------------------------
template <class T> struct ProbePath {
    V3<T> o, d, thp, rad;
    uint32_t src_inst, src_prim;
    T src_off;
    uint32_t self_hits;
    T first_hit, radial_max;
};

template <class T> void probe_trace_radiance(Tracer<T>& tr, ProbePath<T>& p, Rng& rng, uint32_t max_bounces) {
    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        HitRec hit = tr.closest(p.o, p.d, T(0), tr.L.t_max);
        if (!hit.valid) {
            if (bounce == 0u) p.first_hit = p.radial_max;
            p.rad = p.rad + p.thp * tr.L.sky_at(p.d);
            return;
        }
        T ht = T(hit.t);
        if (bounce == 0u) p.first_hit = vmin(ht, p.radial_max);
        uint32_t inst = tr.s.flat_instance[hit.flat], prim = tr.s.flat_prim[hit.flat];
        bool same_prim = inst == p.src_inst && prim == p.src_prim;
        T thr = vmax(T(4) * p.src_off, T(1e-6f));
        bool adjacent = inst == p.src_inst && ht <= thr;
        if (same_prim || adjacent) p.self_hits += 1u;
        Shading<T> sd = shading_data<T>(tr.s, inst, prim, T(hit.b1), T(hit.b2), -p.d);
        p.rad = p.rad + p.thp * sd.emissive;
        T u0 = T(rng.next_1d()), u1 = T(rng.next_1d());
        p.rad = p.rad + p.thp * tr.sun_nee(sd, u0, u1);
        T e0 = T(rng.next_1d()), e1 = T(rng.next_1d());
        V3<T> sdir;
        T pdf;
        cosine_sample_hemisphere<T>(e0, e1, &sdir, &pdf);
        if (pdf <= T(1e-6f)) return;
        V3<T> f = sd.diffuse * Consts<T>::INV_PI;
        p.thp = p.thp * ((f * std::fabs(sdir.z)) / pdf);
        V3<T> next_origin = sd.origin_front;
        V3<T> out_dir = Frame<T>(normalize(sd.face_normal)).to_global(sdir);
        p.o = next_origin;
        p.d = out_dir;
        p.src_inst = inst;
        p.src_prim = prim;
        p.src_off = length(next_origin - sd.position);
    }
}

struct ProbeBuffers {
    float* values;
    uint32_t* counts;
    uint32_t* self_hits;
    uint32_t* radial;
};

// surface_probe_path_tracer.slang:111-149 (moments kept as RG16F)
template <class T>
void accumulate_radial_moment(ProbeBuffers& b, uint32_t probe, uint32_t texel, T nd, uint32_t prev_iter,
                              uint32_t local_count, uint32_t spp) {
    uint32_t packed = b.radial[16 * (size_t)probe + texel];
    float px = f16_to_f32((uint16_t)(packed & 0xffffu));
    float py = f16_to_f32((uint16_t)(packed >> 16));
    float sample = (float)std::min(std::max(nd, T(0)), T(2));
    float smx = sample, smy = sample * sample;
    if (py <= 0.0f) {
        px = smx;
        py = smy;
    } else {
        float pop = ((float)prev_iter * (float)std::max(spp, 1u)) * radial_texel_cosine_probability(texel);
        uint32_t expected = prev_iter == 0u ? local_count - 1u : std::max((uint32_t)pop, 1u);
        float alpha = 1.0f / (float)std::max(std::min(expected + local_count, 4096u), 1u);
        px = px + alpha * (smx - px);
        py = py + alpha * (smy - py);
    }
    px = std::min(std::max(px, 0.0f), 4.0f);
    py = std::min(std::max(py, 0.0f), 4.0f);
    b.radial[16 * (size_t)probe + texel] = (uint32_t)f32_to_f16(px) | ((uint32_t)f32_to_f16(py) << 16);
}

template <class T>
void probe_unit(Tracer<T>& tr, ProbeBuffers& b, const uint8_t* probes, const uint8_t* pinst, uint32_t probe,
                uint32_t iteration, uint32_t spp, uint32_t max_bounces, bool reset, bool independent = false) {
    const uint8_t* rec = probes + 48 * (size_t)probe;
    float nrm[4];
    uint32_t meta[4];
    std::memcpy(nrm, rec + 16, 16);
    std::memcpy(meta, rec + 32, 16);
    uint32_t inst = meta[3] >> 8;
    float params[4];
    std::memcpy(params, pinst + 48 * (size_t)inst + 32, 16);
    float bx, by;
    std::memcpy(&bx, &meta[1], 4);
    std::memcpy(&by, &meta[2], 4);
    uint32_t prim = meta[0];
    uint32_t n = std::max(spp, 1u);
    Rng rng(probe, inst, iteration * n);
    V3<T> view = normalize(mk<T>(T(nrm[0]), T(nrm[1]), T(nrm[2])));
    T kr = vmax(T(params[0]), T(1e-6f));
    // estimate_surface_irradiance (surface_probe_path_tracer.slang:206-278)
    Shading<T> sd = shading_data<T>(tr.s, inst, prim, T(bx), T(by), view);
    V3<T> irr = mk<T>(0, 0, 0);
    uint32_t self_total = 0;
    uint32_t prev_iter = reset ? 0u : b.counts[probe];
    uint32_t local_counts[16] = {0};
    if (reset)
        for (int t = 0; t < 16; ++t) b.radial[16 * (size_t)probe + t] = 0u;
    for (uint32_t k = 0; k < n; ++k) {
        // independent-sample mode (batched baker option): sample k has its own
        // stream RNG(probe, instance, iteration * n + k)
        Rng own(probe, inst, iteration * n + k);
        Rng& r = independent ? own : rng;
        V3<T> si = mk<T>(0, 0, 0);
        T e0 = T(r.next_1d()), e1 = T(r.next_1d());
        V3<T> dir;
        T pdf;
        cosine_sample_hemisphere<T>(e0, e1, &dir, &pdf);
        if (pdf > T(1e-6f)) {
            ProbePath<T> p;
            V3<T> origin = sd.origin_front;
            p.o = origin;
            p.d = Frame<T>(normalize(sd.face_normal)).to_global(dir);
            p.thp = mk<T>(1, 1, 1);
            p.rad = mk<T>(0, 0, 0);
            p.src_inst = inst;
            p.src_prim = prim;
            p.src_off = length(origin - sd.position);
            p.self_hits = 0;
            p.first_hit = T(2) * kr;
            p.radial_max = T(2) * kr;
            probe_trace_radiance<T>(tr, p, r, max_bounces);
            self_total += p.self_hits;
            float u, v;
            hemi_oct_encode((float)dir.x, (float)dir.y, (float)dir.z, &u, &v);
            uint32_t texel = radial_texel_index(u, v);
            local_counts[texel] += 1u;
            accumulate_radial_moment<T>(b, probe, texel, p.first_hit / vmax(kr, T(1e-6f)), prev_iter,
                                        local_counts[texel], spp);
            si = si + ((p.rad * std::fabs(dir.z)) / pdf);
        }
        irr = irr + si;
    }
    irr = irr / T((float)n);
    // store_accumulated_irradiance (:47-65)
    uint32_t prev = reset ? 0u : b.counts[probe];
    float pv[3] = {0, 0, 0};
    if (prev != 0) std::memcpy(pv, b.values + 3 * (size_t)probe, 12);
    uint32_t next = std::min(prev + 1u, 65535u);
    float weight = 1.0f / (float)(prev + 1u);
    float smp[3] = {(float)irr.x, (float)irr.y, (float)irr.z};
    for (int c = 0; c < 3; ++c) b.values[3 * (size_t)probe + c] = pv[c] + weight * (smp[c] - pv[c]);
    b.counts[probe] = next;
    // store_accumulated_self_hit_count (:67-79)
    uint32_t prev_self = reset ? 0u : b.self_hits[probe];
    b.self_hits[probe] = prev_self + self_total;
}

// Mesh Colors resolve (mesh_colors_resolve.slang:29-73) and the frozen RGB9E5
// variant (mesh_colors_frozen_resolve.slang:93-135), one pixel.
template <class T>
void resolve_pixel(Tracer<T>& tr, const OracleCamera& cam, uint32_t w, uint32_t h, uint32_t px, uint32_t py,
                   const uint32_t* face_infos, const uint32_t* instance_infos, const uint32_t* side_infos,
                   uint32_t instance_count, const void* colors, bool packed, float* out) {
    // compute_ray_pinhole (camera.slang:223-236)
    T pxf = (T((float)px) + T(0.5)) / T((float)w);
    T pyf = (T((float)py) + T(0.5)) / T((float)h);
    pxf = pxf + (-T(cam.jitter_x));
    pyf = pyf + T(cam.jitter_y);
    T nx = T(2) * pxf + T(-1);
    T ny = T(-2) * pyf + T(1);
    V3<T> U = load3<T>(cam.image_u), Vv = load3<T>(cam.image_v), W = load3<T>(cam.image_w);
    V3<T> dir = normalize((nx * U + ny * Vv) + W);
    T inv_cos = T(1) / dot(normalize(W), dir);
    V3<T> o = load3<T>(cam.position);
    HitRec hit = tr.closest(o, dir, T(cam.near_clip) * inv_cos, T(cam.far_clip) * inv_cos);
    out[3] = 1.0f;
    if (!hit.valid) {
        V3<T> sky = tr.L.sky_at(dir);
        if (tr.L.sun_disk) sky = sky + tr.sun_disk(dir);
        out[0] = (float)sky.x; out[1] = (float)sky.y; out[2] = (float)sky.z;
        return;
    }
    uint32_t inst = tr.s.flat_instance[hit.flat], prim = tr.s.flat_prim[hit.flat];
    bool back = dot(world_flat_normal<T>(tr.s, inst, prim), -dir) <= T(0);
    out[0] = out[1] = out[2] = 0.0f;
    if (inst >= instance_count) return;
    InstInfo ii{instance_infos[4 * inst], instance_infos[4 * inst + 1], instance_infos[4 * inst + 2],
                instance_infos[4 * inst + 3]};
    uint32_t side_back = side_infos[2 * inst], side_flags = side_infos[2 * inst + 1];
    if (back && !(side_flags & 1u)) return;
    FaceInfo f{face_infos[2 * (ii.face_offset + prim)], face_infos[2 * (ii.face_offset + prim) + 1]};
    auto load = [&](uint32_t front) {
        uint32_t t = back ? side_back + (front - ii.texel_offset) : front;
        float c[3];
        if (packed) {
            unpack_rgb9e5(static_cast<const uint32_t*>(colors)[t], c);
        } else {
            std::memcpy(c, static_cast<const uint8_t*>(colors) + 16 * (size_t)t, 12);
        }
        return mk<T>(T(c[0]), T(c[1]), T(c[2]));
    };
    T b1 = T(hit.b1), b2 = T(hit.b2);
    T b0 = (T(1) - b1) - b2;
    uint32_t R = f.resolution;
    T rf = T((float)R);
    T s0 = saturate(b0) * rf, s1 = saturate(b1) * rf, s2 = saturate(b2) * rf;
    uint32_t i = std::min((uint32_t)s0, R);
    uint32_t j = std::min((uint32_t)s1, R - i);
    T w0 = s0 - std::floor(s0), w1 = s1 - std::floor(s1), w2 = s2 - std::floor(s2);
    bool upper = std::fabs(((w0 + w1) + w2) - T(2)) <= T(1e-3f);
    if (upper) {
        w0 = T(1) - w0;
        w1 = T(1) - w1;
        w2 = T(1) - w2;
    }
    V3<T> irr;
    if ((w0 + w1) + w2 <= T(1e-6f) || i >= R || j >= R - i) {
        irr = load(mc_address(i, j, ii, f));
    } else if (upper) {
        irr = (w0 * load(mc_address(i, j + 1, ii, f)) + w1 * load(mc_address(i + 1, j, ii, f))) +
              w2 * load(mc_address(i + 1, j + 1, ii, f));
    } else {
        irr = (w0 * load(mc_address(i + 1, j, ii, f)) + w1 * load(mc_address(i, j + 1, ii, f))) +
              w2 * load(mc_address(i, j, ii, f));
    }
    Shading<T> sd = shading_data<T>(tr.s, inst, prim, b1, b2, -dir);
    V3<T> c = sd.emissive + (sd.diffuse * Consts<T>::INV_PI) * irr;
    out[0] = (float)c.x; out[1] = (float)c.y; out[2] = (float)c.z;
}

// mesh_colors_sample_irradiance (mesh_colors.slang:365-426) on float32 slots.
V3<float> mc_sample_slots(const uint8_t* slots, float b0, float b1, float b2, const InstInfo& ii, const FaceInfo& f,
                          uint32_t side_back, bool back) {
    auto load = [&](uint32_t front) {
        uint32_t t = back ? side_back + (front - ii.texel_offset) : front;
        float c[3];
        std::memcpy(c, slots + 16 * (size_t)t, 12);
        return mk<float>(c[0], c[1], c[2]);
    };
    uint32_t R = f.resolution;
    float rf = (float)R;
    float s0 = saturate(b0) * rf, s1 = saturate(b1) * rf, s2 = saturate(b2) * rf;
    uint32_t i = std::min((uint32_t)s0, R);
    uint32_t j = std::min((uint32_t)s1, R - i);
    float w0 = s0 - std::floor(s0), w1 = s1 - std::floor(s1), w2 = s2 - std::floor(s2);
    bool upper = std::fabs(((w0 + w1) + w2) - 2.0f) <= 1e-3f;
    if (upper) {
        w0 = 1.0f - w0;
        w1 = 1.0f - w1;
        w2 = 1.0f - w2;
    }
    if ((w0 + w1) + w2 <= 1e-6f || i >= R || j >= R - i) return load(mc_address(i, j, ii, f));
    if (upper)
        return (w0 * load(mc_address(i, j + 1, ii, f)) + w1 * load(mc_address(i + 1, j, ii, f))) +
               w2 * load(mc_address(i + 1, j + 1, ii, f));
    return (w0 * load(mc_address(i + 1, j, ii, f)) + w1 * load(mc_address(i, j + 1, ii, f))) +
           w2 * load(mc_address(i, j, ii, f));
}

// One pass of the one-ring surface filter, mesh_colors_surface_filter.slang:
// 1-253 (float32 like the shader; acos and exp from the C library).
void surface_filter_texel(const uint32_t* face_infos, const InstInfo& ii, uint32_t side_back, uint32_t side_flags,
                          const uint32_t* adjacency, const float* normals, const uint8_t* src, uint8_t* dst,
                          uint32_t local, float neighbor_weight, float sigma) {
    FaceInfo f;
    uint32_t prim;
    if (!find_face(face_infos, ii, local, &f, &prim)) return;
    uint32_t ti, tj;
    address_to_ij(local - f.address, f.resolution, &ti, &tj);
    const float* cnp = normals + 4 * (size_t)(ii.face_offset + prim);
    V3<float> cn = mk<float>(cnp[0], cnp[1], cnp[2]);
    uint32_t front = ii.texel_offset + local;
    const int off[6][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, -1}, {-1, 1}};
    for (int side = 0; side < ((side_flags & 1u) ? 2 : 1); ++side) {
        bool back = side == 1;
        uint32_t center = back ? side_back + (front - ii.texel_offset) : front;
        float c[4];
        std::memcpy(c, src + 16 * (size_t)center, 16);
        V3<float> acc = mk<float>(c[0], c[1], c[2]);
        float wsum = 1.0f;
        int R = (int)f.resolution;
        for (int t = 0; t < 6; ++t) {
            int x = (int)ti + off[t][0], y = (int)tj + off[t][1];
            if (x >= 0 && y >= 0 && x + y <= R) {
                uint32_t ft = mc_address((uint32_t)x, (uint32_t)y, ii, f);
                uint32_t tt = back ? side_back + (ft - ii.texel_offset) : ft;
                float v[3];
                std::memcpy(v, src + 16 * (size_t)tt, 12);
                acc = acc + neighbor_weight * mk<float>(v[0], v[1], v[2]);
                wsum = wsum + neighbor_weight;
                continue;
            }
            uint32_t edge = x < 0 ? 1u : (y < 0 ? 2u : 0u);
            uint32_t packed = adjacency[4 * (size_t)(ii.face_offset + prim) + edge];
            if (packed == 0xffffffffu) continue;
            uint32_t adj_face = ii.face_offset + (packed >> 3);
            uint32_t adj_edge = packed & 3u;
            bool flip = (packed & 4u) != 0;
            // mesh_colors_map_one_edge_tap (mesh_colors.slang:156-203)
            float inv = 1.0f / (float)f.resolution;
            float sb[3] = {(float)x * inv, (float)y * inv, 1.0f - (float)(x + y) * inv};
            uint32_t s_start = edge, s_end = (edge + 1) % 3, s_opp = (edge + 2) % 3;
            uint32_t n_start = adj_edge, n_end = (adj_edge + 1) % 3, n_opp = (adj_edge + 2) % 3;
            float outside = sb[s_opp];
            uint32_t m_start = flip ? n_end : n_start, m_end = flip ? n_start : n_end;
            float nb[3] = {0.0f, 0.0f, 0.0f};
            nb[m_start] = sb[s_start] + outside;
            nb[m_end] = sb[s_end] + outside;
            nb[n_opp] = -outside;
            bool ok = true;
            for (int k = 0; k < 3; ++k)
                if (nb[k] < -1e-5f || nb[k] > 1.0f + 1e-5f) ok = false;
            if (!ok) continue;
            for (int k = 0; k < 3; ++k) nb[k] = std::max(nb[k], 0.0f);
            float sum = std::max((nb[0] + nb[1]) + nb[2], 1e-6f);
            for (int k = 0; k < 3; ++k) nb[k] = nb[k] / sum;
            // mesh_colors_normal_filter_weight (mesh_colors.slang:205-216)
            const float* np_ = normals + 4 * (size_t)adj_face;
            float cosine = std::min(std::max(dot(cn, mk<float>(np_[0], np_[1], np_[2])), 0.0f), 1.0f);
            float nw;
            if (sigma <= 1e-6f) {
                nw = cosine >= 1.0f - 1e-6f ? 1.0f : 0.0f;
            } else {
                float na = std::acos(cosine) / sigma;
                nw = std::exp(-0.5f * na * na);
            }
            float w = neighbor_weight * nw;
            FaceInfo nf{face_infos[2 * adj_face], face_infos[2 * adj_face + 1]};
            V3<float> v = mc_sample_slots(src, nb[0], nb[1], nb[2], ii, nf, side_back, back);
            if (w > 0.0f) {
                acc = acc + w * v;
                wsum = wsum + w;
            }
        }
        V3<float> r = acc / std::max(wsum, 1e-6f);
        float outv[3] = {r.x, r.y, r.z};
        std::memcpy(dst + 16 * (size_t)center, outv, 12);
        std::memcpy(dst + 16 * (size_t)center + 12, &c[3], 4);
    }
}

// PRT L2 field baker, surface_probe_prt_baker.slang:169-371, with the real
// SH L2 basis of surface_probe_sh.slang:5-21.
template <class T> T sh_l2_basis(uint32_t c, V3<T> dir) {
    V3<T> d = normalize(dir);
    T x = d.x, y = d.y, z = d.z;
    switch (c) {
        case 0: return T(0.2820947918f);
        case 1: return T(0.4886025119f) * y;
        case 2: return T(0.4886025119f) * z;
        case 3: return T(0.4886025119f) * x;
        case 4: return T(1.0925484306f) * x * y;
        case 5: return T(1.0925484306f) * y * z;
        case 6: return T(0.3153915653f) * (T(3) * y * y - T(1));
        case 7: return T(1.0925484306f) * x * z;
        default: return T(0.5462742153f) * (x * x - z * z);
    }
}

template <class T>
void probe_prt_unit(Tracer<T>& tr, ProbeBuffers& b, float* static_source, const uint8_t* probes,
                    const uint8_t* pinst, uint32_t probe, uint32_t iteration, uint32_t spp, uint32_t max_bounces,
                    bool reset) {
    const uint8_t* rec = probes + 48 * (size_t)probe;
    float nrm[4];
    uint32_t meta[4];
    std::memcpy(nrm, rec + 16, 16);
    std::memcpy(meta, rec + 32, 16);
    uint32_t inst = meta[3] >> 8;
    float params[4];
    std::memcpy(params, pinst + 48 * (size_t)inst + 32, 16);
    float bx, by;
    std::memcpy(&bx, &meta[1], 4);
    std::memcpy(&by, &meta[2], 4);
    uint32_t prim = meta[0];
    uint32_t n = std::max(spp, 1u);
    Rng rng(probe, inst, iteration * n);
    V3<T> view = normalize(mk<T>(T(nrm[0]), T(nrm[1]), T(nrm[2])));
    T kr = vmax(T(params[0]), T(1e-6f));
    Shading<T> sd = shading_data<T>(tr.s, inst, prim, T(bx), T(by), view);
    V3<T> transport[9];
    for (auto& t : transport) t = mk<T>(0, 0, 0);
    V3<T> stat = mk<T>(0, 0, 0);
    uint32_t self_total = 0;
    uint32_t prev_iter = reset ? 0u : b.counts[probe];
    uint32_t local_counts[16] = {0};
    if (reset)
        for (int t = 0; t < 16; ++t) b.radial[16 * (size_t)probe + t] = 0u;
    for (uint32_t k = 0; k < n; ++k) {
        T e0 = T(rng.next_1d()), e1 = T(rng.next_1d());
        V3<T> dir;
        T pdf;
        cosine_sample_hemisphere<T>(e0, e1, &dir, &pdf);
        if (pdf <= T(1e-6f)) continue;
        V3<T> lt[9];
        for (auto& t : lt) t = mk<T>(0, 0, 0);
        ProbePath<T> p;
        V3<T> origin = sd.origin_front;
        p.o = origin;
        p.d = Frame<T>(normalize(sd.face_normal)).to_global(dir);
        p.thp = mk<T>(1, 1, 1);
        p.rad = mk<T>(0, 0, 0);  // the static source of this path
        p.src_inst = inst;
        p.src_prim = prim;
        p.src_off = length(origin - sd.position);
        p.self_hits = 0;
        p.first_hit = T(2) * kr;
        p.radial_max = T(2) * kr;
        for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
            HitRec hit = tr.closest(p.o, p.d, T(0), tr.L.t_max);
            if (!hit.valid) {
                if (bounce == 0u) p.first_hit = p.radial_max;
                for (uint32_t c = 0; c < 9; ++c) lt[c] = lt[c] + p.thp * sh_l2_basis<T>(c, p.d);
                break;
            }
            T ht = T(hit.t);
            if (bounce == 0u) p.first_hit = vmin(ht, p.radial_max);
            uint32_t hi = tr.s.flat_instance[hit.flat], hp = tr.s.flat_prim[hit.flat];
            bool same_prim = hi == p.src_inst && hp == p.src_prim;
            T thr = vmax(T(4) * p.src_off, T(1e-6f));
            bool adjacent = hi == p.src_inst && ht <= thr;
            if (same_prim || adjacent) p.self_hits += 1u;
            Shading<T> hs = shading_data<T>(tr.s, hi, hp, T(hit.b1), T(hit.b2), -p.d);
            p.rad = p.rad + p.thp * hs.emissive;
            T u0 = T(rng.next_1d()), u1 = T(rng.next_1d());
            p.rad = p.rad + p.thp * tr.sun_nee(hs, u0, u1);
            T f0 = T(rng.next_1d()), f1 = T(rng.next_1d());
            V3<T> sdir;
            T spdf;
            cosine_sample_hemisphere<T>(f0, f1, &sdir, &spdf);
            if (spdf <= T(1e-6f)) break;
            V3<T> f = hs.diffuse * Consts<T>::INV_PI;
            p.thp = p.thp * ((f * std::fabs(sdir.z)) / spdf);
            V3<T> next_origin = hs.origin_front;
            p.d = Frame<T>(normalize(hs.face_normal)).to_global(sdir);
            p.o = next_origin;
            p.src_inst = hi;
            p.src_prim = hp;
            p.src_off = length(next_origin - hs.position);
        }
        self_total += p.self_hits;
        T w = std::fabs(dir.z) / pdf;
        for (int c = 0; c < 9; ++c) transport[c] = transport[c] + w * lt[c];
        stat = stat + w * p.rad;
        float u, v;
        hemi_oct_encode((float)dir.x, (float)dir.y, (float)dir.z, &u, &v);
        uint32_t texel = radial_texel_index(u, v);
        local_counts[texel] += 1u;
        accumulate_radial_moment<T>(b, probe, texel, p.first_hit / vmax(kr, T(1e-6f)), prev_iter,
                                    local_counts[texel], spp);
    }
    T inv = T(1) / T((float)n);
    uint32_t prev = reset ? 0u : b.counts[probe];
    float weight = 1.0f / (float)(prev + 1u);
    for (int c = 0; c < 9; ++c) {
        V3<T> t = transport[c] * inv;
        float* v = b.values + 27 * (size_t)probe + 3 * c;
        float tv[3] = {(float)t.x, (float)t.y, (float)t.z};
        for (int ch = 0; ch < 3; ++ch) {
            float pv = prev == 0u ? 0.0f : v[ch];
            v[ch] = pv + weight * (tv[ch] - pv);
        }
    }
    {
        V3<T> t = stat * inv;
        float* v = static_source + 3 * (size_t)probe;
        float tv[3] = {(float)t.x, (float)t.y, (float)t.z};
        for (int ch = 0; ch < 3; ++ch) {
            float pv = prev == 0u ? 0.0f : v[ch];
            v[ch] = pv + weight * (tv[ch] - pv);
        }
    }
    b.counts[probe] = std::min(prev + 1u, 65535u);
    uint32_t prev_self = reset ? 0u : b.self_hits[probe];
    b.self_hits[probe] = prev_self + self_total;
}

template <class F> void parallel_for(int count, int threads, F&& fn) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    threads = std::max(1, std::min(threads, count));
    if (threads == 1) {
        for (int i = 0; i < count; ++i) fn(i, 0);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t]() {
            for (;;) {
                int i = next.fetch_add(1);
                if (i >= count) break;
                fn(i, t);
            }
        });
    for (auto& th : pool) th.join();
}

void add_counts(OracleRayCounts* dst, const OracleRayCounts& src) {
    if (!dst) return;
    dst->extend_rays += src.extend_rays;
    dst->shadow_rays += src.shadow_rays;
    dst->node_fetches += src.node_fetches;
    dst->triangle_tests += src.triangle_tests;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* oracle_last_error(void) { return g_error.c_str(); }

void oracle_rng_sequence(uint32_t x, uint32_t y, uint32_t sample_index, int count, float* out) {
    Rng r(x, y, sample_index);
    for (int i = 0; i < count; ++i) out[i] = r.next_1d();
}

void oracle_sincos(const float* a, int count, float* s, float* c) {
    for (int i = 0; i < count; ++i) own_sincos(a[i], &s[i], &c[i]);
}

void oracle_atan2_asin(const float* y, const float* x, int count, float* out_atan2, float* out_asin) {
    for (int i = 0; i < count; ++i) {
        out_atan2[i] = own_atan2(y[i], x[i]);
        out_asin[i] = own_asin(y[i]);
    }
}

void oracle_sky_radiance(const OracleLighting* lighting, const float* dirs, int count, int precision, float* out) {
    if (precision == ORACLE_F64) {
        LightCtx<double> L(*lighting);
        for (int i = 0; i < count; ++i) {
            const V3<double> v = L.sky_at(mk<double>(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
            out[3 * i] = (float)v.x;
            out[3 * i + 1] = (float)v.y;
            out[3 * i + 2] = (float)v.z;
        }
        return;
    }
    LightCtx<float> L(*lighting);
    for (int i = 0; i < count; ++i) {
        const V3<float> v = L.sky_at(mk<float>(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    }
}

void oracle_pack_rgb9e5(const float* rgb, int count, uint32_t* out) {
    for (int i = 0; i < count; ++i) out[i] = pack_rgb9e5(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
}

void oracle_unpack_rgb9e5(const uint32_t* p, int count, float* out) {
    for (int i = 0; i < count; ++i) unpack_rgb9e5(p[i], out + 3 * i);
}

void oracle_f32_to_f16(const float* v, int count, uint16_t* out) {
    for (int i = 0; i < count; ++i) out[i] = f32_to_f16(v[i]);
}

void oracle_hemi_oct_encode(const float* d, int count, float* uv) {
    for (int i = 0; i < count; ++i) hemi_oct_encode(d[3 * i], d[3 * i + 1], d[3 * i + 2], &uv[2 * i], &uv[2 * i + 1]);
}

void oracle_hemi_oct_decode(const float* uv, int count, float* d) {
    for (int i = 0; i < count; ++i) hemi_oct_decode(uv[2 * i], uv[2 * i + 1], d + 3 * i);
}

void oracle_cosine_sample_hemisphere(const float* u, int count, float* out4) {
    for (int i = 0; i < count; ++i) {
        V3<float> h;
        float pdf;
        cosine_sample_hemisphere<float>(u[2 * i], u[2 * i + 1], &h, &pdf);
        out4[4 * i] = h.x;
        out4[4 * i + 1] = h.y;
        out4[4 * i + 2] = h.z;
        out4[4 * i + 3] = pdf;
    }
}

void oracle_mesh_colors_address_to_ij(const uint32_t* a, const uint32_t* r, int count, uint32_t* ij) {
    for (int i = 0; i < count; ++i) address_to_ij(a[i], r[i], &ij[2 * i], &ij[2 * i + 1]);
}

void* oracle_scene_create(const float* vertices, int vertex_count, const uint32_t* indices, int triangle_count,
                          const uint32_t* mesh_descs, int mesh_count, const uint32_t* instance_descs,
                          int instance_count, const float* transforms, const float* inverse_transposes,
                          int transform_count, const float* materials, int material_count) {
    Scene* s = new Scene();
    s->vertices.assign(vertices, vertices + 8 * (size_t)vertex_count);
    s->indices.assign(indices, indices + 3 * (size_t)triangle_count);
    s->mesh_descs.assign(mesh_descs, mesh_descs + 4 * (size_t)mesh_count);
    s->instance_descs.assign(instance_descs, instance_descs + 4 * (size_t)instance_count);
    s->transforms.assign(transforms, transforms + 16 * (size_t)transform_count);
    s->inv_transposes.assign(inverse_transposes, inverse_transposes + 16 * (size_t)transform_count);
    s->materials.assign(materials, materials + 8 * (size_t)material_count);
    for (int i = 0; i < instance_count; ++i) {
        const uint32_t* id = &s->instance_descs[4 * (size_t)i];
        const uint32_t* md = &s->mesh_descs[4 * (size_t)id[0]];
        uint32_t tris = md[1] / 3u;
        s->instance_first_flat.push_back((uint32_t)s->flat_instance.size());
        const float* m = &s->transforms[16 * (size_t)id[2]];
        for (uint32_t p = 0; p < tris; ++p) {
            s->flat_instance.push_back((uint32_t)i);
            s->flat_prim.push_back(p);
            for (int k = 0; k < 3; ++k) {
                const float* v = &s->vertices[8 * (size_t)(md[2] + s->indices[md[3] + 3 * p + k])];
                V3<float> wf = xform_point<float>(m, mk<float>(v[0], v[1], v[2]));
                V3<double> wd = xform_point<double>(m, mk<double>(v[0], v[1], v[2]));
                s->world_f.push_back(wf.x);
                s->world_f.push_back(wf.y);
                s->world_f.push_back(wf.z);
                s->world_d.push_back(wd.x);
                s->world_d.push_back(wd.y);
                s->world_d.push_back(wd.z);
            }
        }
    }
    build_bvh(*s);
    return s;
}

void oracle_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

int oracle_scene_triangle_count(void* s) { return (int)static_cast<Scene*>(s)->tri_count(); }

void oracle_scene_world_triangles(void* sp, float* out9) {
    Scene* s = static_cast<Scene*>(sp);
    std::memcpy(out9, s->world_f.data(), s->world_f.size() * sizeof(float));
}

void oracle_scene_bvh_stats(void* sp, double* out3) {
    Scene* s = static_cast<Scene*>(sp);
    double leaves = 0, sah = 0;
    double root_area = s->nodes.empty() ? 1.0 : (double)s->nodes[0].box.half_area();
    for (const BvhNode& n : s->nodes) {
        double a = (double)n.box.half_area() / std::max(root_area, 1e-30);
        if (n.count > 0) {
            leaves += 1;
            sah += a * (double)n.count;
        } else {
            sah += a;
        }
    }
    out3[0] = (double)s->nodes.size();
    out3[1] = leaves;
    out3[2] = sah;
}

void oracle_intersect(void* sp, const float* rays, int count, int mode, uint32_t* ids, float* tb,
                      OracleRayCounts* counts) {
    Scene* s = static_cast<Scene*>(sp);
    for (int i = 0; i < count; ++i) {
        const float* r = rays + 8 * (size_t)i;
        HitRec h;
        OracleRayCounts c{};
        if (mode == 2) {
            RayPre<double> rp = make_ray<double>(mk<double>(r[0], r[1], r[2]), mk<double>(r[4], r[5], r[6]), r[3], r[7]);
            h = trace<double>(*s, rp, false, false, &c);
        } else {
            RayPre<float> rp = make_ray<float>(mk<float>(r[0], r[1], r[2]), mk<float>(r[4], r[5], r[6]), r[3], r[7]);
            h = trace<float>(*s, rp, false, mode == 0, &c);
        }
        add_counts(counts, c);
        ids[4 * i + 0] = h.valid ? 1u : 0u;
        ids[4 * i + 1] = h.valid ? s->flat_instance[h.flat] : 0u;
        ids[4 * i + 2] = h.valid ? s->flat_prim[h.flat] : 0u;
        ids[4 * i + 3] = h.valid ? h.flat : 0xffffffffu;
        tb[3 * i + 0] = (float)h.t;
        tb[3 * i + 1] = (float)h.b1;
        tb[3 * i + 2] = (float)h.b2;
    }
}

void oracle_visibility(void* sp, const float* rays, int count, int mode, float* vis, OracleRayCounts* counts) {
    Scene* s = static_cast<Scene*>(sp);
    for (int i = 0; i < count; ++i) {
        const float* r = rays + 8 * (size_t)i;
        HitRec h;
        OracleRayCounts c{};
        if (mode == 2) {
            RayPre<double> rp = make_ray<double>(mk<double>(r[0], r[1], r[2]), mk<double>(r[4], r[5], r[6]), r[3], r[7]);
            h = trace<double>(*s, rp, true, false, &c);
        } else {
            RayPre<float> rp = make_ray<float>(mk<float>(r[0], r[1], r[2]), mk<float>(r[4], r[5], r[6]), r[3], r[7]);
            h = trace<float>(*s, rp, true, mode == 0, &c);
        }
        add_counts(counts, c);
        vis[i] = h.valid ? 0.0f : 1.0f;
    }
}

int oracle_trace_screen(void* sp, const OracleLighting* lighting, const OracleCamera* camera, uint32_t width,
                        uint32_t height, uint32_t frame, uint32_t max_vertices, const uint32_t* pixels,
                        int pixel_count, int precision, int threads, float* out, OracleRayCounts* counts) {
    Scene* s = static_cast<Scene*>(sp);
    std::vector<OracleRayCounts> per(std::max(1, threads <= 0 ? (int)std::thread::hardware_concurrency() : threads) + 1);
    std::vector<OracleRayCounts> unit_counts((size_t)pixel_count);
    parallel_for(pixel_count, threads, [&](int i, int) {
        uint32_t px = pixels[2 * i], py = pixels[2 * i + 1];
        if (precision == ORACLE_F64) {
            Tracer<double> tr(*s, *lighting);
            screen_pixel<double>(tr, *lighting, *camera, width, height, frame, max_vertices, px, py, out + 4 * (size_t)i);
            unit_counts[i] = tr.cnt;
        } else {
            Tracer<float> tr(*s, *lighting);
            screen_pixel<float>(tr, *lighting, *camera, width, height, frame, max_vertices, px, py, out + 4 * (size_t)i);
            unit_counts[i] = tr.cnt;
        }
    });
    for (auto& c : unit_counts) add_counts(counts, c);
    return 0;
}

int oracle_trace_texels(void* sp, const OracleLighting* lighting, uint8_t* slots, uint32_t payload_count,
                        const uint32_t* face_infos, uint32_t face_count, const uint32_t* instance_infos,
                        const uint32_t* side_infos, uint32_t instance_count, const uint32_t* units, int unit_count,
                        uint32_t iteration, uint32_t spt, uint32_t max_bounces, int reset, int precision, int threads,
                        OracleRayCounts* counts) {
    Scene* s = static_cast<Scene*>(sp);
    (void)face_count;
    std::vector<OracleRayCounts> unit_counts((size_t)unit_count);
    std::atomic<int> bad{0};
    parallel_for(unit_count, threads, [&](int u, int) {
        uint32_t inst_index = units[2 * u], local = units[2 * u + 1];
        if (inst_index >= instance_count) { bad = 1; return; }
        InstInfo inst{instance_infos[4 * inst_index], instance_infos[4 * inst_index + 1],
                      instance_infos[4 * inst_index + 2], instance_infos[4 * inst_index + 3]};
        uint32_t back_offset = side_infos[2 * inst_index], side_flags = side_infos[2 * inst_index + 1];
        if (local >= inst.texel_count) return;
        FaceInfo face;
        uint32_t prim;
        if (!find_face(face_infos, inst, local, &face, &prim)) return;
        uint32_t global_texel = inst.texel_offset + local;
        uint32_t i, j;
        address_to_ij(local - face.address, face.resolution, &i, &j);
        float rf = (float)face.resolution;
        float base_x = (float)i / rf, base_y = (float)j / rf;
        uint32_t n = std::max(spt, 1u);
        Rng rng(global_texel, inst_index, iteration * n);
        float bx = base_x, by = base_y;
        for (uint32_t attempt = 0; attempt < 32; ++attempt) {
            float r0 = rng.next_1d(), r1 = rng.next_1d();
            float cx = base_x + (r0 - 0.5f) / rf;
            float cy = base_y + (r1 - 0.5f) / rf;
            if (cx < 0.0f || cy < 0.0f || cx + cy > 1.0f) continue;
            if (nearest_texel(cx, cy, (1.0f - cx) - cy, inst, face) == global_texel) {
                bx = cx;
                by = cy;
                break;
            }
        }
        float hb1 = by, hb2 = std::max(0.0f, (1.0f - bx) - by);
        bool two = (side_flags & 1u) != 0;
        float front[3], back[3];
        auto run = [&](auto tag) {
            using T = decltype(tag);
            Tracer<T> tr(*s, *lighting);
            V3<T> fnrm = world_flat_normal<T>(*s, inst_index, prim);
            V3<T> f = ts_estimate<T>(tr, inst_index, prim, T(hb1), T(hb2), fnrm, n, rng, max_bounces);
            front[0] = (float)f.x; front[1] = (float)f.y; front[2] = (float)f.z;
            if (two) {
                V3<T> b = ts_estimate<T>(tr, inst_index, prim, T(hb1), T(hb2), -fnrm, n, rng, max_bounces);
                back[0] = (float)b.x; back[1] = (float)b.y; back[2] = (float)b.z;
            }
            unit_counts[u] = tr.cnt;
        };
        if (precision == ORACLE_F64) run(double(0)); else run(float(0));
        if (global_texel >= payload_count) { bad = 1; return; }
        store_running_mean(slots, global_texel, front, reset != 0);
        if (two) {
            uint32_t bt = back_offset + (global_texel - inst.texel_offset);
            if (bt >= payload_count) { bad = 1; return; }
            store_running_mean(slots, bt, back, reset != 0);
        }
    });
    for (auto& c : unit_counts) add_counts(counts, c);
    if (bad) { g_error = "texel index out of range"; return 1; }
    return 0;
}

int oracle_resolve_mesh_colors(void* sp, const OracleLighting* lighting, const OracleCamera* camera, uint32_t width,
                               uint32_t height, const uint32_t* pixels, int pixel_count, const uint32_t* face_infos,
                               const uint32_t* instance_infos, const uint32_t* side_infos, uint32_t instance_count,
                               const void* colors, int packed, int precision, int threads, float* out) {
    Scene* s = static_cast<Scene*>(sp);
    parallel_for(pixel_count, threads, [&](int i, int) {
        uint32_t px = pixels[2 * i], py = pixels[2 * i + 1];
        if (precision == ORACLE_F64) {
            Tracer<double> tr(*s, *lighting);
            resolve_pixel<double>(tr, *camera, width, height, px, py, face_infos, instance_infos, side_infos,
                                  instance_count, colors, packed != 0, out + 4 * (size_t)i);
        } else {
            Tracer<float> tr(*s, *lighting);
            resolve_pixel<float>(tr, *camera, width, height, px, py, face_infos, instance_infos, side_infos,
                                 instance_count, colors, packed != 0, out + 4 * (size_t)i);
        }
    });
    return 0;
}

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------
// Surface-probe resolve, surface_probe_resolve.slang:29-472 with the gather
// of surface_probes.slang:272-535 and surface_probe_irradiance_field.slang:
// 28-81, in float. lerp(a, b, t) = a + t (b - a); exp and log2 are spec_exp
// and spec_log2.
// ---------------------------------------------------------------------------
namespace probe_resolve {

constexpr uint32_t kMaxGather = 32, kMaxCandidates = 96, kStack = 64;
constexpr float kHardCos = 0.17364818f;
using F3 = V3<float>;

struct Layout {
    const float* probes;     // 12 floats per probe
    const uint32_t* nodes;   // 4 per node
    const float* instances;  // 12 floats per instance
    const uint32_t* tri_map; // 4 per record
    uint32_t probe_count, node_count, instance_count, tri_map_count;
    const float* values;
    const uint32_t* counts;
    const uint32_t* self_hits;
    const uint32_t* radial;
};

struct Instance {
    F3 center;
    float extent;
    uint32_t offsets[4];
    float kr, ncos, sigma;
    uint32_t map_offset;
};

struct Cands {
    uint32_t count = 0;
    uint32_t index[kMaxCandidates];
    float weight[kMaxCandidates];
};

struct Gath {
    uint32_t count = 0;
    uint32_t index[kMaxGather];
    float weight[kMaxGather];
};

float sat(float a) { return std::fmin(std::fmax(a, 0.0f), 1.0f); }
float lerpf(float a, float b, float t) { return a + t * (b - a); }
F3 lerp3(F3 a, F3 b, float t) { return a + t * (b - a); }
float smooth(float e0, float e1, float x) {
    float t = sat((x - e0) / (e1 - e0));
    return (t * t) * (3.0f - 2.0f * t);
}
F3 ppos(const Layout& l, uint32_t p) { return mk<float>(l.probes[12 * (size_t)p], l.probes[12 * (size_t)p + 1],
                                                        l.probes[12 * (size_t)p + 2]); }
F3 pnormal(const Layout& l, uint32_t p) { return mk<float>(l.probes[12 * (size_t)p + 4], l.probes[12 * (size_t)p + 5],
                                                           l.probes[12 * (size_t)p + 6]); }
float psupport(const Layout& l, uint32_t p) { return l.probes[12 * (size_t)p + 7]; }
F3 pirr(const Layout& l, uint32_t p) { return mk<float>(l.values[3 * (size_t)p], l.values[3 * (size_t)p + 1],
                                                        l.values[3 * (size_t)p + 2]); }

Instance load_instance(const Layout& l, uint32_t i) {
    const float* r = l.instances + 12 * (size_t)i;
    Instance v;
    v.center = mk<float>(r[0], r[1], r[2]);
    v.extent = r[3];
    std::memcpy(v.offsets, r + 4, 16);
    v.kr = r[8];
    v.ncos = r[9];
    v.sigma = r[10];
    std::memcpy(&v.map_offset, r + 11, 4);
    return v;
}

bool sphere_cube(F3 p, float r, F3 c, float e) {
    F3 a = mk<float>(std::fabs(p.x - c.x), std::fabs(p.y - c.y), std::fabs(p.z - c.z));
    F3 d = mk<float>(std::fmax(a.x - e, 0.0f), std::fmax(a.y - e, 0.0f), std::fmax(a.z - e, 0.0f));
    return dot(d, d) <= r * r;
}

float soft_normal(float nc, float full) {
    float end = std::fmax(full, kHardCos + 1e-3f);
    return smooth(kHardCos, end, nc) * std::fmax(nc, 0.0f);
}

// surface_probes.slang:272-392
void gather(const Layout& l, const Instance& ins, F3 q, F3 qn, float scale, Cands& out, bool* bad) {
    out.count = 0;
    float kr = std::fmax(ins.kr * std::fmax(scale, 1.0f), 1e-6f);
    float ps = std::fmax(ins.sigma, 1e-6f);
    float kr2 = kr * kr;
    uint32_t sn[kStack];
    F3 sc[kStack];
    float se[kStack];
    uint32_t n = 1;
    sn[0] = ins.offsets[0];
    sc[0] = ins.center;
    se[0] = ins.extent;
    while (n > 0) {
        n -= 1;
        uint32_t ni = sn[n];
        F3 c = sc[n];
        float e = se[n];
        if (!sphere_cube(q, kr, c, e)) continue;
        if (ni >= l.node_count) {
            *bad = true;
            continue;
        }
        const uint32_t* node = l.nodes + 4 * (size_t)ni;
        if (node[1] == 0) {
            if (node[2] > l.probe_count || node[3] > l.probe_count - node[2]) {
                *bad = true;
                continue;
            }
            for (uint32_t k = 0; k < node[3]; ++k) {
                uint32_t p = node[2] + k;
                F3 delta = ppos(l, p) - q;
                float d2 = dot(delta, delta);
                if (d2 > kr2) continue;
                float nc = dot(qn, normalize(pnormal(l, p)));
                if (nc < kHardCos) continue;
                float pd = std::fabs(dot(delta, qn));
                float pw = spec_exp((-0.5f * (pd / ps)) * (pd / ps));
                float sp = std::fmax(1.0f - d2 / kr2, 0.0f);
                float w = ((sp * sp) * pw) * soft_normal(nc, ins.ncos);
                if (w <= 1e-6f) continue;
                if (out.count < kMaxCandidates) {
                    out.index[out.count] = p;
                    out.weight[out.count] = w;
                    out.count += 1;
                } else {
                    uint32_t weakest = 0;
                    for (uint32_t i = 1; i < kMaxCandidates; ++i)
                        if (out.weight[i] < out.weight[weakest]) weakest = i;
                    if (w > out.weight[weakest]) {
                        out.index[weakest] = p;
                        out.weight[weakest] = w;
                    }
                }
            }
            continue;
        }
        float ce = e * 0.5f;
        uint32_t compact = 0;
        for (uint32_t o = 0; o < 8; ++o) {
            if (!(node[1] & (1u << o))) continue;
            F3 off = mk<float>((o & 1) ? 1.0f : -1.0f, (o & 2) ? 1.0f : -1.0f, (o & 4) ? 1.0f : -1.0f);
            F3 cc = c + off * ce;
            if (sphere_cube(q, kr, cc, ce) && n < kStack) {
                sn[n] = node[0] + compact;
                sc[n] = cc;
                se[n] = ce;
                n += 1;
            }
            compact += 1;
        }
    }
}

float half_bits_to_float(uint32_t h) { return f16_to_f32((uint16_t)h); }

// surface_probes.slang:134-155, 201-244, 462-535
void hemi_oct(F3 d, float* u, float* v) {
    F3 h = mk<float>(d.x, d.y, std::fmax(d.z, 0.0f));
    float l2 = dot(h, h);
    if (l2 <= 1e-12f) {
        *u = *v = 0.5f;
        return;
    }
    h = h * (1.0f / std::sqrt(l2));
    float inv_l1 = 1.0f / std::fmax((std::fabs(h.x) + std::fabs(h.y)) + h.z, 1e-6f);
    float ox = h.x * inv_l1, oy = h.y * inv_l1;
    *u = sat((ox + oy) * 0.5f + 0.5f);
    *v = sat((ox - oy) * 0.5f + 0.5f);
}

float visibility(const Layout& l, uint32_t p, F3 q, float kr, uint32_t sample_count, bool enabled) {
    if (!enabled) return 1.0f;
    F3 delta = q - ppos(l, p);
    float dist = std::sqrt(dot(delta, delta));
    if (dist <= 1e-6f) return 1.0f;
    F3 dl = mk<float>(delta.x / dist, delta.y / dist, delta.z / dist);
    F3 local = Frame<float>(normalize(pnormal(l, p))).to_local(dl);
    float nd = std::fmin(dist / std::fmax(kr, 1e-6f), 2.0f);
    float u, v;
    hemi_oct(local, &u, &v);
    float tx = sat(u) * 4.0f - 0.5f, ty = sat(v) * 4.0f - 0.5f;
    float fx = std::floor(tx), fy = std::floor(ty);
    int bx = (int)fx, by = (int)fy;
    float ax = tx - fx, ay = ty - fy;
    auto cl = [](int a) { return std::max(std::min(a, 3), 0); };
    int x0 = cl(bx), x1 = cl(bx + 1), y0 = cl(by), y1 = cl(by + 1);
    float w[4] = {(1.0f - ax) * (1.0f - ay), ax * (1.0f - ay), (1.0f - ax) * ay, ax * ay};
    int t[4] = {y0 * 4 + x0, y0 * 4 + x1, y1 * 4 + x0, y1 * 4 + x1};
    float mx = 0.0f, my = 0.0f, vw = 0.0f;
    for (int i = 0; i < 4; ++i) {
        uint32_t packed = l.radial[16 * (size_t)p + t[i]];
        float sx = half_bits_to_float(packed & 0xffffu), sy = half_bits_to_float(packed >> 16);
        if (sy > 0.0f) {
            mx = mx + sx * w[i];
            my = my + sy * w[i];
            vw = vw + w[i];
        }
    }
    if (vw <= 1e-6f) return 1.0f;
    mx = mx / vw;
    my = my / vw;
    float vis = 1.0f;
    if (my > 0.0f) {
        float mean = std::fmax(mx, 0.0f);
        if (!(nd <= mean + 0.035f)) {
            float var = std::fmax(my - mean * mean, 2.5e-3f);
            float diff = nd - mean;
            float prob = var / (var + diff * diff);
            vis = std::fmax(sat((prob - 0.2f) / 0.8f), 0.05f);
        }
    }
    float tc = sat((float)sample_count / 32.0f);
    return lerpf(1.0f, vis, 0.75f * tc);
}

void select(const Cands& c, Gath& out) {
    out.count = 0;
    uint32_t used[3] = {0, 0, 0};
    for (uint32_t sel = 0; sel < c.count && out.count < kMaxGather; ++sel) {
        uint32_t best = 0;
        float bw = -1.0f;
        for (uint32_t i = 0; i < c.count; ++i) {
            bool consumed = (used[i >> 5] >> (i & 31u)) & 1u;
            if (!consumed && c.weight[i] > bw) {
                best = i;
                bw = c.weight[i];
            }
        }
        used[best >> 5] |= 1u << (best & 31u);
        out.index[out.count] = c.index[best];
        out.weight[out.count] = bw;
        out.count += 1;
    }
}

void merge(const Gath& fb, float scale, Gath& g) {
    for (uint32_t k = 0; k < fb.count; ++k) {
        bool dup = false;
        for (uint32_t i = 0; i < g.count; ++i)
            if (g.index[i] == fb.index[k]) {
                dup = true;
                break;
            }
        if (dup) continue;
        float w = fb.weight[k] * scale;
        if (w <= 1e-8f) continue;
        if (g.count < kMaxGather) {
            g.index[g.count] = fb.index[k];
            g.weight[g.count] = w;
            g.count += 1;
        } else {
            uint32_t weakest = 0;
            for (uint32_t i = 1; i < g.count; ++i)
                if (g.weight[i] < g.weight[weakest]) weakest = i;
            if (w > g.weight[weakest]) {
                g.index[weakest] = fb.index[k];
                g.weight[weakest] = w;
            }
        }
    }
}

float ess(const Gath& g) {
    float s = 0.0f, s2 = 0.0f;
    for (uint32_t i = 0; i < g.count; ++i) {
        float w = std::fmax(g.weight[i], 0.0f);
        s = s + w;
        s2 = s2 + w * w;
    }
    return s2 > 1e-12f ? (s * s) / s2 : 0.0f;
}

struct Recon {
    F3 irradiance;
    uint32_t gathered;
    float support, weight_sum, ess, self_hit_rate;
};

void weigh(const Layout& l, Cands& c, F3 q, float kr, bool radial) {
    for (uint32_t i = 0; i < c.count; ++i)
        c.weight[i] = c.weight[i] * visibility(l, c.index[i], q, kr, l.counts[c.index[i]], radial);
}

Recon reconstruct(const Layout& l, const Instance& ins, F3 q, F3 qn, uint32_t min_gather, bool radial, bool* bad) {
    Cands cand;
    Gath g;
    gather(l, ins, q, qn, 1.0f, cand, bad);
    weigh(l, cand, q, ins.kr, radial);
    select(cand, g);
    uint32_t mg = std::min(std::max(min_gather, 1u), 32u);
    float e0 = ess(g);
    float fs = smooth(0.0f, 1.0f, sat(((float)mg - e0) / (float)mg));
    if (fs > 1e-4f) {
        Gath fb;
        gather(l, ins, q, qn, 2.0f, cand, bad);
        weigh(l, cand, q, ins.kr, radial);
        select(cand, fb);
        merge(fb, 0.25f * fs, g);
    }
    Recon r;
    float shs = 0.0f, shw = 0.0f;
    for (uint32_t i = 0; i < g.count; ++i) {
        uint32_t p = g.index[i];
        uint32_t sc = l.counts[p];
        if (sc == 0) continue;
        float rate = (float)l.self_hits[p] / (float)sc;
        shs = shs + g.weight[i] * rate;
        shw = shw + g.weight[i];
    }
    r.self_hit_rate = shw > 1e-6f ? shs / shw : 0.0f;
    F3 acc = mk<float>(0, 0, 0), best = mk<float>(0, 0, 0);
    float ws = 0.0f, wss = 0.0f, ss = 0.0f, ssw = 0.0f, best_w = -1.0f;
    for (uint32_t i = 0; i < g.count; ++i) {
        uint32_t p = g.index[i];
        ss = ss + g.weight[i] * sat(psupport(l, p));
        ssw = ssw + g.weight[i];
        F3 irr = pirr(l, p);
        float conf = l.counts[p] > 0 ? 1.0f : 0.0f;
        float w = g.weight[i] * conf;
        acc = acc + w * irr;
        ws = ws + w;
        wss = wss + w * w;
        if (w > best_w) {
            best_w = w;
            best = irr;
        }
    }
    r.gathered = g.count;
    r.support = ssw > 1e-6f ? sat(ss / ssw) : 0.0f;
    r.weight_sum = ws;
    r.ess = wss > 1e-12f ? (ws * ws) / wss : 0.0f;
    if (ws > 1e-6f)
        r.irradiance = mk<float>(acc.x / ws, acc.y / ws, acc.z / ws);
    else if (best_w >= 0.0f)
        r.irradiance = best;
    else
        r.irradiance = mk<float>(0, 0, 0);
    return r;
}

F3 count_color(uint32_t n) {
    if (n == 0) return mk<float>(1, 0, 1);
    if (n < 4) return lerp3(mk<float>(1, 0, 0), mk<float>(1, 0.5f, 0), (float)(n - 1) / 3.0f);
    if (n < 8) return lerp3(mk<float>(1, 1, 0), mk<float>(0, 1, 0), (float)(n - 4) / 4.0f);
    if (n < 16) return lerp3(mk<float>(0, 1, 0), mk<float>(0, 1, 1), (float)(n - 8) / 8.0f);
    if (n < 24) return lerp3(mk<float>(0, 1, 1), mk<float>(0, 0, 1), (float)(n - 16) / 8.0f);
    return lerp3(mk<float>(0, 0, 1), mk<float>(1, 1, 1), (float)(std::min(n, 32u) - 24) / 8.0f);
}

F3 support_color(float s) {
    float v = sat(s);
    if (v < 0.25f) return lerp3(mk<float>(1, 0, 1), mk<float>(1, 0, 0), v * 4.0f);
    if (v < 0.5f) return lerp3(mk<float>(1, 0, 0), mk<float>(1, 1, 0), (v - 0.25f) * 4.0f);
    if (v < 0.75f) return lerp3(mk<float>(1, 1, 0), mk<float>(0, 1, 0), (v - 0.5f) * 4.0f);
    return lerp3(mk<float>(0, 1, 0), mk<float>(0, 0.25f, 1), (v - 0.75f) * 4.0f);
}

F3 density_color(float s, float maxd) {
    float mx = std::fmax(maxd, 1.0f);
    float density = std::fmin(mx, 1.0f / std::fmax(sat(s), 1.0f / mx));
    float normalized = mx > 1.0f ? spec_log2(density) / spec_log2(mx) : 0.0f;
    return support_color(1.0f - sat(normalized));
}

F3 self_hit_color(float rate) {
    if (rate <= 0.0f) return mk<float>(0, 0, 0.25f);
    float lr = spec_log2(std::fmax(rate, 1e-6f)) / spec_log2(10.0f);
    float v = sat((lr + 6.0f) / 5.0f);
    if (v < 1.0f / 3.0f) return lerp3(mk<float>(0, 0, 0.25f), mk<float>(0, 1, 1), v * 3.0f);
    if (v < 2.0f / 3.0f) return lerp3(mk<float>(0, 1, 1), mk<float>(1, 1, 0), (v - 1.0f / 3.0f) * 3.0f);
    return lerp3(mk<float>(1, 1, 0), mk<float>(1, 0, 0), (v - 2.0f / 3.0f) * 3.0f);
}

F3 decode_rgbm(uint32_t packed, float range) {
    float x = (float)(packed & 255u) / 255.0f, y = (float)((packed >> 8) & 255u) / 255.0f;
    float z = (float)((packed >> 16) & 255u) / 255.0f, w = (float)((packed >> 24) & 255u) / 255.0f;
    return (mk<float>(x, y, z) * w) * range;
}

}  // namespace probe_resolve

void resolve_probe_pixel(Tracer<float>& tr, const OracleCamera& cam, uint32_t w, uint32_t h, uint32_t px,
                         uint32_t py, const probe_resolve::Layout& l, const OracleProbeResolveOptions& o, float* out,
                         bool* bad) {
    using namespace probe_resolve;
    float pxf = ((float)px + 0.5f) / (float)w;
    float pyf = ((float)py + 0.5f) / (float)h;
    pxf = pxf + (-cam.jitter_x);
    pyf = pyf + cam.jitter_y;
    float nx = 2.0f * pxf + -1.0f;
    float ny = -2.0f * pyf + 1.0f;
    F3 U = load3<float>(cam.image_u), Vv = load3<float>(cam.image_v), W = load3<float>(cam.image_w);
    F3 dir = normalize((nx * U + ny * Vv) + W);
    float inv_cos = 1.0f / dot(normalize(W), dir);
    F3 org = load3<float>(cam.position);
    HitRec hit = tr.closest(org, dir, cam.near_clip * inv_cos, cam.far_clip * inv_cos);
    uint32_t view = std::min(o.debug_view, 7u);
    bool beauty = view == 0 || view == 6;
    auto put = [&](F3 c) {
        out[0] = c.x;
        out[1] = c.y;
        out[2] = c.z;
        out[3] = 1.0f;
    };
    if (!hit.valid) {
        F3 c = mk<float>(0.02f, 0.02f, 0.02f);
        if (beauty) {
            c = tr.L.sky_at(dir);
            if (tr.L.sun_disk) c = c + tr.sun_disk(dir);
        }
        put(c);
        return;
    }
    uint32_t inst = tr.s.flat_instance[hit.flat], prim = tr.s.flat_prim[hit.flat];
    float b1 = hit.b1, b2 = hit.b2;
    Shading<float> sd = shading_data<float>(tr.s, inst, prim, b1, b2, -dir);
    F3 sun = mk<float>(0, 0, 0);
    if (beauty) {
        Rng rng(px, py, o.frame_index);
        float ux = rng.next_1d();
        float uy = rng.next_1d();
        sun = tr.sun_nee(sd, ux, uy);
    }
    if (inst >= l.instance_count) {
        *bad = true;
        out[0] = out[1] = out[2] = out[3] = 0.0f;
        return;
    }
    Instance ins = load_instance(l, inst);
    if (ins.offsets[3] == 0) {
        put(beauty ? sd.emissive + sun : count_color(0));
        return;
    }
    Recon r = reconstruct(l, ins, sd.position, normalize(sd.face_normal), o.min_gather_count,
                          o.use_radial_visibility != 0, bad);
    uint32_t side = sd.back_side ? 1u : 0u;
    float b0 = (1.0f - b1) - b2;
    float bary[3] = {b0, b1, b2};
    F3 vertex_irr = mk<float>(0, 0, 0);
    bool has_fallback = false;
    if (o.use_vertex_fallback) {
        uint32_t rec = ins.map_offset + prim * 2u + side;
        if (rec >= l.tri_map_count) {
            *bad = true;
        } else {
            const uint32_t* a = l.tri_map + 4 * (size_t)rec;
            if (a[3] & 1u) {
                F3 acc = mk<float>(0, 0, 0);
                float avail = 0.0f;
                for (int c = 0; c < 3; ++c) {
                    if (a[c] >= l.probe_count) {
                        *bad = true;
                        continue;
                    }
                    if (l.counts[a[c]] == 0) continue;
                    acc = acc + bary[c] * pirr(l, a[c]);
                    avail = avail + bary[c];
                }
                if (avail > 1e-6f) {
                    vertex_irr = mk<float>(acc.x / avail, acc.y / avail, acc.z / avail);
                    has_fallback = true;
                }
            }
        }
    }
    float target = (float)std::min(std::max(o.min_gather_count, 1u), 32u);
    float conf = std::fmin(sat((float)r.gathered / target), sat(r.ess / target));
    if (r.weight_sum <= 1e-6f) conf = 0.0f;
    if (!has_fallback) conf = 1.0f;
    float fallback_weight = 1.0f - conf;
    F3 irr = lerp3(vertex_irr, r.irradiance, conf);
    if (view == 1) return put(count_color(r.gathered));
    if (view == 2) return put(support_color(r.support));
    if (view == 3) return put(density_color(r.support, o.max_density_multiplier));
    if (view == 4) return put(support_color(1.0f - fallback_weight));
    if (view == 5) return put(self_hit_color(r.self_hit_rate));
    bool has_vl = false;
    F3 vl = mk<float>(0, 0, 0);
    float vl_conf = 0.0f;
    float range = std::fmax(o.vertex_lighting_rgbm_range, 1.0f);
    if (o.vertex_lighting_rgbm) {
        uint32_t io = o.vertex_lighting_instance_offsets[2 * (size_t)inst];
        uint32_t rec = io + prim * 2u + side;
        if (rec >= o.vertex_lighting_triangle_record_count) {
            *bad = true;
        } else {
            const uint32_t* vv = o.vertex_lighting_triangle_map + 4 * (size_t)rec;
            if (vv[3] != 0) {
                uint32_t nv = o.vertex_lighting_vertex_count;
                if (vv[0] >= nv || vv[1] >= nv || vv[2] >= nv) {
                    *bad = true;
                } else {
                    const float* t = o.vertex_lighting_target;
                    vl = (b0 * decode_rgbm(o.vertex_lighting_rgbm[vv[0]], range) +
                          b1 * decode_rgbm(o.vertex_lighting_rgbm[vv[1]], range)) +
                         b2 * decode_rgbm(o.vertex_lighting_rgbm[vv[2]], range);
                    vl_conf = (b0 * t[4 * (size_t)vv[0] + 3] + b1 * t[4 * (size_t)vv[1] + 3]) +
                              b2 * t[4 * (size_t)vv[2] + 3];
                    has_vl = true;
                }
            }
        }
    }
    if (view == 6)
        return put(has_vl ? (sd.emissive + sun) + (sd.diffuse * Consts<float>::INV_PI) * vl : mk<float>(1, 0, 1));
    if (view == 7) return put(has_vl ? support_color(vl_conf) : mk<float>(1, 0, 1));
    if (o.use_vertex_lighting && has_vl) irr = vl;
    put((sd.emissive + sun) + (sd.diffuse * Consts<float>::INV_PI) * irr);
}

// ---------------------------------------------------------------------------
// Weighted sample elimination, surface_probes.py:897-985, run as the
// reference runs it: one candidate at a time, the largest weight first
// (lowest index on ties), with a max-heap and stale-entry versions. The
// neighbour test and contribution (1 - d/d_max)^8 are evaluated in float64 in
// the reference's order; each contribution is rounded to units of 2^-50 and
// the weights are integer sums of those units.
// ---------------------------------------------------------------------------
long long wse_contribution(const float* pos, const float* nrm, uint32_t i, uint32_t j, double d_max,
                           double plane_limit, double ncos) {
    const double dx = (double)pos[3 * j] - (double)pos[3 * i];
    const double dy = (double)pos[3 * j + 1] - (double)pos[3 * i + 1];
    const double dz = (double)pos[3 * j + 2] - (double)pos[3 * i + 2];
    const double d2 = (dx * dx + dy * dy) + dz * dz;
    if (!(d2 > 1e-20) || !(d2 < d_max * d_max)) return 0;
    const double nix = nrm[3 * i], niy = nrm[3 * i + 1], niz = nrm[3 * i + 2];
    const double njx = nrm[3 * j], njy = nrm[3 * j + 1], njz = nrm[3 * j + 2];
    const double ndot = (njx * nix + njy * niy) + njz * niz;
    if (!(ndot >= ncos)) return 0;
    const double pa = std::fabs((dx * nix + dy * niy) + dz * niz);
    const double pb = std::fabs((dx * njx + dy * njy) + dz * njz);
    if (!(pa <= plane_limit) || !(pb <= plane_limit)) return 0;
    const double base = std::fmax(1.0 - std::sqrt(d2) / d_max, 0.0);
    const double b2 = base * base;
    const double b4 = b2 * b2;
    return std::llrint((b4 * b4) * 1125899906842624.0);
}

// density == nullptr: one d_max for the whole set (weighted_sample_elimination,
// surface_probes.py:897-985). Otherwise the adaptive elimination
// (_adaptive_weighted_sample_elimination_python, :988-1088): candidate i has
// d_max_i = max(d_max / sqrt(density_i), 1e-6) and plane limit
// max(d_max_i * scale, 1e-8); j contributes to i's weight under i's own d_max,
// so the neighbour relation is one-sided and the removal of k lowers the
// weights of the candidates whose lists hold k.
bool wse_set(const float* pos, const float* nrm, const float* density, uint32_t begin, uint32_t end, uint32_t out,
             double d_max, double plane_scale, double ncos, uint8_t* keep, uint32_t* order) {
    const uint32_t n = end - begin;
    std::vector<double> dmax_of(n, d_max), plane_of(n);
    double cell_size = d_max;
    for (uint32_t k = 0; k < n; ++k) {
        if (density) dmax_of[k] = std::max(d_max / std::sqrt((double)density[begin + k]), 1e-6);
        plane_of[k] = std::max(dmax_of[k] * plane_scale, 1e-8);
        cell_size = density ? (k ? std::max(cell_size, dmax_of[k]) : dmax_of[k]) : d_max;
    }
    struct Key {
        long long x, y, z;
        bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
    };
    struct KeyHash {
        size_t operator()(const Key& k) const {
            return (size_t)(k.x * 73856093LL) ^ (size_t)(k.y * 19349663LL) ^ (size_t)(k.z * 83492791LL);
        }
    };
    const double inv = 1.0 / std::max(cell_size, 1e-8);
    std::unordered_map<Key, std::vector<uint32_t>, KeyHash> grid;
    std::vector<Key> cell(n);
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t i = begin + k;
        cell[k] = {(long long)std::floor((double)pos[3 * i] * inv), (long long)std::floor((double)pos[3 * i + 1] * inv),
                   (long long)std::floor((double)pos[3 * i + 2] * inv)};
        grid[cell[k]].push_back(i);
    }
    std::vector<std::vector<std::pair<uint32_t, long long>>> adj(n);
    std::vector<long long> w(n, 0);
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t i = begin + k;
        for (long long dz = -1; dz <= 1; ++dz)
            for (long long dy = -1; dy <= 1; ++dy)
                for (long long dx = -1; dx <= 1; ++dx) {
                    auto it = grid.find({cell[k].x + dx, cell[k].y + dy, cell[k].z + dz});
                    if (it == grid.end()) continue;
                    for (uint32_t j : it->second) {
                        if (j == i) continue;
                        const long long q = wse_contribution(pos, nrm, i, j, dmax_of[k], plane_of[k], ncos);
                        if (q <= 0) continue;
                        adj[k].push_back({j - begin, q});
                        w[k] += q;
                    }
                }
    }
    for (uint32_t k = 0; k < n; ++k)
        if (adj[k].size() > 8000) return false;  // the GPU's bound on integer weights
    // who loses weight when k goes: the candidates whose lists hold k
    std::vector<std::vector<std::pair<uint32_t, long long>>> out_adj;
    if (density) {
        out_adj.resize(n);
        for (uint32_t k = 0; k < n; ++k)
            for (auto [j, q] : adj[k]) out_adj[j].push_back({k, q});
    }
    const auto& losers = density ? out_adj : adj;
    std::vector<uint8_t> active(n, 1);
    std::vector<uint32_t> version(n, 0);
    // max-heap on (weight, -index); stale entries are skipped by version
    std::priority_queue<std::tuple<long long, long long, uint32_t>> heap;
    for (uint32_t k = 0; k < n; ++k) heap.push({w[k], -(long long)k, 0u});
    uint32_t remaining = n, step = 0;
    while (remaining > out && !heap.empty()) {
        auto [wk, neg, ver] = heap.top();
        heap.pop();
        const uint32_t k = (uint32_t)(-neg);
        if (!active[k] || version[k] != ver) continue;
        active[k] = 0;
        --remaining;
        if (order) order[begin + step] = begin + k;
        ++step;
        for (auto [j, q] : losers[k]) {
            if (!active[j]) continue;
            w[j] = std::max<long long>(0, w[j] - q);
            version[j] += 1;
            heap.push({w[j], -(long long)j, version[j]});
        }
        (void)wk;
    }
    for (uint32_t k = 0; k < n; ++k) keep[begin + k] = active[k];
    return true;
}

// Deficit repair, deficit_repair_python (surface_probe_sampler.py:990-1103)
// with the gather weights of _gather_weights_reference (:949-987) in float32,
// exp from spec_exp, and numpy's float64 pairwise sums for the diagnostics.
float repair_weight(const float* q, const float* qn, const float* p, const float* pn, float r2, float plane_sigma,
                    float span, float eps) {
    const float hard = 0.17364818f;
    const float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    const float d2 = (dx * dx + dy * dy) + dz * dz;
    const float nc = (pn[0] * qn[0] + pn[1] * qn[1]) + pn[2] * qn[2];
    if (!(d2 <= r2) || !(nc >= hard)) return 0.0f;
    const float pd = std::fabs((dx * qn[0] + dy * qn[1]) + dz * qn[2]);
    const float t = pd / plane_sigma;
    const float pw = spec_exp(-0.5f * (t * t));
    const float sp = std::fmax(1.0f - d2 / r2, 0.0f);
    const float g = std::fmin(std::fmax((nc - hard) / span, 0.0f), 1.0f);
    const float soft = ((g * g) * (3.0f - 2.0f * g)) * std::fmax(nc, 0.0f);
    const float w = ((sp * sp) * pw) * soft;
    return w > eps ? w : 0.0f;
}

double numpy_pairwise_sum(const float* v, uint32_t n, bool square) {
    auto at = [&](uint32_t i) { return square ? (double)(v[i] * v[i]) : (double)v[i]; };
    if (n < 8u) {
        double r = 0.0;
        for (uint32_t i = 0; i < n; ++i) r += at(i);
        return r;
    }
    double r[8];
    for (int j = 0; j < 8; ++j) r[j] = at(j);
    uint32_t i = 8;
    for (; i < n - (n % 8u); i += 8)
        for (int j = 0; j < 8; ++j) r[j] += at(i + j);
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += at(i);
    return res;
}

double numpy_pairwise_terms(const float* v, uint32_t n) {
    if (n <= 128u) return numpy_pairwise_sum(v, n, false);
    uint32_t n2 = n / 2u;
    n2 -= n2 % 8u;
    return numpy_pairwise_terms(v, n2) + numpy_pairwise_terms(v + n2, n - n2);
}

// np.sum(float32 array, dtype=float64): the cast runs through numpy's ufunc
// buffers of 8192 elements; each buffer is summed pairwise and the buffer
// sums are added in order.
double numpy_f32_sum_f64(const float* v, uint32_t n) {
    double total = 0.0;
    for (uint32_t s = 0; s < n; s += 8192u) total = total + numpy_pairwise_terms(v + s, std::min(8192u, n - s));
    return total;
}

}  // namespace

extern "C" {

// Audit/repair candidate filter, _deduplicate_audit_candidates and
// _exclude_selected_duplicates (surface_probes.py:782-832) as the C++ form
// computes them (surface_probe_sampler.cpp:1736-1997: float normal dot
// compared with the double threshold), one pass per set in index order.
int oracle_filter_audit_repair(const float* cp, const float* cn, const uint32_t* cs, uint32_t n, const float* bp,
                               const float* bn, const uint32_t* bs, uint32_t base_count, const uint32_t* selected,
                               uint32_t m, uint32_t set_count, const double* cell_sizes, double ncos,
                               uint32_t* audit, uint32_t* audit_count, uint32_t* repair, uint32_t* repair_count) {
    using Cell = std::array<long long, 4>;
    using Exact = std::array<uint32_t, 7>;
    std::map<Cell, std::vector<uint32_t>> reps;
    std::set<Exact> occupied;
    auto exact = [](const float* p, const float* nn, uint32_t set, uint32_t i) {
        Exact k{};
        k[0] = set;
        std::memcpy(k.data() + 1, p + 3 * (size_t)i, 12);
        std::memcpy(k.data() + 4, nn + 3 * (size_t)i, 12);
        return k;
    };
    for (uint32_t e = 0; e < m; ++e) {
        if (selected[e] >= base_count) return 1;
        occupied.insert(exact(bp, bn, bs ? bs[selected[e]] : 0u, selected[e]));
    }
    uint32_t na = 0, nr = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t set = cs ? cs[i] : 0u;
        if (set >= set_count) return 2;
        const double inv = 1.0 / std::max(cell_sizes[set], 1e-8);
        Cell c{(long long)set, (long long)std::floor((double)cp[3 * i] * inv),
               (long long)std::floor((double)cp[3 * i + 1] * inv), (long long)std::floor((double)cp[3 * i + 2] * inv)};
        auto& list = reps[c];
        const float* a = cn + 3 * (size_t)i;
        bool dup = false;
        for (uint32_t r : list) {
            const float* b = cn + 3 * (size_t)r;
            const float d = (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
            if ((double)d >= ncos) {
                dup = true;
                break;
            }
        }
        if (!dup) {
            list.push_back(i);
            audit[na++] = i;
        }
        if (occupied.insert(exact(cp, cn, set, i)).second) repair[nr++] = i;
    }
    *audit_count = na;
    *repair_count = nr;
    return 0;
}

// Support estimate, estimate_support_python (surface_probe_sampler.py:
// 1179-1260), brute force per query over the reference points of its
// instance in index order.
int oracle_estimate_support(const float* ref_p, const float* ref_n, const uint32_t* ref_i, const float* area,
                            uint32_t ref_count, const float* q_p, const float* q_n, const uint32_t* q_i,
                            uint32_t q_count, const float* radii, uint32_t instance_count,
                            float normal_cosine_threshold, float eps, float max_density, float* support_f,
                            float* density_m) {
    const double hard = 0.17364817766693041;
    const float hard_f = 0.17364818f;
    const float span = (float)(std::max((double)normal_cosine_threshold, hard + 1e-3) - hard);
    const double m = std::max(1.0, (double)max_density);
    for (uint32_t i = 0; i < q_count; ++i)
        if (q_i[i] >= instance_count) return 8;
    for (uint32_t j = 0; j < ref_count; ++j)
        if (ref_i[j] >= instance_count) return 8;
    parallel_for((int)q_count, 0, [&](int qi, int) {
        const uint32_t k = q_i[qi];
        const float r2 = radii[k] * radii[k];
        const float sigma = (float)std::max((double)radii[k] * 0.25, 1e-6);
        const float* q = q_p + 3 * (size_t)qi;
        const float* qn = q_n + 3 * (size_t)qi;
        std::vector<float> terms;
        for (uint32_t j = 0; j < ref_count; ++j) {
            if (ref_i[j] != k) continue;
            const float* p = ref_p + 3 * (size_t)j;
            const float* pn = ref_n + 3 * (size_t)j;
            const float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
            const float d2 = (dx * dx + dy * dy) + dz * dz;
            const float nc = (pn[0] * qn[0] + pn[1] * qn[1]) + pn[2] * qn[2];
            if (!(d2 <= r2) || !(nc >= hard_f)) continue;
            const float t = ((dx * qn[0] + dy * qn[1]) + dz * qn[2]) / sigma;
            const float pw = spec_exp(-0.5f * (t * t));
            const float sp = std::fmax(1.0f - d2 / r2, 0.0f);
            const float g = std::fmin(std::fmax((nc - hard_f) / span, 0.0f), 1.0f);
            const float soft = ((g * g) * (3.0f - 2.0f * g)) * std::fmax(nc, 0.0f);
            float kw = ((sp * sp) * pw) * soft;
            kw = kw > eps ? kw : 0.0f;
            terms.push_back(kw * area[j]);
        }
        const double support = numpy_f32_sum_f64(terms.data(), (uint32_t)terms.size());
        const double rr = (double)radii[k];
        const double flat = 3.141592653589793 * rr * rr / 3.0;
        const double v = std::fmin(std::fmax(support / std::fmax(flat, 1e-30), 0.0), 1.0);
        support_f[qi] = (float)v;
        density_m[qi] = (float)std::fmin(m, 1.0 / std::fmax(v, 1.0 / m));
    });
    return 0;
}

int oracle_deficit_repair(const float* base_p, const float* base_n, const uint32_t* base_i, uint32_t base_count,
                          const float* cand_p, const float* cand_n, const uint32_t* cand_i, uint32_t cand_count,
                          const float* audit_p, const float* audit_n, const uint32_t* audit_i, uint32_t audit_count,
                          const float* radii, uint32_t instance_count, uint32_t min_gather, uint32_t max_repair,
                          float normal_cosine_threshold, float eps, uint32_t* selected, uint32_t* repair_count,
                          uint32_t* counts_before, uint32_t* counts_after, float* sums_before, float* sums_after,
                          float* ess_before, float* ess_after) {
    const double hard = 0.17364817766693041;  // cos(80 degrees)
    const float span = (float)(std::max((double)normal_cosine_threshold, hard + 1e-3) - hard);
    auto params = [&](uint32_t k, float* r2, float* sigma) {
        *r2 = radii[k] * radii[k];
        *sigma = (float)std::max((double)radii[k] * 0.25, 1e-6);
    };
    for (uint32_t a = 0; a < audit_count; ++a)
        if (audit_i[a] >= instance_count) return 8;
    auto summarize = [&](const std::vector<uint32_t>& extra, uint32_t* counts, float* sums, float* ess) {
        for (uint32_t a = 0; a < audit_count; ++a) {
            const uint32_t k = audit_i[a];
            float r2, sigma;
            params(k, &r2, &sigma);
            std::vector<float> w;
            auto take = [&](const float* p, const float* n, const uint32_t* inst, uint32_t j) {
                if (inst[j] != k) return;
                const float v = repair_weight(audit_p + 3 * (size_t)a, audit_n + 3 * (size_t)a, p + 3 * (size_t)j,
                                              n + 3 * (size_t)j, r2, sigma, span, eps);
                if (v > 0.0f) w.push_back(v);
            };
            for (uint32_t j = 0; j < base_count; ++j) take(base_p, base_n, base_i, j);
            for (uint32_t j : extra) take(cand_p, cand_n, cand_i, j);
            std::stable_sort(w.begin(), w.end(), [](float x, float y) { return x > y; });
            const uint32_t n = (uint32_t)std::min<size_t>(w.size(), 32);
            counts[a] = n;
            const float s32 = (float)numpy_pairwise_sum(w.data(), n, false);
            const double sq = numpy_pairwise_sum(w.data(), n, true);
            sums[a] = s32;
            ess[a] = sq > 0.0 ? (float)(((double)s32 * (double)s32) / sq) : 0.0f;
        }
    };
    summarize({}, counts_before, sums_before, ess_before);
    std::vector<long long> deficit(audit_count);
    for (uint32_t a = 0; a < audit_count; ++a) deficit[a] = std::max<long long>((long long)min_gather - counts_before[a], 0);
    std::vector<std::vector<uint32_t>> coverage(cand_count);
    for (uint32_t c = 0; c < cand_count; ++c) {
        if (cand_i[c] >= instance_count) continue;
        for (uint32_t a = 0; a < audit_count; ++a) {
            if (deficit[a] <= 0 || audit_i[a] != cand_i[c]) continue;
            float r2, sigma;
            params(audit_i[a], &r2, &sigma);
            if (repair_weight(audit_p + 3 * (size_t)a, audit_n + 3 * (size_t)a, cand_p + 3 * (size_t)c,
                              cand_n + 3 * (size_t)c, r2, sigma, span, eps) > 0.0f)
                coverage[c].push_back(a);
        }
    }
    const uint32_t limit = std::min(max_repair, cand_count);
    std::vector<uint8_t> active(cand_count, 1);
    std::vector<uint32_t> chosen;
    while (chosen.size() < limit) {
        long long best_score = 0;
        int best = -1;
        for (uint32_t c = 0; c < cand_count; ++c) {
            if (!active[c]) continue;
            long long score = 0;
            for (uint32_t a : coverage[c])
                if (deficit[a] > 0) score += 2 * deficit[a] - 1;
            if (score > best_score) {
                best_score = score;
                best = (int)c;
            }
        }
        if (best < 0) break;
        active[best] = 0;
        chosen.push_back((uint32_t)best);
        for (uint32_t a : coverage[best]) deficit[a] = std::max<long long>(deficit[a] - 1, 0);
    }
    for (size_t r = 0; r < chosen.size(); ++r) selected[r] = chosen[r];
    *repair_count = (uint32_t)chosen.size();
    summarize(chosen, counts_after, sums_after, ess_after);
    return 0;
}

int oracle_wse_eliminate(const float* positions, const float* normals, const float* relative_densities,
                         const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                         const float* surface_areas, float normal_cosine_threshold, float plane_distance_scale,
                         uint8_t* keep, float* poisson_radii, uint32_t* order, int threads) {
    std::atomic<int> bad{0};
    parallel_for((int)set_count, threads, [&](int k, int) {
        const uint32_t b = set_offsets[k], e = set_offsets[k + 1];
        const uint32_t count = e - b;
        const uint32_t out = std::max(1u, std::min(output_counts[k], std::max(count, 1u)));
        const double area = std::max((double)surface_areas[k], 1e-20);
        const double r = std::sqrt(area / (2.0 * std::sqrt(3.0) * (double)out));
        const double d_max = std::max(2.0 * r, 1e-6);
        if (poisson_radii)
            poisson_radii[k] = relative_densities ? (float)r
                               : count == out     ? (float)std::sqrt(area / out)
                                                  : (float)(d_max * 0.5);
        if (!wse_set(positions, normals, relative_densities, b, e, out, d_max, (double)plane_distance_scale,
                     (double)normal_cosine_threshold, keep, order))
            bad = 1;
    });
    return bad.load() ? 3 : 0;
}

float own_exp(float x) { return spec_exp(x); }
float own_log2(float x) { return spec_log2(x); }

int oracle_resolve_probes(void* sp, const OracleLighting* lighting, const OracleCamera* camera, uint32_t width,
                          uint32_t height, const uint32_t* pixels, int pixel_count, const float* probes,
                          uint32_t probe_count, const uint32_t* nodes, uint32_t node_count, const float* instances,
                          uint32_t instance_count, const uint32_t* triangle_vertex_probes,
                          uint32_t triangle_vertex_probe_count, const float* values, const uint32_t* sample_counts,
                          const uint32_t* self_hits, const uint32_t* radial, const OracleProbeResolveOptions* options,
                          int threads, float* out) {
    Scene* s = static_cast<Scene*>(sp);
    probe_resolve::Layout l{probes, nodes, instances, triangle_vertex_probes, probe_count, node_count,
                            instance_count, triangle_vertex_probe_count, values, sample_counts, self_hits, radial};
    std::atomic<int> bad{0};
    parallel_for(pixel_count, threads, [&](int i, int) {
        Tracer<float> tr(*s, *lighting);
        bool b = false;
        resolve_probe_pixel(tr, *camera, width, height, pixels[2 * i], pixels[2 * i + 1], l, *options,
                            out + 4 * (size_t)i, &b);
        if (b) bad = 1;
    });
    return bad.load() ? 4 : 0;
}

int oracle_filter_mesh_colors(const uint32_t* face_infos, const uint32_t* instance_infos, const uint32_t* side_infos,
                              uint32_t instance_count, const uint32_t* adjacency, const float* face_normals,
                              const uint8_t* source, uint8_t* destination, float neighbor_weight, float sigma,
                              int threads) {
    std::vector<std::pair<uint32_t, uint32_t>> units;
    for (uint32_t k = 0; k < instance_count; ++k)
        for (uint32_t t = 0; t < instance_infos[4 * k + 3]; ++t) units.emplace_back(k, t);
    parallel_for((int)units.size(), threads, [&](int u, int) {
        uint32_t k = units[u].first;
        InstInfo ii{instance_infos[4 * k], instance_infos[4 * k + 1], instance_infos[4 * k + 2],
                    instance_infos[4 * k + 3]};
        surface_filter_texel(face_infos, ii, side_infos[2 * k], side_infos[2 * k + 1], adjacency, face_normals,
                             source, destination, units[u].second, neighbor_weight, sigma);
    });
    return 0;
}

int oracle_trace_probes_prt(void* sp, const OracleLighting* lighting, float* values, uint32_t* sample_counts,
                            uint32_t* self_hits, uint32_t* radial, float* static_source, const uint8_t* probes,
                            uint32_t probe_count, const uint8_t* probe_instances, const uint32_t* units,
                            int unit_count, uint32_t iteration, uint32_t spp, uint32_t max_bounces, int reset,
                            int precision, int threads) {
    Scene* s = static_cast<Scene*>(sp);
    ProbeBuffers b{values, sample_counts, self_hits, radial};
    parallel_for(unit_count, threads, [&](int u, int) {
        uint32_t p = units[u];
        if (p >= probe_count) return;
        if (precision == ORACLE_F64) {
            Tracer<double> tr(*s, *lighting);
            probe_prt_unit<double>(tr, b, static_source, probes, probe_instances, p, iteration, spp, max_bounces,
                                   reset != 0);
        } else {
            Tracer<float> tr(*s, *lighting);
            probe_prt_unit<float>(tr, b, static_source, probes, probe_instances, p, iteration, spp, max_bounces,
                                  reset != 0);
        }
    });
    return 0;
}

// PRT evaluation, surface_probe_prt_evaluate.slang:20-103: SH L2 projection
// of the escape radiance (the sky term) by the quasi-random sphere rule
// y = 1 - 2 (i + 0.5) / n, phi = 2 pi radical_inverse(i), summed in order;
// then static + sum_c T_c L_c clamped at 0 per probe.
static uint32_t reverse_bits32(uint32_t b) {
    b = (b << 16u) | (b >> 16u);
    b = ((b & 0x55555555u) << 1u) | ((b & 0xAAAAAAAAu) >> 1u);
    b = ((b & 0x33333333u) << 2u) | ((b & 0xCCCCCCCCu) >> 2u);
    b = ((b & 0x0F0F0F0Fu) << 4u) | ((b & 0xF0F0F0F0u) >> 4u);
    b = ((b & 0x00FF00FFu) << 8u) | ((b & 0xFF00FF00u) >> 8u);
    return b;
}

void oracle_prt_project_lighting(const OracleLighting* lighting, uint32_t sample_count, float* sh) {
    LightCtx<float> L(*lighting);
    const uint32_t n = std::max(sample_count, 1u);
    for (uint32_t c = 0; c < 9; ++c) {
        V3<float> acc = mk<float>(0.0f, 0.0f, 0.0f);
        for (uint32_t i = 0; i < n; ++i) {
            const float u = ((float)i + 0.5f) / (float)n;
            const float v = (float)reverse_bits32(i) * 2.3283064365386963e-10f;
            const float y = 1.0f - 2.0f * u;
            const float r = std::sqrt(std::fmax(1.0f - y * y, 0.0f));
            float sn, cs;
            own_sincos(6.28318530717958647692f * v, &sn, &cs);
            const V3<float> dd = mk<float>(r * cs, y, r * sn);
            acc = acc + L.sky_at(dd) * sh_l2_basis<float>(c, dd);
        }
        acc = acc * ((4.0f * 3.14159265358979323846f) / (float)n);
        sh[4 * c] = acc.x;
        sh[4 * c + 1] = acc.y;
        sh[4 * c + 2] = acc.z;
        sh[4 * c + 3] = 0.0f;
    }
}

void oracle_prt_evaluate(const float* values, const uint32_t* sample_counts, const float* static_source,
                         const float* sh, float* out, uint32_t* out_counts, uint32_t probe_count) {
    for (uint32_t p = 0; p < probe_count; ++p) {
        float e[3] = {static_source[3 * p], static_source[3 * p + 1], static_source[3 * p + 2]};
        if (sample_counts[p] > 0u)
            for (int c = 0; c < 9; ++c)
                for (int k = 0; k < 3; ++k) e[k] = e[k] + values[27 * (size_t)p + 3 * c + k] * sh[4 * c + k];
        for (int k = 0; k < 3; ++k) out[3 * p + k] = std::fmax(e[k], 0.0f);
        out_counts[p] = sample_counts[p];
    }
}

void oracle_scene_set_area_lights(void* sp, const float* lights, int count, float power) {
    Scene* s = static_cast<Scene*>(sp);
    s->lights.assign(lights, lights + 16 * (size_t)std::max(count, 0));
    s->light_power = power;
}

int oracle_trace_points(void* sp, const OracleLighting* lighting, const float* points, int count,
                        uint32_t iteration, uint32_t samples, uint32_t max_bounces, uint32_t flags, float* out,
                        int precision, int threads, OracleRayCounts* counts) {
    Scene* s = static_cast<Scene*>(sp);
    std::vector<OracleRayCounts> unit_counts((size_t)count);
    std::atomic<int> bad{0};
    parallel_for(count, threads, [&](int u, int) {
        float* o = out + 4 * (size_t)u;
        uint32_t inst, primw;
        std::memcpy(&inst, points + 4 * (size_t)u + 2, 4);
        std::memcpy(&primw, points + 4 * (size_t)u + 3, 4);
        o[0] = o[1] = o[2] = 0.0f;
        o[3] = -1.0f;
        if (inst == 0xffffffffu) return;
        const uint32_t prim = primw & 0x7fffffffu;
        const bool back = (primw >> 31) != 0;
        if ((size_t)inst * 4 >= s->instance_descs.size() ||
            prim >= s->mesh_descs[4 * (size_t)s->instance_descs[4 * (size_t)inst] + 1] / 3u) {
            bad = 1;
            return;
        }
        const float b1 = points[4 * (size_t)u], b2 = points[4 * (size_t)u + 1];
        const uint32_t n = std::max(samples, 1u);
        Rng rng((uint32_t)u, 0xffffffffu, iteration * n);
        auto run = [&](auto tag) {
            using T = decltype(tag);
            Tracer<T> tr(*s, *lighting);
            V3<T> view = world_flat_normal<T>(*s, inst, prim);
            if (back) view = -view;
            V3<T> e = ts_estimate<T>(tr, inst, prim, T(b1), T(b2), view, n, rng, max_bounces, (flags & 1u) == 0u);
            o[0] = (float)e.x; o[1] = (float)e.y; o[2] = (float)e.z; o[3] = 0.0f;
            unit_counts[u] = tr.cnt;
        };
        if (precision == ORACLE_F64) run(double(0)); else run(float(0));
    });
    for (auto& c : unit_counts) add_counts(counts, c);
    if (bad) { g_error = "point names a triangle outside the scene"; return 1; }
    return 0;
}

static int trace_probes_impl(void* sp, const OracleLighting* lighting, float* values, uint32_t* sample_counts,
                             uint32_t* self_hits, uint32_t* radial, const uint8_t* probes, uint32_t probe_count,
                             const uint8_t* probe_instances, const uint32_t* units, int unit_count,
                             uint32_t iteration, uint32_t spp, uint32_t max_bounces, int reset, int precision,
                             int threads, OracleRayCounts* counts, bool independent) {
    Scene* s = static_cast<Scene*>(sp);
    ProbeBuffers b{values, sample_counts, self_hits, radial};
    std::vector<OracleRayCounts> unit_counts((size_t)unit_count);
    parallel_for(unit_count, threads, [&](int u, int) {
        uint32_t p = units[u];
        if (p >= probe_count) return;
        if (precision == ORACLE_F64) {
            Tracer<double> tr(*s, *lighting);
            probe_unit<double>(tr, b, probes, probe_instances, p, iteration, spp, max_bounces, reset != 0,
                               independent);
            unit_counts[u] = tr.cnt;
        } else {
            Tracer<float> tr(*s, *lighting);
            probe_unit<float>(tr, b, probes, probe_instances, p, iteration, spp, max_bounces, reset != 0,
                              independent);
            unit_counts[u] = tr.cnt;
        }
    });
    for (auto& c : unit_counts) add_counts(counts, c);
    return 0;
}

int oracle_trace_probes(void* sp, const OracleLighting* lighting, float* values, uint32_t* sample_counts,
                        uint32_t* self_hits, uint32_t* radial, const uint8_t* probes, uint32_t probe_count,
                        const uint8_t* probe_instances, uint32_t probe_instance_count, const uint32_t* units,
                        int unit_count, uint32_t iteration, uint32_t spp, uint32_t max_bounces, int reset,
                        int precision, int threads, OracleRayCounts* counts) {
    (void)probe_instance_count;
    return trace_probes_impl(sp, lighting, values, sample_counts, self_hits, radial, probes, probe_count,
                             probe_instances, units, unit_count, iteration, spp, max_bounces, reset, precision,
                             threads, counts, false);
}

int oracle_trace_probes_independent(void* sp, const OracleLighting* lighting, float* values,
                                    uint32_t* sample_counts, uint32_t* self_hits, uint32_t* radial,
                                    const uint8_t* probes, uint32_t probe_count, const uint8_t* probe_instances,
                                    uint32_t probe_instance_count, const uint32_t* units, int unit_count,
                                    uint32_t iteration, uint32_t spp, uint32_t max_bounces, int reset,
                                    int precision, int threads, OracleRayCounts* counts) {
    (void)probe_instance_count;
    return trace_probes_impl(sp, lighting, values, sample_counts, self_hits, radial, probes, probe_count,
                             probe_instances, units, unit_count, iteration, spp, max_bounces, reset, precision,
                             threads, counts, true);
}

}  // extern "C"

// ===========================================================================
// Restatement of this library's default BVH builder (nan_bvh.cu, k_sah_* and
// the collapse/emission that follow it). This is the library's own
// algorithm, not the reference's: the reference leaves the BVH to the
// driver. It pins the GPU builder's tree through its node count and SAH cost.
//   * top-down binned SAH: 32 bins of each node's centroid bounds per axis,
//     cost = left half-area x left count + right half-area x right count,
//     the first minimum over axes 0..2 and bins 0..30; a node whose
//     centroids coincide on every axis halves its range; split down to
//     single triangles; stable partitions;
//   * bottom-up collapse (k_subtree): a subtree of at most 3 triangles becomes
//     one leaf when tris <= 1 + (aa ca + ab cb) / ap (C_trav = C_int = 1);
//   * cost sum (k_emit_dfs): per kept interior node its half-area / the
//     root's, plus each leaf child's half-area / the root's x its triangles.
// ===========================================================================
namespace {

struct SahBox {
    float lo[3], hi[3];
};

float sah_half_area_f(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float dx = hx - lx, dy = hy - ly, dz = hz - lz;
    if (!(dx >= 0.0f)) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

float sah_half_area4(const SahBox& b) {  // half_area4: no empty-box test
    const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return x * y + y * z + z * x;
}

int sah_bin_of(float c, float lo, float hi) {
    const float ext = hi - lo;
    if (!(ext > 0.0f)) return 0;
    const float scale = 32.0f / ext;
    const int b = (int)((c - lo) * scale);
    return std::min(std::max(b, 0), 31);
}

}  // namespace

extern "C" {

// tris9: n world triangles (9 floats each, the flattened order). out3 =
// (kept interior nodes, unused, SAH cost).
int oracle_sah_build_stats(const float* tris9, uint32_t n, double* out3) {
    out3[0] = out3[1] = out3[2] = 0.0;
    if (n == 0) return 0;
    std::vector<SahBox> box(n);
    std::vector<float> cent(3 * (size_t)n);
    for (uint32_t t = 0; t < n; ++t) {
        for (int a = 0; a < 3; ++a) {
            const float v0 = tris9[9 * (size_t)t + a], v1 = tris9[9 * (size_t)t + 3 + a], v2 = tris9[9 * (size_t)t + 6 + a];
            box[t].lo[a] = std::min(std::min(v0, v1), v2);
            box[t].hi[a] = std::max(std::max(v0, v1), v2);
            cent[3 * (size_t)t + a] = 0.5f * (box[t].lo[a] + box[t].hi[a]);
        }
    }
    if (n == 1) {
        out3[2] = 1.0;
        return 0;
    }
    // binary tree down to single triangles: child refs, >= 0 interior, ~t leaf
    std::vector<std::array<int, 2>> child;
    std::vector<SahBox> nbox;
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; ++i) ids[i] = i;
    child.reserve(n - 1);
    nbox.reserve(n - 1);
    struct Item {
        uint32_t first, count;
        int node;
    };
    child.push_back({0, 0});
    nbox.push_back(SahBox{});
    std::vector<Item> stack{{0u, n, 0}};
    std::vector<uint32_t> tmp;
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        SahBox b, cb;
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = cb.lo[a] = INFINITY;
            b.hi[a] = cb.hi[a] = -INFINITY;
        }
        for (uint32_t k = 0; k < it.count; ++k) {
            const uint32_t p = ids[it.first + k];
            for (int a = 0; a < 3; ++a) {
                b.lo[a] = std::min(b.lo[a], box[p].lo[a]);
                b.hi[a] = std::max(b.hi[a], box[p].hi[a]);
                cb.lo[a] = std::min(cb.lo[a], cent[3 * (size_t)p + a]);
                cb.hi[a] = std::max(cb.hi[a], cent[3 * (size_t)p + a]);
            }
        }
        nbox[it.node] = b;
        float best_cost = INFINITY;
        int best_axis = -1, best_bin = 0;
        for (int a = 0; a < 3; ++a) {
            if (!(cb.hi[a] - cb.lo[a] > 0.0f)) continue;
            SahBox bins[32];
            uint32_t nb[32] = {0};
            for (auto& x : bins)
                for (int k = 0; k < 3; ++k) {
                    x.lo[k] = INFINITY;
                    x.hi[k] = -INFINITY;
                }
            for (uint32_t k = 0; k < it.count; ++k) {
                const uint32_t p = ids[it.first + k];
                const int bi = sah_bin_of(cent[3 * (size_t)p + a], cb.lo[a], cb.hi[a]);
                nb[bi]++;
                for (int q = 0; q < 3; ++q) {
                    bins[bi].lo[q] = std::min(bins[bi].lo[q], box[p].lo[q]);
                    bins[bi].hi[q] = std::max(bins[bi].hi[q], box[p].hi[q]);
                }
            }
            float right_area[32];
            uint32_t right_n[32];
            float rl[3] = {INFINITY, INFINITY, INFINITY}, rh[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t rn = 0;
            for (int bi = 31; bi >= 1; --bi) {
                for (int q = 0; q < 3; ++q) {
                    rl[q] = std::min(rl[q], bins[bi].lo[q]);
                    rh[q] = std::max(rh[q], bins[bi].hi[q]);
                }
                rn += nb[bi];
                right_area[bi] = sah_half_area_f(rl[0], rl[1], rl[2], rh[0], rh[1], rh[2]);
                right_n[bi] = rn;
            }
            float ll[3] = {INFINITY, INFINITY, INFINITY}, lh[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t ln = 0;
            for (int bi = 0; bi < 31; ++bi) {
                for (int q = 0; q < 3; ++q) {
                    ll[q] = std::min(ll[q], bins[bi].lo[q]);
                    lh[q] = std::max(lh[q], bins[bi].hi[q]);
                }
                ln += nb[bi];
                if (ln == 0 || right_n[bi + 1] == 0) continue;
                const float c = sah_half_area_f(ll[0], ll[1], ll[2], lh[0], lh[1], lh[2]) * (float)ln +
                                right_area[bi + 1] * (float)right_n[bi + 1];
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_bin = bi;
                }
            }
        }
        uint32_t left = it.count / 2;
        if (best_axis >= 0) {
            tmp.clear();
            left = 0;
            for (uint32_t k = 0; k < it.count; ++k) {
                const uint32_t p = ids[it.first + k];
                if (sah_bin_of(cent[3 * (size_t)p + best_axis], cb.lo[best_axis], cb.hi[best_axis]) <= best_bin)
                    ids[it.first + left++] = p;
                else
                    tmp.push_back(p);
            }
            for (size_t k = 0; k < tmp.size(); ++k) ids[it.first + left + k] = tmp[k];
        }
        const uint32_t counts[2] = {left, it.count - left};
        for (int s = 0; s < 2; ++s) {
            const uint32_t f = it.first + (s ? left : 0u);
            if (counts[s] == 1) {
                child[it.node][s] = ~(int)ids[f];
            } else {
                const int id = (int)child.size();
                child.push_back({0, 0});
                nbox.push_back(SahBox{});
                child[it.node][s] = id;
                stack.push_back({f, counts[s], id});
            }
        }
    }
    // collapse, bottom-up (children have larger ids than their parent)
    const size_t m = child.size();
    std::vector<uint32_t> tris(m);
    std::vector<float> cost(m);
    std::vector<char> collapsed(m);
    for (size_t i = m; i-- > 0;) {
        uint32_t t2[2];
        float c2[2], a2[2];
        for (int s = 0; s < 2; ++s) {
            const int c = child[i][s];
            if (c < 0) {
                t2[s] = 1;
                c2[s] = 1.0f;
                a2[s] = sah_half_area4(box[~c]);
            } else {
                t2[s] = tris[c];
                c2[s] = cost[c];
                a2[s] = sah_half_area4(nbox[c]);
            }
        }
        const float ap = std::max(sah_half_area4(nbox[i]), 1e-30f);
        const float split = 1.0f + (a2[0] * c2[0] + a2[1] * c2[1]) / ap;
        tris[i] = t2[0] + t2[1];
        if (tris[i] <= 3u && (float)tris[i] <= split) {
            cost[i] = (float)tris[i];
            collapsed[i] = 1;
        } else {
            cost[i] = split;
            collapsed[i] = 0;
        }
    }
    if (collapsed[0]) {
        out3[2] = (double)n;
        return 0;
    }
    const float root_area = std::max(sah_half_area4(nbox[0]), 1e-30f);
    double sah = 0.0, kept = 0.0;
    std::vector<int> walk{0};
    while (!walk.empty()) {
        const int i = walk.back();
        walk.pop_back();
        kept += 1.0;
        sah += (double)(sah_half_area4(nbox[i]) / root_area);
        for (int s = 0; s < 2; ++s) {
            const int c = child[i][s];
            if (c < 0) {
                sah += (double)(sah_half_area4(box[~c]) / root_area) * 1.0;
            } else if (collapsed[c]) {
                sah += (double)(sah_half_area4(nbox[c]) / root_area) * (double)tris[c];
            } else {
                walk.push_back(c);
            }
        }
    }
    out3[0] = kept;
    out3[2] = sah;
    return 0;
}

}  // extern "C"
