// pe_math.h — scalar/vector arithmetic shared by the host scene builder (g++) and the sm_100a
// kernels (nvcc).  Everything here is compiled without FMA contraction (-ffp-contract=off on the
// host, -fmad=false on the device) and written with the operand order of the reference's
// Vec3f (src/core/math/vec.h:111-157), so ray setup, triangle tests and hit records round
// exactly as the reference's CPU path does.  min/max/clamp follow std::min/std::max/std::clamp
// semantics, including what they return for NaN, which fminf/fmaxf do not.
#pragma once

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define PE_HD __host__ __device__ __forceinline__
// Large BSDF / light routines stay out of line on the device: the shading kernel runs many
// different ones in one warp and inlining them all overflows the instruction cache.
#define PE_HDN __host__ __device__ __noinline__
#else
#define PE_HD inline
#define PE_HDN inline
#endif

namespace pe {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 2.0f * kPi;
constexpr float kInvPi = 1.0f / kPi;
constexpr float kInvTwoPi = 1.0f / kTwoPi;
constexpr float kPiOver2 = kPi / 2.0f;
constexpr float kPiOver4 = kPi / 4.0f;
constexpr float kFltMax = 3.402823466e+38f; // the reference's INFINITY_F (constants.h)

// std::max(a, b) == (a < b) ? b : a ; std::min(a, b) == (b < a) ? b : a
PE_HD float smax(float a, float b) { return (a < b) ? b : a; }
PE_HD float smin(float a, float b) { return (b < a) ? b : a; }
PE_HD int imax(int a, int b) { return (a < b) ? b : a; }
PE_HD int imin(int a, int b) { return (b < a) ? b : a; }
PE_HD float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
PE_HD int iclamp(int v, int lo, int hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
PE_HD float smax3(float a, float b, float c) { return smax(smax(a, b), c); }

PE_HD uint32_t fbits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    union { float f; uint32_t u; } c; c.f = f; return c.u;
#endif
}
PE_HD float bitsf(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    union { float f; uint32_t u; } c; c.u = u; return c.f;
#endif
}
// Exponent test that no compiler flag can fold away (src/core/math/float_bits.h:19-21).
PE_HD bool finitef(float x) { return (fbits(x) & 0x7f800000u) != 0x7f800000u; }

// PBRT-v4 NextFloatUp / NextFloatDown (float_bits.h:29-48).
PE_HD float nextUp(float v) {
    if (!finitef(v) && v > 0.0f) return v;
    if (v == -0.0f) v = 0.0f;
    uint32_t ui = fbits(v);
    if (v >= 0.0f) ++ui; else --ui;
    return bitsf(ui);
}
PE_HD float nextDown(float v) {
    if (!finitef(v) && v < 0.0f) return v;
    if (v == 0.0f) v = -0.0f;
    uint32_t ui = fbits(v);
    if (v > 0.0f) --ui; else ++ui;
    return bitsf(ui);
}
// γ(n) = nε/(1 − nε), ε = 2^-24 (float_bits.h:53-56).
PE_HD float gammaN(int n) {
    const float eps = 5.9604645e-8f;
    return (static_cast<float>(n) * eps) / (1.0f - static_cast<float>(n) * eps);
}

struct V3 {
    float x, y, z;
};
struct V2 {
    float x, y;
};

PE_HD V3 mk(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
PE_HD V3 mk(float s) { return mk(s, s, s); }
PE_HD V2 mk2(float x, float y) { V2 r; r.x = x; r.y = y; return r; }
PE_HD V3 m3f(const float* p) { return mk(p[0], p[1], p[2]); }
PE_HD V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
PE_HD V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
PE_HD V3 operator*(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
PE_HD V3 operator/(V3 a, V3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
PE_HD V3 operator*(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
PE_HD V3 operator*(float s, V3 a) { return a * s; }
// Vec3f::operator/(float) multiplies by the reciprocal (vec.h:118).
PE_HD V3 operator/(V3 a, float s) { const float inv = 1.0f / s; return mk(a.x * inv, a.y * inv, a.z * inv); }
PE_HD V3 operator-(V3 a) { return mk(-a.x, -a.y, -a.z); }
PE_HD V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
PE_HD V3& operator*=(V3& a, V3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
PE_HD V3& operator*=(V3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }
PE_HD V3& operator/=(V3& a, float s) { const float inv = 1.0f / s; a.x *= inv; a.y *= inv; a.z *= inv; return a; }
PE_HD float get(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
PE_HD void set(V3& a, int i, float v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }

PE_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PE_HD V3 cross(V3 a, V3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
PE_HD float len2(V3 a) { return dot(a, a); }
PE_HD float length(V3 a) { return sqrtf(len2(a)); }
PE_HD V3 normalize(V3 a) {
    const float l = length(a);
    if (l <= 1e-20f) return mk(0.0f);
    return a / l;
}
PE_HD V3 vabs(V3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
PE_HD V3 vmin(V3 a, V3 b) { return mk(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)); }
PE_HD V3 vmax(V3 a, V3 b) { return mk(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)); }
PE_HD float maxComp(V3 a) { return smax(smax(a.x, a.y), a.z); }
PE_HD bool isBlack(V3 c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
PE_HD bool isFinite3(V3 c) { return finitef(c.x) && finitef(c.y) && finitef(c.z); }
// BT.709 luminance (src/core/color/spectrum.h:68-70).
PE_HD float luminance(V3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }
// Color3f lerp is a(1−t) + bt (spectrum.h:113); the scalar lerp is a + t(b − a) (utils.h:32).
PE_HD V3 lerp3(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
PE_HD float lerpf(float a, float b, float t) { return a + t * (b - a); }
// Color3f::clamp = max(lo, min(v, hi)) per channel (spectrum.h:57-62).
PE_HD V3 clamp3(V3 c, float lo, float hi) { return mk(smax(lo, smin(c.x, hi)), smax(lo, smin(c.y, hi)), smax(lo, smin(c.z, hi))); }

// Orthonormal basis of Duff et al. 2017 (src/core/math/frame.h:32-44).
struct Frame {
    V3 s, t, n;
};
PE_HD Frame frameFromNormal(V3 n) {
    Frame f;
    f.n = n;
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    f.s = mk(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    f.t = mk(b, sign + n.y * n.y * a, -n.y);
    return f;
}
PE_HD Frame frame3(V3 s, V3 t, V3 n) { Frame f; f.s = s; f.t = t; f.n = n; return f; }
PE_HD V3 toLocal(const Frame& f, V3 v) { return mk(dot(v, f.s), dot(v, f.t), dot(v, f.n)); }
PE_HD V3 toWorld(const Frame& f, V3 v) { return f.s * v.x + f.t * v.y + f.n * v.z; }

// Veach power heuristic (src/core/math/utils.h:108-113).
PE_HD float powerHeuristic(int nf, float fPdf, int ng, float gPdf) {
    const float f = static_cast<float>(nf) * fPdf;
    const float g = static_cast<float>(ng) * gPdf;
    const float f2 = f * f;
    return f2 / (f2 + g * g);
}
PE_HD V3 reflectV(V3 wo, V3 n) { return 2.0f * dot(wo, n) * n - wo; }
PE_HD bool refractV(V3 wi, V3 n, float eta, V3& wt) {
    const float cosThetaI = dot(n, wi);
    const float sin2ThetaI = smax(0.0f, 1.0f - cosThetaI * cosThetaI);
    const float sin2ThetaT = eta * eta * sin2ThetaI;
    if (sin2ThetaT >= 1.0f) return false;
    const float cosThetaT = sqrtf(1.0f - sin2ThetaT);
    wt = eta * (-wi) + (eta * cosThetaI - cosThetaT) * n;
    return true;
}
// Unpolarised dielectric Fresnel; indices swap unless cosθi > 0 (src/core/math/utils.h:203-226).
PE_HD float fresnelDielectric(float cosThetaI, float etaI, float etaT) {
    cosThetaI = sclamp(cosThetaI, -1.0f, 1.0f);
    if (!(cosThetaI > 0.0f)) {
        const float t = etaI; etaI = etaT; etaT = t;
        cosThetaI = fabsf(cosThetaI);
    }
    const float sinThetaI = sqrtf(smax(0.0f, 1.0f - cosThetaI * cosThetaI));
    const float sinThetaT = (etaI / etaT) * sinThetaI;
    if (sinThetaT >= 1.0f) return 1.0f;
    const float cosThetaT = sqrtf(smax(0.0f, 1.0f - sinThetaT * sinThetaT));
    const float rs = (etaT * cosThetaI - etaI * cosThetaT) / (etaT * cosThetaI + etaI * cosThetaT);
    const float rp = (etaI * cosThetaI - etaT * cosThetaT) / (etaI * cosThetaI + etaT * cosThetaT);
    return 0.5f * (rs * rs + rp * rp);
}

// ---- sampling warps (src/core/sampling/sampling.h) --------------------------------------
PE_HD V2 sampleDiskConcentric(V2 u) {
    const float sx = 2.0f * u.x - 1.0f;
    const float sy = 2.0f * u.y - 1.0f;
    if (sx == 0.0f && sy == 0.0f) return mk2(0.0f, 0.0f);
    float r, theta;
    if (fabsf(sx) > fabsf(sy)) {
        r = sx;
        theta = kPiOver4 * (sy / sx);
    } else {
        r = sy;
        theta = kPiOver2 - kPiOver4 * (sx / sy);
    }
    return mk2(r * cosf(theta), r * sinf(theta));
}
PE_HD V3 sampleCosineHemisphere(V2 u) {
    const V2 d = sampleDiskConcentric(u);
    const float z = sqrtf(smax(0.0f, 1.0f - d.x * d.x - d.y * d.y));
    return mk(d.x, d.y, z);
}
PE_HD float cosineHemispherePdf(float c) { return c * kInvPi; }
PE_HD V3 sampleUniformSphere(V2 u) {
    const float z = 1.0f - 2.0f * u.x;
    const float r = sqrtf(smax(0.0f, 1.0f - z * z));
    const float phi = kTwoPi * u.y;
    return mk(r * cosf(phi), r * sinf(phi), z);
}
PE_HD float uniformSpherePdf() { return 0.25f * kInvPi; }
PE_HD V2 sampleUniformTriangle(V2 u) {
    const float su0 = sqrtf(u.x);
    return mk2(1.0f - su0, u.y * su0);
}

// ---- Owen-scrambled Sobol (Burley 2020), src/samplers/sobol_sampler.cpp -----------------
PE_HD uint32_t rev32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
#endif
}
// Laine–Karras permutation with Burley's constants.
PE_HD uint32_t lkPermute(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
// lowbias32 hash.
PE_HD uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
PE_HD uint32_t hashMix(uint32_t h, uint32_t v) { return hash32(h ^ (v + 0x9e3779b9u + (h << 6) + (h >> 2))); }
PE_HD float unitFloat24(uint32_t x) { return static_cast<float>(x >> 8) * 5.9604644775390625e-08f; }
PE_HD uint32_t pixelHashOf(uint64_t seed, int x, int y) {
    uint32_t h = hash32(static_cast<uint32_t>(seed) ^ hash32(static_cast<uint32_t>(seed >> 32)));
    h = hashMix(h, static_cast<uint32_t>(x));
    return hashMix(h, static_cast<uint32_t>(y));
}
// Second Sobol dimension, bit-reversed: generator v_k = v_{k-1} ^ (v_{k-1} >> 1), v_0 = 2^31.
// Computed with the byte-table decomposition from a 4x256 table (built by sobolTableEntry).
PE_HD uint32_t sobolDim1(uint32_t index) {
    uint32_t r = 0;
    for (uint32_t v = 0x80000000u; index != 0; index >>= 1, v ^= v >> 1)
        if (index & 1u) r ^= v;
    return r;
}
PE_HD uint32_t sobolTableEntry(int k, uint32_t b) { return rev32(sobolDim1(b << (8 * k))); }

} // namespace pe
