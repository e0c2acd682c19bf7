// pe_guide.cuh — the learned directional proposal: a multiresolution hash grid over the scene
// box (16 levels × 2 features) plus the shading normal and the view direction feed a 3×64 MLP
// whose 40 outputs are an 8-lobe von Mises–Fisher mixture over incident directions.  It stands
// beside the reference's SD-tree guiding (src/integrators/path_guiding.cpp) as its learned
// counterpart: trained online on the tracer's own radiance samples, drawn with one-sample MIS
// against the BSDF (50/50, as the reference's guided sampling, path_tracer.cpp:703-735).
//
// Inference runs on the tensor cores (kGuideInfer: tcgen05.mma with TMEM accumulators, FP16
// operands, FP32 accumulation).  Training evaluates the same network in FP32 on the SIMT cores
// (kGuideTrain: forward, negative-log-likelihood gradient of the mixture, backward into the MLP
// and the hash grid) and steps Adam (kGuideAdam).
#pragma once

#include "pe_math.h"

#include <cuda_fp16.h>
#include <cstdint>

namespace pe {

// ---- network shape -------------------------------------------------------------------------
constexpr int kGridLevels = 16;
constexpr int kGridFeatures = 2;
constexpr int kGridLog2Table = 18;                 // 2^18 entries per level
constexpr int kGridTable = 1 << kGridLog2Table;
constexpr int kGridParams = kGridLevels * kGridTable * kGridFeatures;
constexpr int kNetIn = 48;                        // 32 grid + 3 normal + 3 view + 10 zero padding
constexpr int kNetHidden = 64;
constexpr int kNetOut = 64;                       // 40 used: 8 lobes × (direction 3, log κ, weight logit)
constexpr int kLobes = 8;
constexpr int kNetUsedOut = kLobes * 5;
// FP32 parameter block: W1 [64][48], b1 [64], W2 [64][64], b2, W3 [64][64], b3, W4 [64][64], b4 [64]
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kNetHidden * kNetIn;
constexpr int kOffW2 = kOffB1 + kNetHidden;
constexpr int kOffB2 = kOffW2 + kNetHidden * kNetHidden;
constexpr int kOffW3 = kOffB2 + kNetHidden;
constexpr int kOffB3 = kOffW3 + kNetHidden * kNetHidden;
constexpr int kOffW4 = kOffB3 + kNetHidden;
constexpr int kOffB4 = kOffW4 + kNetOut * kNetHidden;
constexpr int kNetParams = kOffB4 + kNetOut;
constexpr float kLogKappaMin = -6.0f, kLogKappaMax = 7.0f;

struct GuideNet {
    const float* mlp;       // kNetParams FP32 master copy
    const __half* mlp16;    // FP16 copy of the weights for the tensor cores (biases stay FP32)
    const float* grid;      // kGridParams FP32 features
    float boxMin[3], boxInv[3]; // position → [0,1]^3
};

// ---- hash-grid encoding (Müller et al. 2022) --------------------------------------------------
// Level resolutions 16 · 2^(7l/15) rounded (16 … 2048): a fixed table, so that no rounding of a
// transcendental function decides a grid cell.
PE_HD float gridScale(int level) {
    constexpr float kRes[kGridLevels] = {16, 22, 31, 42, 58, 81, 111, 154, 213, 294, 406, 562, 776, 1072, 1482, 2048};
    return kRes[level];
}

PE_HD uint32_t gridIndex(int level, uint32_t x, uint32_t y, uint32_t z, uint32_t res) {
    const uint64_t r1 = static_cast<uint64_t>(res) + 1;
    uint32_t i;
    if (r1 * r1 * r1 <= static_cast<uint64_t>(kGridTable))
        i = x + y * static_cast<uint32_t>(r1) + z * static_cast<uint32_t>(r1 * r1);
    else
        i = (x * 1u) ^ (y * 2654435761u) ^ (z * 805459861u);
    return static_cast<uint32_t>(level) * kGridTable + (i & (kGridTable - 1));
}

// Corner indices and trilinear weights of one level at unit-cube position u.
struct GridCorners {
    uint32_t idx[8];
    float w[8];
};

PE_HD void gridCorners(int level, V3 u, GridCorners& c) {
    const float res = gridScale(level);
    const float px = u.x * res, py = u.y * res, pz = u.z * res;
    const float fx0 = floorf(px), fy0 = floorf(py), fz0 = floorf(pz);
    const float fx = px - fx0, fy = py - fy0, fz = pz - fz0;
    const uint32_t x0 = static_cast<uint32_t>(fx0), y0 = static_cast<uint32_t>(fy0), z0 = static_cast<uint32_t>(fz0);
    const uint32_t r = static_cast<uint32_t>(res);
    for (int k = 0; k < 8; ++k) {
        const uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        c.idx[k] = gridIndex(level, x0 + dx, y0 + dy, z0 + dz, r);
        c.w[k] = (dx ? fx : 1.0f - fx) * (dy ? fy : 1.0f - fy) * (dz ? fz : 1.0f - fz);
    }
}

PE_HD V3 guideUnit(const GuideNet& g, V3 p) {
    V3 u = mk((p.x - g.boxMin[0]) * g.boxInv[0], (p.y - g.boxMin[1]) * g.boxInv[1], (p.z - g.boxMin[2]) * g.boxInv[2]);
    u.x = sclamp(u.x, 0.0f, 1.0f);
    u.y = sclamp(u.y, 0.0f, 1.0f);
    u.z = sclamp(u.z, 0.0f, 1.0f);
    return u;
}

// Network input row for a query (position, shading normal, direction towards the viewer).
PE_HD void guideInput(const GuideNet& g, V3 p, V3 n, V3 wo, float* x) {
    const V3 u = guideUnit(g, p);
    for (int l = 0; l < kGridLevels; ++l) {
        GridCorners c;
        gridCorners(l, u, c);
        float f0 = 0.0f, f1 = 0.0f;
        for (int k = 0; k < 8; ++k) {
            f0 += c.w[k] * g.grid[2 * c.idx[k] + 0];
            f1 += c.w[k] * g.grid[2 * c.idx[k] + 1];
        }
        x[2 * l + 0] = f0;
        x[2 * l + 1] = f1;
    }
    x[32] = n.x;
    x[33] = n.y;
    x[34] = n.z;
    x[35] = wo.x;
    x[36] = wo.y;
    x[37] = wo.z;
    for (int i = 38; i < kNetIn; ++i) x[i] = 0.0f;
}

// ---- the vMF mixture ------------------------------------------------------------------------
struct Lobes {
    V3 mu[kLobes];
    float kappa[kLobes];
    float weight[kLobes];
};

// Network outputs → mixture: direction normalised, κ = exp(clamped log κ), softmax weights.
PE_HD void decodeLobes(const float* o, Lobes& L) {
    float mx = -1e30f;
    for (int k = 0; k < kLobes; ++k) mx = smax(mx, o[5 * k + 4]);
    float sum = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        const V3 m = mk(o[5 * k + 0], o[5 * k + 1], o[5 * k + 2]);
        const float len = sqrtf(len2(m)) + 1e-6f;
        L.mu[k] = mk(m.x / len, m.y / len, m.z / len);
        L.kappa[k] = expf(sclamp(o[5 * k + 3], kLogKappaMin, kLogKappaMax));
        L.weight[k] = expf(o[5 * k + 4] - mx);
        sum += L.weight[k];
    }
    for (int k = 0; k < kLobes; ++k) L.weight[k] /= sum;
}

// vMF density on the sphere: κ / (2π (1 − e^{−2κ})) · e^{κ (μ·ω − 1)}.
PE_HD float vmfPdf(V3 mu, float kappa, V3 w) {
    const float norm = kappa / (2.0f * kPi * -expm1f(-2.0f * kappa));
    return norm * expf(kappa * (dot(mu, w) - 1.0f));
}

PE_HD float lobesPdf(const Lobes& L, V3 w) {
    float p = 0.0f;
    for (int k = 0; k < kLobes; ++k) p += L.weight[k] * vmfPdf(L.mu[k], L.kappa[k], w);
    return p;
}

// One direction from the mixture: lobe by uLobe, then the vMF sample of Jakob 2012
// ("Numerically stable sampling of the von Mises–Fisher distribution on S²").
PE_HD V3 lobesSample(const Lobes& L, float uLobe, V2 u) {
    int k = 0;
    float acc = L.weight[0];
    while (k < kLobes - 1 && uLobe >= acc) {
        ++k;
        acc += L.weight[k];
    }
    const float kappa = L.kappa[k];
    const float cosT = 1.0f + logf(u.x + (1.0f - u.x) * expf(-2.0f * kappa)) / kappa;
    const float c = sclamp(cosT, -1.0f, 1.0f);
    const float s = sqrtf(smax(0.0f, 1.0f - c * c));
    const float phi = 2.0f * kPi * u.y;
    const Frame f = frameFromNormal(L.mu[k]);
    return normalize(toWorld(f, mk(s * cosf(phi), s * sinf(phi), c)));
}

// ∂(−log q(ω))/∂(network outputs) for the mixture decoded from o.
PE_HD float nllGrad(const float* o, V3 w, float* g) {
    Lobes L;
    decodeLobes(o, L);
    float v[kLobes];
    float q = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        v[k] = vmfPdf(L.mu[k], L.kappa[k], w);
        q += L.weight[k] * v[k];
    }
    q = smax(q, 1e-20f);
    for (int i = 0; i < kNetOut; ++i) g[i] = 0.0f;
    for (int k = 0; k < kLobes; ++k) {
        const float r = L.weight[k] * v[k] / q; // responsibility
        // weight logits (softmax)
        g[5 * k + 4] = L.weight[k] - r;
        // log κ (zero gradient where the clamp is active)
        const float lk = o[5 * k + 3];
        if (lk > kLogKappaMin && lk < kLogKappaMax) {
            const float kap = L.kappa[k];
            const float dlogv = 1.0f / kap - 2.0f / expm1f(2.0f * kap) + (dot(L.mu[k], w) - 1.0f);
            g[5 * k + 3] = -r * dlogv * kap;
        }
        // raw direction m, μ = m / (|m| + ε): ∂log v/∂μ = κ ω, ∂μ/∂m = (I − μ μᵀ)/|m| (ε dropped)
        const V3 m = mk(o[5 * k + 0], o[5 * k + 1], o[5 * k + 2]);
        const float len = sqrtf(len2(m)) + 1e-6f;
        const float mw = dot(L.mu[k], w);
        const float s = -r * L.kappa[k] / len;
        g[5 * k + 0] = s * (w.x - mw * L.mu[k].x);
        g[5 * k + 1] = s * (w.y - mw * L.mu[k].y);
        g[5 * k + 2] = s * (w.z - mw * L.mu[k].z);
    }
    return -logf(q);
}

// ---- FP32 network (training and the reference for the tensor-core path) ------------------------
PE_HD void mlpForward(const float* P, const float* x, float* h1, float* h2, float* h3, float* o) {
    for (int j = 0; j < kNetHidden; ++j) {
        float a = P[kOffB1 + j];
        for (int i = 0; i < kNetIn; ++i) a += P[kOffW1 + j * kNetIn + i] * x[i];
        h1[j] = smax(a, 0.0f);
    }
    for (int j = 0; j < kNetHidden; ++j) {
        float a = P[kOffB2 + j];
        for (int i = 0; i < kNetHidden; ++i) a += P[kOffW2 + j * kNetHidden + i] * h1[i];
        h2[j] = smax(a, 0.0f);
    }
    for (int j = 0; j < kNetHidden; ++j) {
        float a = P[kOffB3 + j];
        for (int i = 0; i < kNetHidden; ++i) a += P[kOffW3 + j * kNetHidden + i] * h2[i];
        h3[j] = smax(a, 0.0f);
    }
    for (int j = 0; j < kNetOut; ++j) {
        float a = P[kOffB4 + j];
        for (int i = 0; i < kNetHidden; ++i) a += P[kOffW4 + j * kNetHidden + i] * h3[i];
        o[j] = a;
    }
}

} // namespace pe
