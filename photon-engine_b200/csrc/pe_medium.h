// pe_medium.h — participating media, random-walk subsurface steps and spectral sampling.
//
//   spectralRaw / sampleWavelength   src/core/color/spectral.cpp:13-87
//   expNeg / sampleFreeFlight        src/integrators/path_tracer.cpp:85-128
//   sampleHG                         src/core/sampling/phase.h:26-39
//   MediaStack                       src/integrators/path_tracer.cpp:63-82
#pragma once

#include "pe_math.h"
#include "pe_scene.h"

namespace pe {

// Wyman–Sloan–Shirley 2013 piecewise-Gaussian CIE fit → linear sRGB (D65), negatives clipped.
PE_HD float spectralPiece(float x, float mu, float s1, float s2) {
    const float t = (x - mu) / (x < mu ? s1 : s2);
    return expf(-0.5f * t * t);
}
PE_HD V3 spectralRaw(float l) {
    const float X = 1.056f * spectralPiece(l, 599.8f, 37.9f, 31.0f) + 0.362f * spectralPiece(l, 442.0f, 16.0f, 26.7f) -
                    0.065f * spectralPiece(l, 501.1f, 20.4f, 26.2f);
    const float Y = 0.821f * spectralPiece(l, 568.8f, 46.9f, 40.5f) + 0.286f * spectralPiece(l, 530.9f, 16.3f, 31.1f);
    const float Z = 1.217f * spectralPiece(l, 437.0f, 11.8f, 36.0f) + 0.681f * spectralPiece(l, 459.0f, 26.0f, 13.8f);
    const float r = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    const float gg = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    const float b = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
    return mk(smax(0.0f, r), smax(0.0f, gg), smax(0.0f, b));
}

constexpr float kLambdaMin = 380.0f, kLambdaMax = 730.0f;
constexpr int kSpectralBins = 350;

// One wavelength for a path that meets a dispersive surface, importance-sampled ∝ r+g+b of the
// normalised colour-matching weights; `weight` = w(λ) / (range · pdf(λ)).
PE_HD float sampleWavelength(const TablesGPU* T, float u, V3& weight) {
    // upper_bound over the 351-entry CDF
    int lo = 0, n = kSpectralBins + 1;
    while (n > 0) {
        const int half = n >> 1;
        if (!(u < T->spectralCdf[lo + half])) {
            lo += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    int i = lo - 1;
    i = i < 0 ? 0 : (i > kSpectralBins - 1 ? kSpectralBins - 1 : i);
    const float a = T->spectralCdf[i], b = T->spectralCdf[i + 1];
    const float f = b > a ? sclamp((u - a) / (b - a), 0.0f, 1.0f) : 0.5f;
    const float bw = (kLambdaMax - kLambdaMin) / static_cast<float>(kSpectralBins);
    const float lambda = kLambdaMin + (static_cast<float>(i) + f) * bw;
    const V3 rgb = spectralRaw(lambda) * mk(T->spectralNorm[0], T->spectralNorm[1], T->spectralNorm[2]);
    weight = rgb / ((kLambdaMax - kLambdaMin) * T->spectralPdf[i]);
    return lambda;
}

PE_HD V3 expNeg(V3 sigma, float t) { return mk(expf(-sigma.x * t), expf(-sigma.y * t), expf(-sigma.z * t)); }

// Homogeneous free flight with spectral MIS over the three channels (one-sample mixture of
// per-channel exponentials, channel chosen ∝ channelWeights).  Returns true when the flight
// scatters at tScatter < tMax; otherwise the segment reached the surface (or infinity) and the
// throughput carries the transmittance over the mixture probability.
PE_HD bool sampleFreeFlight(V3 sigmaT, V3 sigmaS, float tMax, bool hitSurface, V3 channelWeights, float uc, float u,
                            V3& throughput, float& tScatter) {
    float wsum = channelWeights.x + channelWeights.y + channelWeights.z;
    if (!(wsum > 0.0f)) {
        channelWeights = mk(1.0f);
        wsum = 3.0f;
    }
    const V3 pc = channelWeights / wsum;
    const int c = uc < pc.x ? 0 : (uc < pc.x + pc.y ? 1 : 2);
    const float st = get(sigmaT, c);
    const float t = st > 0.0f ? -logf(smax(1.0f - u, 1e-12f)) / st : kFltMax;
    if (t < tMax) {
        const V3 Tr = expNeg(sigmaT, t);
        const float pdf = pc.x * sigmaT.x * Tr.x + pc.y * sigmaT.y * Tr.y + pc.z * sigmaT.z * Tr.z;
        if (!(pdf > 0.0f)) {
            throughput = mk(0.0f);
            return false;
        }
        throughput *= sigmaS * Tr / pdf;
        tScatter = t;
        return true;
    }
    V3 Tr;
    for (int k = 0; k < 3; ++k)
        set(Tr, k, hitSurface ? expf(-get(sigmaT, k) * tMax) : (get(sigmaT, k) > 0.0f ? 0.0f : 1.0f));
    const float P = pc.x * Tr.x + pc.y * Tr.y + pc.z * Tr.z;
    throughput = P > 0.0f ? throughput * Tr / P : mk(0.0f);
    return false;
}

// Henyey–Greenstein direction about the propagation direction d (inverse CDF of cosθ).
PE_HD V3 sampleHG(V3 d, float g, V2 u) {
    float cosTheta;
    if (fabsf(g) < 1e-3f) {
        cosTheta = 1.0f - 2.0f * u.x;
    } else {
        const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u.x);
        cosTheta = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    cosTheta = sclamp(cosTheta, -1.0f, 1.0f);
    const float sinTheta = sqrtf(smax(0.0f, 1.0f - cosTheta * cosTheta));
    const float phi = kTwoPi * u.y;
    const Frame f = frameFromNormal(d);
    return normalize(toWorld(f, mk(sinTheta * cosf(phi), sinTheta * sinf(phi), cosTheta)));
}

// Per-path stack of the volume-boundary materials a refracted path is inside (at most four;
// overflow is ignored, as in the reference).  Packed into 16-bit slots of material index + 1;
// the top entry's material supplies the current medium when it has one.
struct MediaStack {
    uint32_t lo, hi; // slots 0,1 | slots 2,3
    int n;
    PE_HD int at(int i) const {
        const uint32_t w = i < 2 ? lo : hi;
        return static_cast<int>((w >> ((i & 1) * 16)) & 0xFFFFu) - 1;
    }
    PE_HD void put(int i, int mat) {
        uint32_t& w = i < 2 ? lo : hi;
        const int sh = (i & 1) * 16;
        w = (w & ~(0xFFFFu << sh)) | (static_cast<uint32_t>(mat + 1) << sh);
    }
    PE_HD int top() const { return n > 0 ? at(n - 1) : -1; }
    PE_HD void enter(int mat) {
        if (n < 4) put(n++, mat);
    }
    PE_HD void leave(int mat) {
        for (int i = n - 1; i >= 0; --i) {
            if (at(i) != mat) continue;
            for (int j = i; j < n - 1; ++j) put(j, at(j + 1));
            put(n - 1, -1);
            --n;
            return;
        }
    }
};

} // namespace pe
