// pe_light.h — light sampling on the device, following the reference's light set:
//
//   AreaLight / TriangleLight   src/lights/area_light.cpp:15-275 (spherical rectangles:
//                               Ureña, Fajardo, King 2013; triangle area sampling)
//   EnvironmentLight            src/lights/environment_light.cpp:21-325 (two-level CDF over the
//                               MIS-compensated image, sun cone mixture, bilinear equirect)
//   LightBounds                 src/lights/light_bounds.cpp:37-109
//   LightSampler                src/lights/light_sampler.cpp:150-284 (≤33 candidates:
//                               importance-proportional 85 % + 15 % uniform; else top level +
//                               light-BVH descent with bit-trail pmf)
#pragma once

#include "pe_math.h"
#include "pe_scene.h"

namespace pe {

struct LightSample {
    V3 wi;
    V3 Li;
    float pdf;
    float distance;
};
PE_HD bool lsValid(const LightSample& s) { return s.pdf > 0.0f && !isBlack(s.Li); }

PE_HD V3 lightRadiance(const LightGPU& l) { return mk(l.radiance_r, l.radiance_g, l.radiance_b); }

PE_HD float areaSolidAnglePdf(float distSq, float cosAbs, float area) {
    if (!(cosAbs > 1e-6f) || !(area > 0.0f) || !(distSq > 0.0f)) return 0.0f;
    return distSq / (area * cosAbs);
}
PE_HD float receiverCosine(V3 n, V3 toLight) {
    const float c = dot(n, toLight);
    return c > 0.05f ? c : 0.05f;
}
PE_HD float safeAsinf(float x) { return asinf(sclamp(x, -1.0f, 1.0f)); }
PE_HD float angleBetween(V3 a, V3 b) {
    if (dot(a, b) < 0.0f) return kPi - 2.0f * safeAsinf(length(a + b) * 0.5f);
    return 2.0f * safeAsinf(length(b - a) * 0.5f);
}

struct SphRect {
    Frame frame;
    float x0, y0, z0, x1, y1, b0, b1, g2g3, solidAngle;
};
PE_HD SphRect setupSphRect(V3 ref, V3 corner, V3 ex, V3 ey) {
    SphRect r;
    r.x0 = r.y0 = r.z0 = r.x1 = r.y1 = r.b0 = r.b1 = r.g2g3 = r.solidAngle = 0.0f;
    const float exl = length(ex), eyl = length(ey);
    const V3 x = ex / exl, y = ey / eyl;
    V3 z = cross(x, y);
    const V3 d = corner - ref;
    r.z0 = dot(d, z);
    if (r.z0 > 0.0f) {
        z = -z;
        r.z0 = -r.z0;
    }
    r.frame = frame3(x, y, z);
    r.x0 = dot(d, x);
    r.y0 = dot(d, y);
    r.x1 = r.x0 + exl;
    r.y1 = r.y0 + eyl;
    if (r.z0 > -1e-7f) return r;
    const V3 v00 = mk(r.x0, r.y0, r.z0), v01 = mk(r.x0, r.y1, r.z0), v10 = mk(r.x1, r.y0, r.z0),
             v11 = mk(r.x1, r.y1, r.z0);
    const V3 n0 = normalize(cross(v00, v10));
    const V3 n1 = normalize(cross(v10, v11));
    const V3 n2 = normalize(cross(v11, v01));
    const V3 n3 = normalize(cross(v01, v00));
    const float g0 = angleBetween(-n0, n1), g1 = angleBetween(-n1, n2);
    const float g2 = angleBetween(-n2, n3), g3 = angleBetween(-n3, n0);
    r.solidAngle = g0 + g1 + g2 + g3 - kTwoPi;
    r.b0 = n0.z;
    r.b1 = n2.z;
    r.g2g3 = g2 + g3;
    return r;
}
PE_HD V3 sampleSphRect(const SphRect& r, V2 u) {
    const float au = u.x * r.solidAngle - r.g2g3;
    const float fu = (cosf(au) * r.b0 - r.b1) / sinf(au);
    float cu = copysignf(1.0f, fu) / sqrtf(fu * fu + r.b0 * r.b0);
    cu = sclamp(cu, -0.9999999f, 0.9999999f);
    float xu = -(cu * r.z0) / sqrtf(smax(0.0f, 1.0f - cu * cu));
    xu = sclamp(xu, r.x0, r.x1);
    const float dd = sqrtf(xu * xu + r.z0 * r.z0);
    const float h0 = r.y0 / sqrtf(dd * dd + r.y0 * r.y0);
    const float h1 = r.y1 / sqrtf(dd * dd + r.y1 * r.y1);
    const float hv = h0 + u.y * (h1 - h0);
    const float hv2 = hv * hv;
    const float yv = hv2 < 1.0f - 1e-6f ? hv * dd / sqrtf(1.0f - hv2) : r.y1;
    return toWorld(r.frame, mk(xu, sclamp(yv, r.y0, r.y1), r.z0));
}
constexpr float kMinSolidAngle = 1e-3f;

// ---- explicit lights ------------------------------------------------------------------------
PE_HDN LightSample sampleLight(const LightGPU& l, V3 p, V2 u) {
    LightSample ls;
    ls.wi = mk(0.0f);
    ls.Li = mk(0.0f);
    ls.pdf = 0.0f;
    ls.distance = 0.0f;
    const V3 rad = lightRadiance(l);
    const V3 nrm = m3f(l.normal);
    if (l.type == LT_TRIANGLE) {
        if (!(l.area > 0.0f) || isBlack(rad)) return ls;
        const V2 b = sampleUniformTriangle(u);
        const V3 pL = m3f(l.p0) * (1.0f - b.x - b.y) + m3f(l.p1) * b.x + m3f(l.p2) * b.y;
        const V3 toL = pL - p;
        const float distSq = len2(toL);
        ls.distance = sqrtf(distSq);
        if (!(ls.distance > 0.0f)) return ls;
        ls.wi = toL / ls.distance;
        const float pdf = areaSolidAnglePdf(distSq, fabsf(dot(ls.wi, nrm)), l.area);
        if (!(pdf > 0.0f)) return ls;
        ls.Li = rad;
        ls.pdf = pdf;
        return ls;
    }
    // rectangle
    const V3 pos = m3f(l.p0), lu = m3f(l.p1), lv = m3f(l.p2);
    if (l.rectangle) {
        const SphRect r = setupSphRect(p, pos, lu, lv);
        if (r.solidAngle >= kMinSolidAngle) {
            const V3 toL = sampleSphRect(r, u);
            const float dist = length(toL);
            if (!(dist > 0.0f)) return ls;
            ls.distance = dist;
            ls.wi = toL / dist;
            ls.Li = rad;
            ls.pdf = 1.0f / r.solidAngle;
            return ls;
        }
    }
    const V3 pL = pos + lu * u.x + lv * u.y;
    const V3 toL = pL - p;
    const float distSq = len2(toL);
    ls.distance = sqrtf(distSq);
    if (ls.distance > 0.0f) {
        ls.wi = toL / ls.distance;
        const float cosL = fabsf(dot(ls.wi, nrm));
        const float pdf = areaSolidAnglePdf(distSq, cosL, l.area);
        if (pdf > 0.0f) {
            ls.Li = rad;
            ls.pdf = pdf;
        }
    }
    return ls;
}

// Light::pdfLiHit for a BSDF ray from ref that hit the light's geometry at pHit.
PE_HDN float lightPdfHit(const LightGPU& l, V3 ref, V3 pHit) {
    const V3 nrm = m3f(l.normal);
    if (l.type == LT_TRIANGLE) {
        const V3 toL = pHit - ref;
        const float distSq = len2(toL);
        if (!(distSq > 0.0f)) return 0.0f;
        return areaSolidAnglePdf(distSq, fabsf(dot(toL / sqrtf(distSq), nrm)), l.area);
    }
    const V3 pos = m3f(l.p0), lu = m3f(l.p1), lv = m3f(l.p2);
    const V3 d = pHit - pos;
    const float scale = smax(length(lu) + length(lv), 1.0f);
    if (fabsf(dot(d, nrm)) > 1e-3f * scale) return 0.0f;
    const float uu = dot(lu, lu), vv = dot(lv, lv), uv = dot(lu, lv);
    const float du = dot(d, lu), dv = dot(d, lv);
    const float det = uu * vv - uv * uv;
    if (!(fabsf(det) > 1e-12f * uu * vv)) return 0.0f;
    const float s = (vv * du - uv * dv) / det;
    const float t = (uu * dv - uv * du) / det;
    const float eps = 1e-3f;
    if (s < -eps || t < -eps || s > 1.0f + eps || t > 1.0f + eps) return 0.0f;
    if (l.rectangle) {
        const float omega = setupSphRect(ref, pos, lu, lv).solidAngle;
        if (omega >= kMinSolidAngle) return 1.0f / omega;
    }
    const V3 toL = pHit - ref;
    const float distSq = len2(toL);
    if (distSq <= 0.0f) return 0.0f;
    const V3 wi = toL / sqrtf(distSq);
    return areaSolidAnglePdf(distSq, fabsf(dot(wi, nrm)), l.area);
}

// Light::importance (area_light.cpp:104-113 and :206-215).
PE_HD float lightImportance(const LightGPU& l, V3 p, V3 n) {
    V3 c;
    if (l.type == LT_TRIANGLE) c = (m3f(l.p0) + m3f(l.p1) + m3f(l.p2)) * (1.0f / 3.0f);
    else c = m3f(l.p0) + (m3f(l.p1) + m3f(l.p2)) * 0.5f;
    const V3 d = c - p;
    const float dist2 = len2(d);
    const float lum = smax(0.0f, luminance(lightRadiance(l)));
    if (!(dist2 > 0.0f)) return lum * kTwoPi;
    const V3 w = d / sqrtf(dist2);
    const float cosL = smax(fabsf(dot(w, m3f(l.normal))), 0.2f);
    const float omega = smin(l.area * cosL / dist2, kTwoPi);
    return lum * omega * receiverCosine(n, w);
}

// ---- environment ----------------------------------------------------------------------------
PE_HD V2 dirToEquirect(V3 direction, float rotation) {
    const V3 d = normalize(direction);
    const float theta = acosf(sclamp(d.y, -1.0f, 1.0f));
    float phi = atan2f(-d.z, d.x) + kPi + rotation;
    phi = fmodf(phi, kTwoPi);
    if (phi < 0.0f) phi += kTwoPi;
    return mk2(phi / kTwoPi, theta / kPi);
}
PE_HD V3 equirectToDir(float u, float v, float rotation) {
    const float theta = v * kPi;
    const float a = u * kTwoPi - kPi - rotation;
    const float st = sinf(theta);
    return mk(st * cosf(a), cosf(theta), -st * sinf(a));
}
PE_HD V3 envPixel(const EnvGPU& e, int x, int y) {
    const float* p = e.image + 3 * (static_cast<size_t>(y) * static_cast<size_t>(e.width) + static_cast<size_t>(x));
    return mk(p[0], p[1], p[2]);
}
PE_HD V3 sampleEquirect(const EnvGPU& e, float u, float v) {
    const int w = e.width, h = e.height;
    u -= floorf(u);
    v = sclamp(v, 0.0f, 1.0f);
    const float x = u * static_cast<float>(w) - 0.5f;
    const float y = v * static_cast<float>(h) - 0.5f;
    const int x0 = static_cast<int>(floorf(x));
    const int y0 = static_cast<int>(floorf(y));
    const float fx = x - static_cast<float>(x0);
    const float fy = y - static_cast<float>(y0);
    int xa = x0 % w; if (xa < 0) xa += w;
    int xb = (x0 + 1) % w; if (xb < 0) xb += w;
    const int ya = iclamp(y0, 0, h - 1), yb = iclamp(y0 + 1, 0, h - 1);
    const V3 c0 = envPixel(e, xa, ya) * (1.0f - fx) + envPixel(e, xb, ya) * fx;
    const V3 c1 = envPixel(e, xa, yb) * (1.0f - fx) + envPixel(e, xb, yb) * fx;
    return c0 * (1.0f - fy) + c1 * fy;
}
PE_HD V3 envEvalSky(const EnvGPU& e, V3 dir) {
    if (!e.hasImage) return mk(0.5f) * e.intensity;
    const V2 uv = dirToEquirect(dir, e.rotation);
    return sampleEquirect(e, uv.x, uv.y) * e.intensity;
}
PE_HDN V3 envEval(const EnvGPU& e, V3 dir) {
    V3 sun = mk(0.0f);
    if (e.sunPdfWeight > 0.0f && dot(normalize(dir), m3f(e.sunDir)) >= e.sunCosMax) sun = m3f(e.sunRadiance);
    return envEvalSky(e, dir) + sun;
}
PE_HD float envImagePdf(const EnvGPU& e, V3 wi) {
    if (!e.valid || e.width <= 0 || e.height <= 0) return uniformSpherePdf();
    const V3 d = normalize(wi);
    const V2 uv = dirToEquirect(d, e.rotation);
    int x = imin(static_cast<int>(uv.x * static_cast<float>(e.width)), e.width - 1);
    int y = imin(static_cast<int>(uv.y * static_cast<float>(e.height)), e.height - 1);
    if (x < 0) x = 0;
    if (y < 0) y = 0;
    const float sinTheta = sqrtf(smax(0.0f, 1.0f - d.y * d.y));
    if (sinTheta < 1e-4f) return 0.0f;
    const float f = e.func[static_cast<size_t>(y) * static_cast<size_t>(e.width) + static_cast<size_t>(x)];
    return (f / e.funcInt) * static_cast<float>(e.width * e.height) / (kTwoPi * kPi * sinTheta);
}
PE_HDN float envPdf(const EnvGPU& e, V3 wi) {
    if (e.sunPdfWeight <= 0.0f) return envImagePdf(e, wi);
    float pdf = 0.0f;
    if (dot(normalize(wi), m3f(e.sunDir)) >= e.sunCosMax) pdf += e.sunPdfWeight / (kTwoPi * (1.0f - e.sunCosMax));
    if (e.sunPdfWeight < 1.0f) pdf += (1.0f - e.sunPdfWeight) * envImagePdf(e, wi);
    return pdf;
}
// First i with cdf[i] > u over n+1 entries (std::upper_bound), minus one, clamped to [0, n-1].
PE_HD int cdfFind(const float* cdf, int n, float u) {
    int lo = 0, count = n + 1;
    while (count > 0) {
        const int step = count / 2;
        const int it = lo + step;
        if (!(u < cdf[it])) {
            lo = it + 1;
            count -= step + 1;
        } else {
            count = step;
        }
    }
    int i = lo - 1;
    if (i < 0) i = 0;
    if (i >= n) i = n - 1;
    return i;
}
PE_HD void sampleCdf(const float* cdf, int n, float u, int& index, float& pdf, float& coord) {
    const int i = cdfFind(cdf, n, u);
    pdf = cdf[i + 1] - cdf[i];
    float du = pdf > 0.0f ? (u - cdf[i]) / pdf : 0.0f;
    du = sclamp(du, 0.0f, 1.0f);
    index = i;
    coord = (static_cast<float>(i) + du) / static_cast<float>(n);
}
PE_HD LightSample envSampleImage(const EnvGPU& e, V2 s) {
    LightSample ls;
    ls.distance = kFltMax;
    if (!e.valid || e.width <= 0) {
        ls.wi = sampleUniformSphere(s);
        ls.pdf = uniformSpherePdf();
        ls.Li = envEval(e, ls.wi);
        return ls;
    }
    int ri, ci;
    float rpdf, rc, cpdf, cc;
    sampleCdf(e.marginalCdf, e.height, s.y, ri, rpdf, rc);
    const float* cond = e.condCdf + static_cast<size_t>(ri) * static_cast<size_t>(e.width + 1);
    sampleCdf(cond, e.width, s.x, ci, cpdf, cc);
    const float theta = rc * kPi;
    const float sinTheta = smax(sinf(theta), 1e-6f);
    ls.wi = normalize(equirectToDir(cc, rc, e.rotation));
    ls.pdf = (rpdf * cpdf) * static_cast<float>(e.width * e.height) / (kTwoPi * kPi * sinTheta);
    ls.Li = envEval(e, ls.wi);
    return ls;
}
PE_HDN LightSample envSample(const EnvGPU& e, V2 s) {
    LightSample ls;
    ls.wi = mk(0.0f);
    ls.Li = mk(0.0f);
    ls.pdf = 0.0f;
    ls.distance = kFltMax;
    if (e.sunPdfWeight > 0.0f) {
        if (s.x < e.sunPdfWeight) {
            const float ux = smin(s.x / e.sunPdfWeight, 0.99999994f);
            const float cosT = 1.0f - ux * (1.0f - e.sunCosMax);
            const float sinT = sqrtf(smax(0.0f, 1.0f - cosT * cosT));
            const float phi = kTwoPi * s.y;
            const Frame f = frameFromNormal(m3f(e.sunDir));
            ls.wi = normalize(toWorld(f, mk(sinT * cosf(phi), sinT * sinf(phi), cosT)));
            ls.Li = envEval(e, ls.wi);
            ls.pdf = envPdf(e, ls.wi);
            return ls;
        }
        if (e.sunPdfWeight >= 1.0f) return ls;
        s.x = smin((s.x - e.sunPdfWeight) / (1.0f - e.sunPdfWeight), 0.99999994f);
    }
    LightSample img = envSampleImage(e, s);
    if (e.sunPdfWeight > 0.0f && img.pdf > 0.0f) img.pdf = envPdf(e, img.wi);
    return img;
}

// EnvironmentLight::sampleLiFull (environment_light.cpp:239-252): the sun cone as sampleLi, the
// rest from the uncompensated image distribution (`full`: the same light with that
// distribution's tables), its pdf then the full mixture's (pdfLiFull, :254-260).
PE_HDN LightSample envSampleFull(const EnvGPU& e, const EnvGPU& full, V2 sample) {
    if (e.sunPdfWeight > 0.0f && sample.x < e.sunPdfWeight) return envSample(e, sample);
    V2 s = sample;
    if (e.sunPdfWeight > 0.0f) {
        if (e.sunPdfWeight >= 1.0f) {
            LightSample none;
            none.wi = mk(0.0f);
            none.Li = mk(0.0f);
            none.pdf = 0.0f;
            none.distance = kFltMax;
            return none;
        }
        s.x = smin((sample.x - e.sunPdfWeight) / (1.0f - e.sunPdfWeight), 0.99999994f);
    }
    LightSample ls = envSampleImage(full, s);
    if (e.sunPdfWeight > 0.0f && ls.pdf > 0.0f) ls.pdf = envPdf(full, ls.wi);
    return ls;
}
PE_HD float envImportance(const EnvGPU& e, V3 n) {
    float imp = kPi * e.meanLuminance;
    if (e.sunPdfWeight > 0.0f)
        imp += smax(0.0f, luminance(m3f(e.sunRadiance))) * kTwoPi * (1.0f - e.sunCosMax) * receiverCosine(n, m3f(e.sunDir));
    return imp;
}

// ---- light BVH bounds -----------------------------------------------------------------------
PE_HD float safeSqrtf(float x) { return sqrtf(smax(0.0f, x)); }
PE_HD float cosSubClamped(float sinA, float cosA, float sinB, float cosB) {
    if (cosA > cosB) return 1.0f;
    return cosA * cosB + sinA * sinB;
}
PE_HD float sinSubClamped(float sinA, float cosA, float sinB, float cosB) {
    if (cosA > cosB) return 0.0f;
    return sinA * cosB - cosA * sinB;
}
PE_HD float boundsImportance(const LightNodeGPU& b, V3 p, V3 n) {
    if (!(b.phi > 0.0f)) return 0.0f;
    const V3 bmin = m3f(b.bmin), bmax = m3f(b.bmax);
    const V3 pc = (bmin + bmax) * 0.5f;
    const V3 diag = bmax - bmin;
    const float d2 = smax(len2(p - pc), 0.25f * len2(diag));
    if (!(d2 > 0.0f)) return b.phi;
    V3 wi = p - pc;
    const float len = length(wi);
    wi = len > 0.0f ? wi / len : m3f(b.w);
    float cosW = dot(m3f(b.w), wi);
    if (b.twoSided) cosW = fabsf(cosW);
    const float sinW = safeSqrtf(1.0f - cosW * cosW);
    const float r2 = 0.25f * len2(diag);
    const float dc2 = len2(p - pc);
    const float cosB = dc2 <= r2 ? -1.0f : safeSqrtf(1.0f - r2 / dc2);
    const float sinB = safeSqrtf(1.0f - cosB * cosB);
    const float sinO = safeSqrtf(1.0f - b.cosThetaO * b.cosThetaO);
    const float cosX = cosSubClamped(sinW, cosW, sinO, b.cosThetaO);
    const float sinX = sinSubClamped(sinW, cosW, sinO, b.cosThetaO);
    const float cosP = cosSubClamped(sinX, cosX, sinB, cosB);
    if (cosP < b.cosThetaE) return 0.0f;
    float imp = b.phi * cosP / d2;
    if (len2(n) > 0.0f) {
        const float cosI = fabsf(dot(wi, n));
        const float sinI = safeSqrtf(1.0f - cosI * cosI);
        imp *= cosSubClamped(sinI, cosI, sinB, cosB);
    }
    return smax(imp, 0.0f);
}

// ---- light sampler --------------------------------------------------------------------------
// Per-vertex selection distribution (LightSampler::Context): p, n and the top-level pmf.
struct LightCtx {
    V3 p, n;
    bool owner;     // false = default-constructed context (pmf 0)
    bool uniform;
    int topCount;
    float pmf[kMaxExhaustive];
};

PE_HD float candidateImportance(const SceneGPU& S, int idx, V3 p, V3 n) {
    if (idx < S.nLights) return lightImportance(S.lights[idx], p, n);
    return envImportance(S.env, n);
}

PE_HDN void lightPrepare(const SceneGPU& S, V3 p, V3 n, LightCtx& c) {
    c.p = p;
    c.n = n;
    c.owner = true;
    c.uniform = true;
    c.topCount = 0;
    if (S.lightCount <= 1 || S.lightMode == 0) return;
    int count;
    if (S.lightMode == 1) {
        count = S.lightCount;
        for (int i = 0; i < count; ++i) {
            const float w = candidateImportance(S, i, p, n);
            c.pmf[i] = (w > 0.0f && finitef(w)) ? w : 0.0f;
        }
    } else {
        count = S.nInfinite + (S.nLightNodes > 0 ? 1 : 0);
        for (int k = 0; k < S.nInfinite; ++k) {
            const float w = candidateImportance(S, S.infinite[k], p, n);
            c.pmf[k] = (w > 0.0f && finitef(w)) ? w : 0.0f;
        }
        if (S.nLightNodes > 0) {
            const float w = boundsImportance(S.lightNodes[0], p, n) * kInvPi;
            c.pmf[S.nInfinite] = (w > 0.0f && finitef(w)) ? w : 0.0f;
        }
    }
    c.topCount = count;
    float sum = 0.0f;
    for (int i = 0; i < count; ++i) sum += c.pmf[i];
    if (!(sum > 0.0f) || !finitef(sum)) {
        for (int i = 0; i < count; ++i) c.pmf[i] = 1.0f / static_cast<float>(count);
    } else {
        const float a = (1.0f - 0.15f) / sum, b = 0.15f / static_cast<float>(count);
        for (int i = 0; i < count; ++i) c.pmf[i] = c.pmf[i] * a + b;
    }
    c.uniform = false;
}

PE_HDN int bvhLightSample(const SceneGPU& S, V3 p, V3 n, float u, float& pmf) {
    pmf = 1.0f;
    int node = 0;
    for (int guard = 0; guard < 128; ++guard) {
        const LightNodeGPU& nd = S.lightNodes[node];
        if (nd.light >= 0) return nd.light;
        const int c0 = node + 1, c1 = nd.child1;
        const float i0 = boundsImportance(S.lightNodes[c0], p, n);
        const float i1 = boundsImportance(S.lightNodes[c1], p, n);
        if (!(i0 > 0.0f) && !(i1 > 0.0f)) {
            pmf = 0.0f;
            return -1;
        }
        const float p0 = i0 / (i0 + i1);
        if (u < p0) {
            node = c0;
            u = smin(u / p0, 0.99999994f);
            pmf *= p0;
        } else {
            node = c1;
            u = smin((u - p0) / (1.0f - p0), 0.99999994f);
            pmf *= 1.0f - p0;
        }
    }
    pmf = 0.0f;
    return -1;
}
PE_HDN float bvhLightPmf(const SceneGPU& S, V3 p, V3 n, int index) {
    if (index < 0 || index >= S.lightCount) return 0.0f;
    unsigned long long trail = S.trail[index];
    const int depth = S.trailDepth[index];
    float pmf = 1.0f;
    int node = 0;
    for (int d = 0; d < depth; ++d) {
        const LightNodeGPU& nd = S.lightNodes[node];
        if (nd.light >= 0) break;
        const int c0 = node + 1, c1 = nd.child1;
        const float i0 = boundsImportance(S.lightNodes[c0], p, n);
        const float i1 = boundsImportance(S.lightNodes[c1], p, n);
        const float sum = i0 + i1;
        if (!(sum > 0.0f)) return 0.0f;
        if (trail & 1ull) {
            pmf *= i1 / sum;
            node = c1;
        } else {
            pmf *= i0 / sum;
            node = c0;
        }
        trail >>= 1;
    }
    return S.lightNodes[node].light == index ? pmf : 0.0f;
}

// Context::sample (light_sampler.cpp:195-228): candidate index (env = nLights) or -1.
PE_HDN int lightCtxSample(const SceneGPU& S, const LightCtx& c, float u, float& pmf) {
    pmf = 0.0f;
    if (!c.owner) return -1;
    const int n = S.lightCount;
    if (n <= 0) return -1;
    if (c.uniform) {
        pmf = 1.0f / static_cast<float>(n);
        return imin(static_cast<int>(u * static_cast<float>(n)), n - 1);
    }
    float acc = 0.0f;
    int k = c.topCount - 1;
    for (int i = 0; i < c.topCount - 1; ++i) {
        if (u < acc + c.pmf[i]) {
            k = i;
            break;
        }
        acc += c.pmf[i];
    }
    const float pk = c.pmf[k];
    if (S.lightMode == 1) {
        pmf = pk;
        return k;
    }
    if (k < S.nInfinite) {
        pmf = pk;
        return S.infinite[k];
    }
    const float ur = smin((u - acc) / pk, 0.99999994f);
    float treePmf = 0.0f;
    const int light = bvhLightSample(S, c.p, c.n, smax(ur, 0.0f), treePmf);
    pmf = pk * treePmf;
    return light;
}

// Context::pmf (light_sampler.cpp:230-241).
PE_HDN float lightCtxPmf(const SceneGPU& S, const LightCtx& c, int index) {
    if (!c.owner) return 0.0f;
    if (index < 0 || index >= S.lightCount) return 0.0f;
    if (c.uniform) return 1.0f / static_cast<float>(S.lightCount);
    if (S.lightMode == 1) return c.pmf[index];
    const int slot = S.topSlot[index];
    if (slot >= 0) return c.pmf[slot];
    if (S.nLightNodes <= 0) return 0.0f;
    return c.pmf[S.nInfinite] * bvhLightPmf(S, c.p, c.n, index);
}

} // namespace pe
