// pe_bsdf.h — BSDFs of the reference's material set, evaluated per shading point on the GPU
// (and on the host, where the energy tables are integrated once per scene build).
//
//   microfacet / tables   src/materials/microfacet.h:26-163, microfacet.cpp:13-163
//   Fresnel models        src/materials/fresnel.h:21-107
//   EON diffuse           src/materials/eon.h:23-53
//   Lambertian            src/materials/lambertian.cpp:8-62
//   Disney / OpenPBR      src/materials/disney.cpp:26-757
//   Dielectric            src/materials/dielectric.cpp:18-294
//   Mirror                src/materials/mirror.cpp:7-43
//
// All directions are world space unless named *Local; wo and wi point away from the surface.
#pragma once

#include "pe_math.h"
#include "pe_scene.h"

namespace pe {

// ---------------------------------------------------------------------------------------------
// microfacet
constexpr float kGgxMinAlpha = 1e-4f;
PE_HD float ggxClampAlpha(float a) { return smax(a, kGgxMinAlpha); }
PE_HD float pow5(float x) {
    const float x2 = x * x;
    return x2 * x2 * x;
}
PE_HD float ggxD(V3 h, float ax, float ay) {
    if (h.z <= 0.0f) return 0.0f;
    ax = ggxClampAlpha(ax);
    ay = ggxClampAlpha(ay);
    const float e = (h.x * h.x) / (ax * ax) + (h.y * h.y) / (ay * ay) + h.z * h.z;
    return 1.0f / (kPi * ax * ay * e * e);
}
PE_HD float ggxLambda(V3 w, float ax, float ay) {
    const float z2 = w.z * w.z;
    if (z2 <= 1e-12f) return 1e12f;
    ax = ggxClampAlpha(ax);
    ay = ggxClampAlpha(ay);
    const float t2 = (ax * ax * w.x * w.x + ay * ay * w.y * w.y) / z2;
    return 0.5f * (-1.0f + sqrtf(1.0f + t2));
}
PE_HD float ggxG1(V3 w, float ax, float ay) { return 1.0f / (1.0f + ggxLambda(w, ax, ay)); }
PE_HD float ggxG(V3 wo, V3 wi, float ax, float ay) {
    return 1.0f / (1.0f + ggxLambda(wo, ax, ay) + ggxLambda(wi, ax, ay));
}
PE_HD float ggxVisiblePdf(V3 wo, V3 h, float ax, float ay) {
    const float cosO = fabsf(wo.z);
    if (cosO <= 0.0f) return 0.0f;
    return ggxG1(wo, ax, ay) * fabsf(dot(wo, h)) * ggxD(h, ax, ay) / cosO;
}
// Heitz 2018 visible-normal sampling.
PE_HD V3 ggxSampleVisibleNormal(V3 wo, float ax, float ay, float u1, float u2) {
    ax = ggxClampAlpha(ax);
    ay = ggxClampAlpha(ay);
    if (wo.z < 0.0f) wo = -wo;
    const V3 vh = normalize(mk(ax * wo.x, ay * wo.y, wo.z));
    const float lenSq = vh.x * vh.x + vh.y * vh.y;
    const V3 t1 = lenSq > 0.0f ? mk(-vh.y, vh.x, 0.0f) / sqrtf(lenSq) : mk(1.0f, 0.0f, 0.0f);
    const V3 t2 = cross(vh, t1);
    const float r = sqrtf(u1);
    const float phi = kTwoPi * u2;
    const float p1 = r * cosf(phi);
    float p2 = r * sinf(phi);
    const float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * sqrtf(smax(0.0f, 1.0f - p1 * p1)) + s * p2;
    const V3 nh = t1 * p1 + t2 * p2 + vh * sqrtf(smax(0.0f, 1.0f - p1 * p1 - p2 * p2));
    return normalize(mk(ax * nh.x, ay * nh.y, smax(1e-6f, nh.z)));
}
// Charlie sheen (Estevez & Kulla 2017) with Neubelt visibility.
PE_HD float charlieD(float cosH, float roughness) {
    const float a = smax(roughness * roughness, 1e-4f);
    const float inv = 1.0f / a;
    const float sin2 = smax(0.0f, 1.0f - cosH * cosH);
    return (2.0f + inv) * powf(sin2, 0.5f * inv) * (0.5f * kInvPi);
}
PE_HD float charlieV(float cosI, float cosO) { return 1.0f / smax(4.0f * (cosI + cosO - cosI * cosO), 1e-6f); }

// Bilinear lookup on a 32x32 table with nodes at i/31 (microfacet.cpp:19-33).
PE_HD float tableLookup2D(const float* t, float mu, float alpha) {
    const float x = sclamp(mu, 0.0f, 1.0f) * (kTableN - 1);
    const float y = sclamp(alpha, 0.0f, 1.0f) * (kTableN - 1);
    const int x0 = iclamp(static_cast<int>(floorf(x)), 0, kTableN - 1);
    const int y0 = iclamp(static_cast<int>(floorf(y)), 0, kTableN - 1);
    const int x1 = imin(x0 + 1, kTableN - 1), y1 = imin(y0 + 1, kTableN - 1);
    const float fx = sclamp(x - static_cast<float>(x0), 0.0f, 1.0f);
    const float fy = sclamp(y - static_cast<float>(y0), 0.0f, 1.0f);
    const float a = t[y0 * kTableN + x0] * (1.0f - fx) + t[y0 * kTableN + x1] * fx;
    const float b = t[y1 * kTableN + x0] * (1.0f - fx) + t[y1 * kTableN + x1] * fx;
    return a * (1.0f - fy) + b * fy;
}
PE_HD float tableLookup1D(const float* t, float alpha) {
    const float y = sclamp(alpha, 0.0f, 1.0f) * (kTableN - 1);
    const int y0 = iclamp(static_cast<int>(floorf(y)), 0, kTableN - 1);
    const int y1 = imin(y0 + 1, kTableN - 1);
    const float fy = sclamp(y - static_cast<float>(y0), 0.0f, 1.0f);
    return t[y0] * (1.0f - fy) + t[y1] * fy;
}
PE_HD float ggxDirectionalAlbedo(const TablesGPU* T, float cosTheta, float alpha) {
    return sclamp(tableLookup2D(T->ggxE, cosTheta, alpha), 1e-3f, 1.0f);
}
PE_HD float ggxSchlickAlbedo(const TablesGPU* T, float cosTheta, float alpha, float f0) {
    const float E = sclamp(tableLookup2D(T->ggxE, cosTheta, alpha), 1e-3f, 1.0f);
    const float ss = f0 * tableLookup2D(T->ggxEa, cosTheta, alpha) + tableLookup2D(T->ggxEb, cosTheta, alpha);
    return sclamp(ss * (1.0f + f0 * (1.0f / E - 1.0f)), 0.0f, 1.0f);
}
PE_HD float ggxSchlickAverageAlbedo(const TablesGPU* T, float alpha, float f0) {
    const float v = tableLookup1D(T->avg0, alpha) + f0 * tableLookup1D(T->avg1, alpha) +
                    f0 * f0 * tableLookup1D(T->avg2, alpha);
    return sclamp(v, 0.0f, 1.0f);
}
PE_HD float charlieSheenAlbedo(const TablesGPU* T, float cosTheta, float roughness) {
    return smax(tableLookup2D(T->sheenE, cosTheta, roughness), 0.0f);
}

// ---------------------------------------------------------------------------------------------
// Fresnel
PE_HD float schlickF(float f0, float cosTheta) {
    const float m = 1.0f - sclamp(cosTheta, 0.0f, 1.0f);
    const float m2 = m * m;
    return f0 + (1.0f - f0) * m2 * m2 * m;
}
PE_HD V3 fresnelF82Tint(V3 f0, V3 tint, float cosTheta) {
    const float muBar = 1.0f / 7.0f;
    const float oneMinus = 1.0f - muBar;
    const float denom = muBar * oneMinus * oneMinus * oneMinus * oneMinus * oneMinus * oneMinus;
    const float mu = sclamp(cosTheta, 0.0f, 1.0f);
    const float m = 1.0f - mu;
    const float m6 = m * m * m * m * m * m;
    V3 out;
    for (int c = 0; c < 3; ++c) {
        const float fsBar = schlickF(get(f0, c), muBar);
        const float b = fsBar * (1.0f - get(tint, c)) / denom;
        set(out, c, sclamp(schlickF(get(f0, c), mu) - b * mu * m6, 0.0f, 1.0f));
    }
    return out;
}

struct Cx {
    float re, im;
};
PE_HD Cx cx(float r, float i) { Cx c; c.re = r; c.im = i; return c; }
PE_HD Cx operator+(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
PE_HD Cx operator-(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
PE_HD Cx operator*(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
PE_HD Cx operator*(float s, Cx a) { return cx(s * a.re, s * a.im); }
PE_HD Cx operator/(Cx a, Cx b) {
    const float d = b.re * b.re + b.im * b.im;
    return cx((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
PE_HD float cnorm(Cx a) { return a.re * a.re + a.im * a.im; }
PE_HD Cx csqrt(Cx z) {
    if (z.re == 0.0f && z.im == 0.0f) return cx(0.0f, z.im);
    const float m = sqrtf(z.re * z.re + z.im * z.im);
    const float t = sqrtf(0.5f * (fabsf(z.re) + m));
    if (z.re >= 0.0f) return cx(t, z.im / (2.0f * t));
    return cx(fabsf(z.im) / (2.0f * t), copysignf(t, z.im));
}
// Gulbrandsen 2014 artist-friendly metal IOR (fresnel.h:44-53).
PE_HD Cx gulbrandsenIor(float r, float g) {
    r = sclamp(r, 0.0f, 0.99f);
    g = sclamp(g, 0.0f, 1.0f);
    const float sr = sqrtf(r);
    const float nMin = (1.0f - r) / (1.0f + r);
    const float nMax = (1.0f + sr) / (1.0f - sr);
    const float n = g * nMin + (1.0f - g) * nMax;
    const float k2 = (r * (n + 1.0f) * (n + 1.0f) - (n - 1.0f) * (n - 1.0f)) / (1.0f - r);
    return cx(n, sqrtf(smax(0.0f, k2)));
}
// Airy summation of a thin film between n1 and a (complex) base n3 (fresnel.h:72-90).
PE_HD float thinFilmReflectance(float cos1, float n1, float n2, Cx n3, float thicknessNm, float lambdaNm) {
    cos1 = sclamp(cos1, 0.0f, 1.0f);
    const float sin1sq = 1.0f - cos1 * cos1;
    const float sin2sq = (n1 / n2) * (n1 / n2) * sin1sq;
    if (sin2sq >= 1.0f) return 1.0f;
    const float cos2 = sqrtf(1.0f - sin2sq);
    const Cx cos3 = csqrt(cx(1.0f, 0.0f) - cx(n1 * n1 * sin1sq, 0.0f) / (n3 * n3));
    const float r12s = (n1 * cos1 - n2 * cos2) / (n1 * cos1 + n2 * cos2);
    const float r12p = (n2 * cos1 - n1 * cos2) / (n2 * cos1 + n1 * cos2);
    const Cx n2c = cx(n2, 0.0f);
    const Cx r23s = (cx(n2 * cos2, 0.0f) - n3 * cos3) / (cx(n2 * cos2, 0.0f) + n3 * cos3);
    const Cx r23p = (n3 * cx(cos2, 0.0f) - n2c * cos3) / (n3 * cx(cos2, 0.0f) + n2c * cos3);
    const float delta = 4.0f * kPi * n2 * thicknessNm * cos2 / lambdaNm;
    const Cx e = cx(cosf(delta), sinf(delta));
    const Cx rs = (cx(r12s, 0.0f) + r23s * e) / (cx(1.0f, 0.0f) + r12s * (r23s * e));
    const Cx rp = (cx(r12p, 0.0f) + r23p * e) / (cx(1.0f, 0.0f) + r12p * (r23p * e));
    return sclamp(0.5f * (cnorm(rs) + cnorm(rp)), 0.0f, 1.0f);
}
PE_HDN V3 thinFilmRGB(float cos1, float filmIor, const Cx baseIor[3], float thicknessNm) {
    const float lam[3][3] = {{610.0f, 640.0f, 670.0f}, {515.0f, 540.0f, 565.0f}, {440.0f, 465.0f, 490.0f}};
    V3 out;
    for (int c = 0; c < 3; ++c) {
        float s = 0.0f;
        for (int k = 0; k < 3; ++k) s += thinFilmReflectance(cos1, 1.0f, filmIor, baseIor[c], thicknessNm, lam[c][k]);
        set(out, c, s / 3.0f);
    }
    return out;
}

// ---------------------------------------------------------------------------------------------
// EON diffuse (Portsmouth, Kutz, Hill 2025)
constexpr float kFonC1 = 0.5f - 2.0f / (3.0f * kPi);
constexpr float kFonC2 = 2.0f / 3.0f - 28.0f / (15.0f * kPi);
PE_HD float fonAlbedo(float mu, float r) {
    mu = sclamp(mu, 1e-4f, 1.0f);
    const float AF = 1.0f / (1.0f + kFonC1 * r);
    const float BF = r * AF;
    const float Si = sqrtf(smax(0.0f, 1.0f - mu * mu));
    const float G = Si * (acosf(mu) - Si * mu) + (2.0f / 3.0f) * ((Si / mu) * (1.0f - Si * Si * Si) - Si);
    return AF + (BF * kInvPi) * G;
}
PE_HD V3 eonEval(V3 rho, float r, V3 wi, V3 wo) {
    const float muI = wi.z, muO = wo.z;
    if (r <= 0.0f) return rho * kInvPi;
    const float s = dot(wi, wo) - muI * muO;
    const float sOverT = s > 0.0f ? s / smax(muI, muO) : s;
    const float AF = 1.0f / (1.0f + kFonC1 * r);
    const V3 fss = rho * (kInvPi * AF * (1.0f + r * sOverT));
    const float EFo = fonAlbedo(muO, r), EFi = fonAlbedo(muI, r);
    const float avgEF = AF * (1.0f + kFonC2 * r);
    V3 rhoMs;
    for (int c = 0; c < 3; ++c) {
        const float rc = get(rho, c);
        set(rhoMs, c, rc * rc * avgEF / smax(1e-6f, 1.0f - rc * (1.0f - avgEF)));
    }
    const float eps = 1e-7f;
    const float ms = smax(eps, 1.0f - EFo) * smax(eps, 1.0f - EFi) / smax(eps, 1.0f - avgEF);
    return fss + rhoMs * (kInvPi * ms);
}

// ---------------------------------------------------------------------------------------------
// Shading point as seen by a material (the SurfaceInteraction fields materials read).
struct ShadePoint {
    V2 uv;                  // surface uv (texture lookups)
    const TexGPU* textures; // the scene's image textures (may be null)
    float footprint;        // ray-cone footprint at the hit (0: none; mip LOD)
    float uvDensity;
    V3 p;        // point
    V3 n;        // shading normal, facing the incoming ray
    V3 ng;       // outward geometric normal
    V3 tangent;
    bool frontFace;
    float wavelength;
};

struct BsdfSample {
    V3 wi;
    V3 f;
    float pdf;
    bool delta, passThrough, subsurface;
    V3 weight;
};

PE_HD V3 m3(const float* p) { return m3f(p); }

// Disney ShadingParams (disney.h:185-211) for a texture-free material.
struct DisneyParams {
    V3 base;
    float metallic, roughness, specular, clearCoat, clearCoatRoughness, ior, specTrans, coatIor;
    V3 coatTint, sheenColor;
    bool hasSheenColor;
    float anisotropy, sheen, sheenRoughness, diffuseRoughness, diffuseTransmission, subsurface;
    V3 edgeTint;
    float thinFilmThickness, thinFilmIor;
    bool inFlake;
    V3 flakeNormal, flakeColor;
    V3 normal, tangent;
    bool frontFace;
};

PE_HD uint32_t flakeHashCell(int x, int y, int z) {
    return hash32(static_cast<uint32_t>(x) * 0x8da6b343u ^
                  hash32(static_cast<uint32_t>(y) * 0xd8163841u ^ hash32(static_cast<uint32_t>(z) * 0xcb1ab31fu)));
}

// Metallic flakes as a 3-D Voronoi of hashed cells (disney.cpp:420-454).
PE_HD void resolveFlake(V3 point, float size, float density, float rough, DisneyParams& p) {
    const V3 q = point / size;
    const int cx0 = static_cast<int>(floorf(q.x));
    const int cy0 = static_cast<int>(floorf(q.y));
    const int cz0 = static_cast<int>(floorf(q.z));
    float best = 1e30f;
    uint32_t bestHash = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const uint32_t h = flakeHashCell(cx0 + dx, cy0 + dy, cz0 + dz);
                const V3 f = mk(static_cast<float>(cx0 + dx) + unitFloat24(h),
                                static_cast<float>(cy0 + dy) + unitFloat24(hash32(h ^ 0x68e31da4u)),
                                static_cast<float>(cz0 + dz) + unitFloat24(hash32(h ^ 0xb5297a4du)));
                const float d2 = len2(q - f);
                if (d2 < best) {
                    best = d2;
                    bestHash = h;
                }
            }
    if (unitFloat24(hash32(bestHash ^ 0x1b56c4e9u)) >= density) return;
    const float u1 = smin(unitFloat24(hash32(bestHash ^ 0x2c1b3c6du)), 0.999f);
    const float u2 = unitFloat24(hash32(bestHash ^ 0x297a2d39u));
    const float tan2 = rough * rough * u1 / (1.0f - u1);
    const float cosT = 1.0f / sqrtf(1.0f + tan2);
    const float sinT = sqrtf(smax(0.0f, 1.0f - cosT * cosT));
    const float phi = kTwoPi * u2;
    const Frame f = frameFromNormal(p.normal);
    p.inFlake = true;
    p.flakeNormal = normalize(toWorld(f, mk(sinT * cosf(phi), sinT * sinf(phi), cosT)));
}

// Image::sampleLevel (image.cpp:168-225): bilinear with wrap, texel centres at +0.5, on mip
// level `level` (clamped to the last; 0 without mipmaps).
PE_HD V3 texBilinear(const TexGPU& t, float u, float v, int level = 0) {
    if (t.width <= 0 || t.height <= 0) return mk(0.0f);
    const int l = t.levels > 1 && level > 0 ? (level < t.levels ? level : t.levels - 1) : 0;
    const int w = t.levelW[l], h = t.levelH[l];
    const float* texels = t.texels + t.levelOffset[l];
    u = u - floorf(u);
    v = v - floorf(v);
    const float x = u * static_cast<float>(w) - 0.5f;
    const float y = v * static_cast<float>(h) - 0.5f;
    const int x0 = static_cast<int>(floorf(x));
    const int y0 = static_cast<int>(floorf(y));
    const float fx = x - static_cast<float>(x0);
    const float fy = y - static_cast<float>(y0);
    auto wrap = [](int i, int n) {
        i %= n;
        return i < 0 ? i + n : i;
    };
    const int xa = wrap(x0, w), xb = wrap(x0 + 1, w), ya = wrap(y0, h), yb = wrap(y0 + 1, h);
    auto at = [&](int px, int py) {
        const float* c = texels + (static_cast<size_t>(py) * static_cast<size_t>(w) + static_cast<size_t>(px)) * 3;
        return mk(c[0], c[1], c[2]);
    };
    const V3 c0 = at(xa, ya) * (1.0f - fx) + at(xb, ya) * fx;
    const V3 c1 = at(xa, yb) * (1.0f - fx) + at(xb, yb) * fx;
    return c0 * (1.0f - fy) + c1 * fy;
}

// Image::sampleMip (image.cpp:227-239): trilinear between the two levels around `lod`.
PE_HD V3 texMip(const TexGPU& t, float u, float v, float lod) {
    if (t.levels <= 1 || lod <= 0.0f) return texBilinear(t, u, v, 0);
    const int maxLvl = t.levels - 1;
    const float clamped = sclamp(lod, 0.0f, static_cast<float>(maxLvl));
    const int l0 = static_cast<int>(floorf(clamped));
    const int l1 = l0 + 1 < maxLvl ? l0 + 1 : maxLvl;
    const float frac = clamped - static_cast<float>(l0);
    if (l0 == l1 || frac <= 1e-5f) return texBilinear(t, u, v, l0);
    return texBilinear(t, u, v, l0) * (1.0f - frac) + texBilinear(t, u, v, l1) * frac;
}

// sampleTex (disney.cpp:530-539): with a ray footprint and mipmaps, the level whose texels match
// the footprint; else level 0.
PE_HD V3 texLookup(const TexGPU& t, V2 uv, const ShadePoint& sp, float texScale) {
    if (sp.footprint > 0.0f && t.levels > 1) {
        const float density = sp.uvDensity > 0.0f ? sp.uvDensity : 1.0f;
        const float texelExtent = sqrtf(static_cast<float>(t.width) * static_cast<float>(t.height));
        const float footprintTexels = sp.footprint * density * texScale * texelExtent;
        const float lod = footprintTexels > 1.0f ? log2f(footprintTexels) : 0.0f;
        return texMip(t, uv.x, uv.y, lod);
    }
    return texBilinear(t, uv.x, uv.y, 0);
}

// DisneyMaterial::textureCoord (disney.cpp:517-526): the uv scaled, or a box projection of the
// point onto the plane across the geometric normal's largest axis.
PE_HD V2 textureCoord(const MatGPU& m, const ShadePoint& sp) {
    V2 uv;
    if (m.texMapping == 0) {
        uv = sp.uv;
    } else {
        const V3 n = len2(sp.ng) > 0.0f ? sp.ng : sp.n;
        const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
        const V3 p = sp.p;
        uv = (ax >= ay && ax >= az) ? mk2(p.z, p.y) : (ay >= az ? mk2(p.x, p.z) : mk2(p.x, p.y));
    }
    return mk2(uv.x * m.texScale, uv.y * m.texScale);
}

// The image maps of DisneyMaterial::resolve (disney.cpp:565-596): base colour, roughness (green),
// metalness (blue) and a tangent-space normal map.
PE_HDN void applyTextures(const MatGPU& m, const ShadePoint& sp, V3& base, float& roughness, float& metallic,
                          V3& normal) {
    const V2 uv = textureCoord(m, sp);
    if (m.texAlbedo >= 0) base = texLookup(sp.textures[m.texAlbedo], uv, sp, m.texScale);
    if (m.texRoughness >= 0) roughness = smax(0.001f, texLookup(sp.textures[m.texRoughness], uv, sp, m.texScale).y);
    if (m.texMetalness >= 0)
        metallic = sclamp(texLookup(sp.textures[m.texMetalness], uv, sp, m.texScale).z, 0.0f, 1.0f);
    if (m.texNormal >= 0) {
        const V3 c = texLookup(sp.textures[m.texNormal], uv, sp, m.texScale);
        const V3 nTs = mk(c.x * 2.0f - 1.0f, c.y * 2.0f - 1.0f, c.z * 2.0f - 1.0f);
        const V3 N = sp.n;
        V3 T = sp.tangent;
        if (len2(T) < 1e-8f) T = frameFromNormal(N).s;
        V3 B = cross(N, T);
        if (len2(B) < 1e-8f) {
            const Frame f = frameFromNormal(N);
            B = f.t;
            T = f.s;
        } else {
            B = normalize(B);
            T = normalize(cross(B, N));
        }
        normal = normalize(T * nTs.x + B * nTs.y + N * nTs.z);
        if (dot(normal, N) < 0.0f) normal = -normal;
    }
}

PE_HD DisneyParams disneyResolve(const MatGPU& m, const ShadePoint& sp) {
    DisneyParams p;
    p.base = m3(m.base);
    p.metallic = m.metallic;
    p.roughness = m.roughness;
    p.specular = m.specular;
    p.clearCoat = m.clearcoat;
    p.clearCoatRoughness = m.clearcoatRoughness;
    p.ior = m.ior;
    p.specTrans = m.specTrans;
    p.coatIor = m.coatIor;
    p.coatTint = m3(m.coatTint);
    p.sheenColor = m3(m.sheenColor);
    p.hasSheenColor = m.hasSheenColor != 0;
    p.anisotropy = m.anisotropy;
    p.sheen = m.sheen;
    p.sheenRoughness = m.sheenRoughness;
    p.diffuseRoughness = m.diffuseRoughness;
    p.diffuseTransmission = m.diffuseTransmission;
    p.subsurface = m.subsurface;
    p.normal = sp.n;
    p.tangent = sp.tangent;
    p.frontFace = sp.frontFace;
    if (sp.textures && (m.texAlbedo >= 0 || m.texRoughness >= 0 || m.texMetalness >= 0 || m.texNormal >= 0))
        applyTextures(m, sp, p.base, p.roughness, p.metallic, p.normal);
    p.edgeTint = m3(m.edgeTint);
    p.thinFilmThickness = m.thinFilmThickness;
    p.thinFilmIor = m.thinFilmIor;
    p.flakeColor = m3(m.flakeColor);
    p.inFlake = false;
    p.flakeNormal = mk(0.0f, 1.0f, 0.0f);
    if (m.flakeDensity > 0.0f) resolveFlake(sp.p, m.flakeSize, m.flakeDensity, m.flakeRoughness, p);
    return p;
}

PE_HD float f0FromIor(float ior) {
    const float r = (ior - 1.0f) / (ior + 1.0f);
    return r * r;
}
PE_HD float dielectricWeight(const DisneyParams& p) { return sclamp(2.0f * p.specular, 0.0f, 1.0f); }
PE_HD float dielectricF0(const DisneyParams& p) {
    return sclamp(f0FromIor(p.ior) * smax(1.0f, 2.0f * p.specular), 0.0f, 1.0f);
}
PE_HD float coatF0(const DisneyParams& p) { return sclamp(f0FromIor(p.coatIor), 0.0f, 1.0f); }
PE_HD float schlickClamped(float f0, float cosTheta) {
    return f0 + (1.0f - f0) * pow5(1.0f - sclamp(cosTheta, 0.0f, 1.0f));
}
PE_HD void anisoAlpha(float roughness, float anisotropy, float& ax, float& ay) {
    const float aspect = sqrtf(smax(0.1f, 1.0f - 0.9f * sclamp(anisotropy, 0.0f, 1.0f)));
    const float a = roughness * roughness;
    ax = a / aspect;
    ay = a * aspect;
}
PE_HD Frame shadingFrame(V3 nIn, V3 tangentIn) {
    const V3 n = len2(nIn) > 0.0f ? normalize(nIn) : mk(0.0f, 1.0f, 0.0f);
    V3 t = tangentIn - n * dot(tangentIn, n);
    if (len2(t) < 1e-8f) return frameFromNormal(n);
    t = normalize(t);
    V3 b = cross(n, t);
    if (len2(b) < 1e-8f) return frameFromNormal(n);
    b = normalize(b);
    t = normalize(cross(b, n));
    return frame3(t, b, n);
}
constexpr float kFlakeAlpha = 0.06f;

PE_HD V3 specularFresnel(const DisneyParams& p, float cosD) {
    const float f0d = dielectricF0(p);
    const float w = dielectricWeight(p);
    if (p.thinFilmThickness <= 0.0f) {
        const V3 fd = mk(w * schlickF(f0d, cosD));
        if (p.metallic <= 0.0f) return fd;
        return lerp3(fd, fresnelF82Tint(p.base, p.edgeTint, cosD), p.metallic);
    }
    const float sd = sqrtf(sclamp(f0d, 0.0f, 0.99f));
    const Cx nd = cx((1.0f + sd) / (1.0f - sd), 0.0f);
    const Cx diel[3] = {nd, nd, nd};
    const V3 fd = thinFilmRGB(cosD, p.thinFilmIor, diel, p.thinFilmThickness) * w;
    if (p.metallic <= 0.0f) return fd;
    Cx metal[3];
    for (int c = 0; c < 3; ++c) metal[c] = gulbrandsenIor(get(p.base, c), get(p.edgeTint, c));
    return lerp3(fd, thinFilmRGB(cosD, p.thinFilmIor, metal, p.thinFilmThickness), p.metallic);
}
PE_HD V3 multiScatterFactor(const TablesGPU* T, const DisneyParams& p, float cosO, float ax, float ay) {
    const float E = ggxDirectionalAlbedo(T, cosO, sqrtf(ax * ay));
    const V3 f0 = lerp3(mk(dielectricF0(p)), p.base, p.metallic);
    return mk(1.0f) + f0 * (1.0f / E - 1.0f);
}
PE_HD V3 evalFlake(V3 wo, V3 wi, const DisneyParams& p) {
    const Frame ff = frameFromNormal(p.flakeNormal);
    const V3 o = toLocal(ff, wo), i = toLocal(ff, wi);
    if (o.z <= 0.0f || i.z <= 0.0f) return mk(0.0f);
    const V3 h = normalize(o + i);
    const float D = ggxD(h, kFlakeAlpha, kFlakeAlpha);
    const float G = ggxG(o, i, kFlakeAlpha, kFlakeAlpha);
    const float c = dot(o, h);
    V3 F;
    for (int k = 0; k < 3; ++k) set(F, k, schlickF(get(p.flakeColor, k), c));
    return F * (D * G / (4.0f * o.z * i.z));
}
PE_HD float pdfFlake(V3 wo, V3 wi, const DisneyParams& p) {
    const Frame ff = frameFromNormal(p.flakeNormal);
    const V3 o = toLocal(ff, wo), i = toLocal(ff, wi);
    if (o.z <= 0.0f || i.z <= 0.0f) return 0.0f;
    const V3 h = normalize(o + i);
    const float c = dot(o, h);
    if (c <= 0.0f) return 0.0f;
    return ggxVisiblePdf(o, h, kFlakeAlpha, kFlakeAlpha) / (4.0f * c);
}

// Kulla–Conty layering of the dielectric specular over the base (disney.cpp:146-162).
struct DielectricLayer {
    float alpha, f0, weight, invOneMinusAvg;
};
PE_HD DielectricLayer makeLayer(const TablesGPU* T, const DisneyParams& p) {
    DielectricLayer l;
    float ax, ay;
    anisoAlpha(p.roughness, p.anisotropy, ax, ay);
    l.alpha = sqrtf(ax * ay);
    l.f0 = dielectricF0(p);
    l.weight = dielectricWeight(p);
    l.invOneMinusAvg = 1.0f / smax(1e-4f, 1.0f - l.weight * ggxSchlickAverageAlbedo(T, l.alpha, l.f0));
    return l;
}
PE_HD float layerTransmit(const TablesGPU* T, const DielectricLayer& l, float mu) {
    return smax(0.0f, 1.0f - l.weight * ggxSchlickAlbedo(T, mu, l.alpha, l.f0));
}
PE_HD float layerFactor(const TablesGPU* T, const DielectricLayer& l, float muO, float muI) {
    return layerTransmit(T, l, muO) * layerTransmit(T, l, muI) * l.invOneMinusAvg;
}
PE_HD float coatTransmit(const TablesGPU* T, const DisneyParams& p, float mu) {
    if (p.clearCoat <= 0.0f) return 1.0f;
    const float alphaC = p.clearCoatRoughness * p.clearCoatRoughness;
    return 1.0f - p.clearCoat * ggxSchlickAlbedo(T, mu, alphaC, coatF0(p));
}
PE_HD V3 coatTintFactor(const DisneyParams& p) {
    return p.clearCoat > 0.0f ? lerp3(mk(1.0f), p.coatTint, p.clearCoat) : mk(1.0f);
}
PE_HD V3 resolvedSheenColor(const DisneyParams& p) {
    if (p.sheen <= 0.0f || p.metallic >= 1.0f) return mk(0.0f);
    if (p.hasSheenColor) return p.sheenColor * (p.sheen * (1.0f - p.metallic));
    const float lum = luminance(p.base);
    const V3 tint = lum > 1e-6f ? p.base * (1.0f / lum) : mk(1.0f);
    return (mk(0.5f) + clamp3(tint, 0.0f, 1.0f) * 0.5f) * (p.sheen * (1.0f - p.metallic));
}
PE_HD float sheenScale(const TablesGPU* T, const DisneyParams& p, float s, float muO, float muI) {
    if (s <= 0.0f) return 1.0f;
    const float eo = smin(1.0f, charlieSheenAlbedo(T, muO, p.sheenRoughness));
    const float ei = smin(1.0f, charlieSheenAlbedo(T, muI, p.sheenRoughness));
    return smax(0.0f, smin(1.0f - s * eo, 1.0f - s * ei));
}
PE_HD V3 evalSheen(const TablesGPU* T, V3 color, const DisneyParams& p, float cosO, float cosI, float cosH) {
    const float norm = smax(smax(1.0f, charlieSheenAlbedo(T, cosO, p.sheenRoughness)),
                            charlieSheenAlbedo(T, cosI, p.sheenRoughness));
    return color * (charlieD(cosH, p.sheenRoughness) * charlieV(cosI, cosO) / norm);
}
PE_HD V3 evalSpecTransmission(V3 woL, V3 wiL, const DisneyParams& p) {
    const float stW = p.inFlake ? 0.0f : sclamp(p.specTrans, 0.0f, 1.0f) * (1.0f - p.metallic);
    if (stW <= 0.0f || woL.z <= 0.0f || wiL.z >= 0.0f) return mk(0.0f);
    const float etap = p.frontFace ? p.ior : (1.0f / p.ior);
    V3 wm = wiL * etap + woL;
    if (len2(wm) <= 1e-12f) return mk(0.0f);
    wm = normalize(wm);
    if (wm.z < 0.0f) wm = -wm;
    const float woDotH = dot(woL, wm);
    const float wiDotH = dot(wiL, wm);
    if (woDotH <= 0.0f || wiDotH >= 0.0f) return mk(0.0f);
    const float alpha = ggxClampAlpha(p.roughness * p.roughness);
    const float F = fresnelDielectric(p.frontFace ? woDotH : -woDotH, 1.0f, p.ior);
    const float D = ggxD(wm, alpha, alpha);
    const float G = ggxG(woL, mk(wiL.x, wiL.y, -wiL.z), alpha, alpha);
    const float s = wiDotH + woDotH / etap;
    const float denom = s * s * fabsf(wiL.z * woL.z);
    if (denom <= 1e-12f) return mk(0.0f);
    const float ft = D * (1.0f - F) * G * fabsf(wiDotH * woDotH) / (denom * etap * etap);
    return p.base * (stW * ft);
}
PE_HD float pdfSpecTransmission(V3 woL, V3 wiL, const DisneyParams& p) {
    if (woL.z <= 0.0f || wiL.z >= 0.0f) return 0.0f;
    const float etap = p.frontFace ? p.ior : (1.0f / p.ior);
    V3 wm = wiL * etap + woL;
    if (len2(wm) <= 1e-12f) return 0.0f;
    wm = normalize(wm);
    if (wm.z < 0.0f) wm = -wm;
    const float woDotH = dot(woL, wm);
    const float wiDotH = dot(wiL, wm);
    if (woDotH <= 0.0f || wiDotH >= 0.0f) return 0.0f;
    const float alpha = ggxClampAlpha(p.roughness * p.roughness);
    const float visible = ggxVisiblePdf(woL, wm, alpha, alpha);
    const float s = wiDotH + woDotH / etap;
    if (s * s <= 1e-12f) return 0.0f;
    return visible * fabsf(wiDotH) / (s * s);
}

// f(wo, wi) in the lobe groups of the render passes (LobeSplit, material.h:53-57).
struct LobeSplit3 {
    V3 diffuse, glossy, transmission;
};

// Sum of all lobes f(wo, wi) (disney.cpp:223-311).  split (may be null) receives the sum in
// lobe groups as DisneyMaterial::evalSplit forms it (disney.cpp:654-658).
PE_HDN V3 disneyEval(const TablesGPU* T, V3 wo, V3 wi, const DisneyParams& p, LobeSplit3* split) {
    const Frame frame = shadingFrame(p.normal, p.tangent);
    const V3 woL = toLocal(frame, wo);
    const V3 wiL = toLocal(frame, wi);
    if (split) split->diffuse = split->glossy = split->transmission = mk(0.0f);
    if (woL.z <= 0.0f) return mk(0.0f);
    const float cosThetaO = woL.z;
    const float coatO = coatTransmit(T, p, cosThetaO);
    const V3 cTint = coatTintFactor(p);
    const float stW = p.inFlake ? 0.0f : sclamp(p.specTrans, 0.0f, 1.0f) * (1.0f - p.metallic);
    const float opaqueDielectric = (1.0f - p.metallic) * (1.0f - sclamp(p.specTrans, 0.0f, 1.0f));
    const float trans = p.inFlake ? 0.0f : sclamp(p.diffuseTransmission, 0.0f, 1.0f) * opaqueDielectric;
    if (wiL.z <= 0.0f) {
        V3 ft = mk(0.0f);
        if (trans > 0.0f) {
            const float muI = -wiL.z;
            const DielectricLayer dl = makeLayer(T, p);
            const V3 sc = resolvedSheenColor(p);
            const float sh = sheenScale(T, p, smax3(sc.x, sc.y, sc.z), cosThetaO, muI);
            ft += p.base * (trans * kInvPi * coatO * layerFactor(T, dl, cosThetaO, muI) * sh) * cTint;
        }
        if (stW > 0.0f) ft += evalSpecTransmission(woL, wiL, p) * coatO * cTint;
        if (split) split->transmission = ft;
        return ft;
    }
    const V3 hL = normalize(woL + wiL);
    const float cosThetaI = wiL.z;
    const float cosThetaD = dot(woL, hL);
    V3 base, baseDiffuse = mk(0.0f);
    if (p.inFlake) {
        base = evalFlake(wo, wi, p);
    } else {
        const DielectricLayer dl = makeLayer(T, p);
        const float diffW = opaqueDielectric * (1.0f - sclamp(p.diffuseTransmission, 0.0f, 1.0f)) * (1.0f - p.subsurface);
        const V3 fDiffuse = diffW > 0.0f ? eonEval(p.base, p.diffuseRoughness, wiL, woL) *
                                               (diffW * layerFactor(T, dl, cosThetaO, cosThetaI))
                                         : mk(0.0f);
        float ax, ay;
        anisoAlpha(p.roughness, p.anisotropy, ax, ay);
        const float D = ggxD(hL, ax, ay);
        const float G = ggxG(woL, wiL, ax, ay);
        V3 F = specularFresnel(p, cosThetaD);
        if (stW > 0.0f && !p.frontFace) {
            const float fInt = fresnelDielectric(-cosThetaD, 1.0f, p.ior);
            F = lerp3(F, mk(fInt), stW);
        }
        const V3 fSpecular = (F * D * G) / (4.0f * cosThetaO * cosThetaI) * multiScatterFactor(T, p, cosThetaO, ax, ay);
        base = fDiffuse + fSpecular;
        baseDiffuse = fDiffuse;
        const V3 sc = resolvedSheenColor(p);
        if (!isBlack(sc)) {
            const float s = sheenScale(T, p, smax3(sc.x, sc.y, sc.z), cosThetaO, cosThetaI);
            base = base * s + evalSheen(T, sc, p, cosThetaO, cosThetaI, hL.z);
            baseDiffuse = baseDiffuse * s;
        }
    }
    if (p.clearCoat <= 0.0f) {
        if (split) {
            split->diffuse = baseDiffuse;
            split->glossy = base - baseDiffuse;
        }
        return base;
    }
    const float alphaC = p.clearCoatRoughness * p.clearCoatRoughness;
    const float Dc = ggxD(hL, alphaC, alphaC);
    const float Gc = ggxG(woL, wiL, alphaC, alphaC);
    const float f0c = coatF0(p);
    const float Fc = schlickClamped(f0c, cosThetaD);
    const float msC = 1.0f + f0c * (1.0f / ggxDirectionalAlbedo(T, cosThetaO, alphaC) - 1.0f);
    const V3 fCoat = mk(p.clearCoat * Fc * Dc * Gc / (4.0f * cosThetaO * cosThetaI) * msC);
    const V3 coatAtt = cTint * (coatO * coatTransmit(T, p, cosThetaI));
    if (split) {
        split->diffuse = baseDiffuse * coatAtt;
        split->glossy = (base - baseDiffuse) * coatAtt + fCoat;
    }
    return base * coatAtt + fCoat;
}

struct LobeWeights {
    float coat, spec, diffRefl, trans, sss, specTrans;
};
PE_HD LobeWeights disneyLobeWeights(const DisneyParams& p) {
    LobeWeights w;
    w.coat = 0.25f * p.clearCoat;
    if (p.inFlake) {
        w.spec = 1.0f - w.coat;
        w.diffRefl = w.trans = w.sss = w.specTrans = 0.0f;
        return w;
    }
    const float rem = 1.0f - w.coat;
    const float st = sclamp(p.specTrans, 0.0f, 1.0f) * (1.0f - p.metallic);
    w.spec = rem * lerpf(0.5f * (st > 0.0f ? 1.0f : dielectricWeight(p)), 1.0f, p.metallic);
    float pRest = rem - w.spec;
    w.specTrans = pRest * st;
    pRest -= w.specTrans;
    const float dTrans = sclamp(p.diffuseTransmission, 0.0f, 1.0f);
    w.trans = pRest * dTrans;
    w.diffRefl = pRest - w.trans;
    w.sss = p.metallic < 1.0f ? w.diffRefl * p.subsurface : 0.0f;
    w.diffRefl -= w.sss;
    return w;
}

PE_HDN float disneyPdf(V3 wo, V3 wi, const DisneyParams& p) {
    const Frame frame = shadingFrame(p.normal, p.tangent);
    const V3 woL = toLocal(frame, wo);
    const V3 wiL = toLocal(frame, wi);
    if (woL.z <= 0.0f) return 0.0f;
    const LobeWeights lw = disneyLobeWeights(p);
    if (wiL.z <= 0.0f) {
        float pdf = 0.0f;
        if (lw.trans > 0.0f) pdf += lw.trans * cosineHemispherePdf(-wiL.z);
        if (lw.specTrans > 0.0f) pdf += lw.specTrans * pdfSpecTransmission(woL, wiL, p);
        return pdf;
    }
    const V3 hL = normalize(woL + wiL);
    const float cosThetaD = dot(woL, hL);
    if (cosThetaD <= 0.0f) return 0.0f;
    const float pdfDiffuse = cosineHemispherePdf(wiL.z);
    float pdfSpecular;
    if (p.inFlake) {
        pdfSpecular = pdfFlake(wo, wi, p);
    } else {
        float ax, ay;
        anisoAlpha(p.roughness, p.anisotropy, ax, ay);
        pdfSpecular = ggxVisiblePdf(woL, hL, ax, ay) / (4.0f * cosThetaD);
    }
    float pdfCoat = 0.0f;
    if (lw.coat > 0.0f) {
        const float alphaC = p.clearCoatRoughness * p.clearCoatRoughness;
        pdfCoat = ggxVisiblePdf(woL, hL, alphaC, alphaC) / (4.0f * cosThetaD);
    }
    return lw.diffRefl * pdfDiffuse + lw.spec * pdfSpecular + lw.coat * pdfCoat;
}

PE_HD bool disneySampleSpecularLobe(const DisneyParams& p, const Frame& frame, V3 wo, V3 woL, float u1, float u2,
                                    V3& wiL) {
    if (p.inFlake) {
        const Frame ff = frameFromNormal(p.flakeNormal);
        const V3 o = toLocal(ff, wo);
        if (o.z <= 0.0f) return false;
        const V3 i = reflectV(o, ggxSampleVisibleNormal(o, kFlakeAlpha, kFlakeAlpha, u1, u2));
        if (i.z <= 0.0f) return false;
        wiL = toLocal(frame, toWorld(ff, i));
    } else {
        float ax, ay;
        anisoAlpha(p.roughness, p.anisotropy, ax, ay);
        wiL = reflectV(woL, ggxSampleVisibleNormal(woL, ax, ay, u1, u2));
    }
    return wiL.z > 0.0f;
}
PE_HD bool disneySampleSpecTransLobe(const DisneyParams& p, V3 woL, float u1, float u2, V3& wiL) {
    const float alpha = ggxClampAlpha(p.roughness * p.roughness);
    const V3 wm = ggxSampleVisibleNormal(woL, alpha, alpha, u1, u2);
    const float eta = p.frontFace ? (1.0f / p.ior) : p.ior;
    if (!refractV(woL, wm, eta, wiL)) return false;
    return wiL.z < 0.0f;
}

// DisneyMaterial::sampleFull (disney.cpp:680-729).
PE_HDN bool disneySample(const TablesGPU* T, V3 wo, const DisneyParams& p, float uc, V2 u, BsdfSample& out) {
    out.delta = false;
    out.subsurface = false;
    out.passThrough = false;
    out.weight = mk(0.0f);
    const Frame frame = shadingFrame(p.normal, p.tangent);
    const V3 woL = toLocal(frame, wo);
    if (woL.z <= 0.0f) return false;
    const LobeWeights lw = disneyLobeWeights(p);
    V3 wiL;
    if (uc < lw.coat) {
        const float alphaC = p.clearCoatRoughness * p.clearCoatRoughness;
        wiL = reflectV(woL, ggxSampleVisibleNormal(woL, alphaC, alphaC, u.x, u.y));
        if (wiL.z <= 0.0f) return false;
    } else if (uc < lw.coat + lw.spec) {
        if (!disneySampleSpecularLobe(p, frame, wo, woL, u.x, u.y, wiL)) return false;
    } else if (uc < lw.coat + lw.spec + lw.specTrans) {
        if (!disneySampleSpecTransLobe(p, woL, u.x, u.y, wiL)) return false;
    } else if (uc < lw.coat + lw.spec + lw.specTrans + lw.diffRefl) {
        wiL = sampleCosineHemisphere(u);
    } else if (uc < lw.coat + lw.spec + lw.specTrans + lw.diffRefl + lw.sss) {
        wiL = sampleCosineHemisphere(u);
        wiL.z = -wiL.z;
        const float opaqueDielectric = (1.0f - p.metallic) * (1.0f - sclamp(p.specTrans, 0.0f, 1.0f));
        const float trans = sclamp(p.diffuseTransmission, 0.0f, 1.0f);
        const float coatO = coatTransmit(T, p, woL.z);
        const V3 sc = resolvedSheenColor(p);
        const float sheenO = sheenScale(T, p, smax3(sc.x, sc.y, sc.z), woL.z, 1.0f);
        const float layerO = layerTransmit(T, makeLayer(T, p), woL.z);
        const float w = p.subsurface * opaqueDielectric * (1.0f - trans) * coatO * sheenO * layerO / smax(lw.sss, 1e-6f);
        out.wi = normalize(toWorld(frame, wiL));
        out.subsurface = true;
        out.weight = coatTintFactor(p) * w;
        out.pdf = lw.sss * cosineHemispherePdf(-wiL.z);
        out.f = out.weight * out.pdf / smax(-wiL.z, 1e-6f);
        return out.pdf > 0.0f;
    } else {
        wiL = sampleCosineHemisphere(u);
        wiL.z = -wiL.z;
    }
    out.wi = normalize(toWorld(frame, wiL));
    out.f = disneyEval(T, wo, out.wi, p, nullptr);
    out.pdf = disneyPdf(wo, out.wi, p);
    return out.pdf > 0.0f;
}

// Chiang 2016 albedo inversion for the random-walk coefficients (disney.cpp:738-757).
PE_HD bool disneySubsurfaceCoeffs(const MatGPU& m, const DisneyParams& p, V3& sigmaT, V3& albedo, float& g) {
    if (m.subsurface <= 0.0f) return false;
    g = m.ssAniso;
    for (int c = 0; c < 3; ++c) {
        const float A = sclamp(get(p.base, c), 0.0f, 0.999f);
        const float d = smax(m.ssRadius[c] * m.ssScale, 1e-7f);
        const float alpha = 1.0f - expf(A * (-5.09406f + A * (2.61188f - 4.31805f * A)));
        const float sVal = 1.9f - A + 3.5f * (A - 0.8f) * (A - 0.8f);
        float sT = 1.0f / smax(d * sVal, 1e-12f);
        float sS = alpha * sT;
        const float sA = sT - sS;
        sS /= (1.0f - g);
        sT = sS + sA;
        set(sigmaT, c, sT);
        set(albedo, c, sT > 0.0f ? sS / sT : 0.0f);
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// Lambertian
PE_HD V3 lambertEval(const MatGPU& m, V3 wo, V3 wi, V3 n, float& pdf) {
    const Frame f = frameFromNormal(n);
    const float cosI = toLocal(f, wi).z;
    const float cosO = toLocal(f, wo).z;
    if (cosI <= 0.0f || cosO <= 0.0f) {
        pdf = 0.0f;
        return mk(0.0f);
    }
    pdf = cosineHemispherePdf(cosI);
    return m3(m.base) * kInvPi;
}
PE_HD bool lambertSample(const MatGPU& m, V3 wo, V3 n, V2 u, BsdfSample& out) {
    out.delta = false;
    out.passThrough = false;
    out.subsurface = false;
    out.weight = mk(0.0f);
    const Frame f = frameFromNormal(n);
    const V3 woL = toLocal(f, wo);
    if (woL.z <= 0.0f) return false;
    const V3 wiL = sampleCosineHemisphere(u);
    out.wi = normalize(toWorld(f, wiL));
    const float cosI = wiL.z;
    if (cosI <= 0.0f) return false;
    out.f = m3(m.base) * kInvPi;
    out.pdf = cosineHemispherePdf(cosI);
    return true;
}

// ---------------------------------------------------------------------------------------------
// Mirror
PE_HD bool mirrorSample(const MatGPU& m, V3 wo, V3 n, BsdfSample& out) {
    out.delta = true;
    out.passThrough = false;
    out.subsurface = false;
    out.weight = mk(0.0f);
    const Frame f = frameFromNormal(n);
    const V3 woL = toLocal(f, wo);
    if (woL.z <= 0.0f) return false;
    const V3 wiL = mk(-woL.x, -woL.y, woL.z);
    out.wi = normalize(toWorld(f, wiL));
    out.pdf = 1.0f;
    out.f = m3(m.base) / wiL.z;
    return true;
}

// ---------------------------------------------------------------------------------------------
// Dielectric (smooth / rough / thin-walled)
struct GlassLocal {
    Frame frame;
    V3 wo;
};
PE_HD GlassLocal glassFrame(V3 woW, const ShadePoint& sp) {
    const V3 outward = sp.frontFace ? sp.n : -sp.n;
    const V3 ng = len2(sp.ng) > 1e-12f ? normalize(sp.ng) : normalize(outward);
    V3 ns = len2(sp.n) > 1e-12f ? normalize(sp.n) : ng;
    if (dot(ns, ng) < 0.0f) ns = -ns;
    if (dot(woW, ns) * dot(woW, ng) <= 0.0f) ns = ng;
    GlassLocal g;
    g.frame = frameFromNormal(ns);
    g.wo = toLocal(g.frame, woW);
    return g;
}
PE_HD bool generalizedHalf(V3 wo, V3 wi, float ior, V3& wm, float& etap) {
    const float cosO = wo.z, cosI = wi.z;
    if (cosO == 0.0f || cosI == 0.0f) return false;
    const bool reflect = cosO * cosI > 0.0f;
    etap = reflect ? 1.0f : (cosO > 0.0f ? ior : 1.0f / ior);
    wm = wi * etap + wo;
    if (len2(wm) <= 1e-12f) return false;
    wm = normalize(wm);
    if (wm.z < 0.0f) wm = -wm;
    if (dot(wm, wi) * cosI <= 0.0f || dot(wm, wo) * cosO <= 0.0f) return false;
    return true;
}
PE_HD V3 glassEvalRough(V3 wo, V3 wi, float ior, float alpha, V3 tint) {
    V3 wm;
    float etap = 1.0f;
    if (!generalizedHalf(wo, wi, ior, wm, etap)) return mk(0.0f);
    const float cosO = wo.z, cosI = wi.z;
    const float woDotH = dot(wo, wm), wiDotH = dot(wi, wm);
    const float F = fresnelDielectric(woDotH, 1.0f, ior);
    const float D = ggxD(wm, alpha, alpha);
    const float G = ggxG(wo, wi, alpha, alpha);
    if (cosO * cosI > 0.0f) return tint * (D * G * F / fabsf(4.0f * cosI * cosO));
    const float s = wiDotH + woDotH / etap;
    const float denom = s * s * cosI * cosO;
    if (fabsf(denom) <= 1e-12f) return mk(0.0f);
    const float ft = D * (1.0f - F) * G * fabsf(wiDotH * woDotH / denom);
    return tint * (ft / (etap * etap));
}
PE_HD float glassPdfRough(V3 wo, V3 wi, float ior, float alpha) {
    V3 wm;
    float etap = 1.0f;
    if (!generalizedHalf(wo, wi, ior, wm, etap)) return 0.0f;
    const float woDotH = dot(wo, wm), wiDotH = dot(wi, wm);
    const float R = fresnelDielectric(woDotH, 1.0f, ior);
    const float visible = ggxVisiblePdf(wo, wm, alpha, alpha);
    if (wo.z * wi.z > 0.0f) return visible / (4.0f * fabsf(woDotH)) * R;
    const float s = wiDotH + woDotH / etap;
    if (s * s <= 1e-12f) return 0.0f;
    return visible * fabsf(wiDotH) / (s * s) * (1.0f - R);
}
// Cauchy dispersion from the Abbe number (src/core/color/spectral.cpp:89-97).
PE_HD float cauchyIor(float nd, float abbe, float lambdaNm) {
    if (abbe <= 0.0f) return nd;
    const float lD = 0.58756f, lF = 0.48613f, lC = 0.65627f;
    const float B = (nd - 1.0f) / (abbe * (1.0f / (lF * lF) - 1.0f / (lC * lC)));
    const float A = nd - B / (lD * lD);
    const float l = lambdaNm * 1e-3f;
    return A + B / (l * l);
}
PE_HD float glassIorAt(const MatGPU& m, float wavelength) {
    if (m.abbe <= 0.0f || wavelength <= 0.0f) return m.ior;
    return smax(1.0001f, cauchyIor(m.ior, m.abbe, wavelength));
}
PE_HD V3 thinWallReflectance(const MatGPU& m, float cosTheta) {
    cosTheta = sclamp(fabsf(cosTheta), 0.0f, 1.0f);
    if (m.filmThickness > 0.0f) {
        const Cx air[3] = {cx(1.0f, 0.0f), cx(1.0f, 0.0f), cx(1.0f, 0.0f)};
        return thinFilmRGB(cosTheta, m.ior, air, m.filmThickness);
    }
    const float R = fresnelDielectric(cosTheta, 1.0f, m.ior);
    return mk(2.0f * R / (1.0f + R));
}
PE_HD V3 glassShadowTransmittance(const MatGPU& m, V3 ng, V3 n, V3 dir) {
    if (!m.thinWalled) return mk(0.0f);
    const V3 nn = len2(ng) > 0.0f ? normalize(ng) : n;
    return (mk(1.0f) - thinWallReflectance(m, dot(dir, nn))) * m3(m.base);
}
PE_HDN V3 glassEval(const MatGPU& m, V3 wo, V3 wi, const ShadePoint& sp, float& pdf) {
    pdf = 0.0f;
    if (m.glassRoughness <= 1e-3f) return mk(0.0f);
    const GlassLocal g = glassFrame(wo, sp);
    const float ior = glassIorAt(m, sp.wavelength);
    const float alpha = ggxClampAlpha(m.glassRoughness * m.glassRoughness);
    const V3 wiL = toLocal(g.frame, wi);
    pdf = glassPdfRough(g.wo, wiL, ior, alpha);
    return glassEvalRough(g.wo, wiL, ior, alpha, m3(m.base));
}
// Dielectric::sampleFull / sampleWithLobe (dielectric.cpp:166-294).
PE_HDN bool glassSample(const MatGPU& m, V3 woW, const ShadePoint& sp, float uc, V2 u, BsdfSample& out) {
    out.subsurface = false;
    out.passThrough = false;
    out.weight = mk(0.0f);
    const V3 tint = m3(m.base);
    if (m.thinWalled) {
        out.delta = true;
        const V3 n = sp.n;
        const float cosO = dot(woW, n);
        if (cosO == 0.0f) return false;
        const V3 R = thinWallReflectance(m, cosO);
        const float pr = sclamp((R.x + R.y + R.z) / 3.0f, 1e-4f, 1.0f - 1e-4f);
        const float c = fabsf(cosO);
        if (uc < pr) {
            out.wi = normalize(n * (2.0f * cosO) - woW);
            out.pdf = pr;
            out.f = tint * R / c;
        } else {
            out.wi = -woW;
            out.pdf = 1.0f - pr;
            out.f = tint * (mk(1.0f) - R) / c;
            out.passThrough = true;
        }
        return true;
    }
    const bool sharp = m.glassRoughness <= 1e-3f;
    out.delta = sharp;
    const GlassLocal g = glassFrame(woW, sp);
    const V3 wo = g.wo;
    if (wo.z == 0.0f) return false;
    const bool entering = wo.z > 0.0f;
    const float ior = glassIorAt(m, sp.wavelength);
    const float eta = entering ? (1.0f / ior) : ior;
    if (sharp) {
        const float F = fresnelDielectric(wo.z, 1.0f, ior);
        V3 wiL = mk(-wo.x, -wo.y, wo.z);
        V3 weight;
        if (uc < F) {
            out.pdf = F;
            weight = tint * F;
        } else {
            const V3 n = mk(0.0f, 0.0f, entering ? 1.0f : -1.0f);
            if (!refractV(wo, n, eta, wiL)) {
                wiL = mk(-wo.x, -wo.y, wo.z);
                out.pdf = 1.0f;
                weight = tint;
            } else {
                out.pdf = 1.0f - F;
                weight = tint * ((1.0f - F) * eta * eta);
            }
        }
        out.wi = normalize(toWorld(g.frame, wiL));
        out.f = weight / smax(fabsf(dot(out.wi, sp.n)), 1e-6f);
        return true;
    }
    const float alpha = ggxClampAlpha(m.glassRoughness * m.glassRoughness);
    const V3 wm = ggxSampleVisibleNormal(wo, alpha, alpha, u.x, u.y);
    const float R = fresnelDielectric(dot(wo, wm), 1.0f, ior);
    V3 wiL;
    if (uc < R) {
        wiL = reflectV(wo, wm);
        if (wiL.z * wo.z <= 0.0f) return false;
    } else {
        const V3 n = entering ? wm : -wm;
        if (!refractV(wo, n, eta, wiL)) return false;
        if (wiL.z * wo.z >= 0.0f) return false;
    }
    out.f = glassEvalRough(wo, wiL, ior, alpha, tint);
    out.pdf = glassPdfRough(wo, wiL, ior, alpha);
    out.wi = normalize(toWorld(g.frame, wiL));
    return out.pdf > 0.0f && !isBlack(out.f);
}

// ---------------------------------------------------------------------------------------------
// Dispatch (Material::evalPdf / sampleFull).  MT >= 0 fixes the material type at compile time
// (a kernel that shades one material kind carries only that kind's code); MT < 0 reads m.type.
template <int MT>
PE_HD V3 bsdfEvalPdfT(const TablesGPU* T, const MatGPU& m, V3 wo, V3 wi, const ShadePoint& sp, float& pdf,
                      LobeSplit3* split) {
    const int type = MT >= 0 ? MT : m.type;
    if (split) split->diffuse = split->glossy = split->transmission = mk(0.0f);
    V3 f;
    switch (type) {
        case 0:
            f = lambertEval(m, wo, wi, sp.n, pdf);
            break;
        case 1: {
            const DisneyParams p = disneyResolve(m, sp);
            pdf = disneyPdf(wo, wi, p);
            return disneyEval(T, wo, wi, p, split);
        }
        case 2:
            f = glassEval(m, wo, wi, sp, pdf);
            break;
        default:
            pdf = 0.0f;
            return mk(0.0f);
    }
    if (split) {
        // Material::evalSplit (material.h:154-160) and Dielectric::evalSplit (dielectric.cpp:279-286):
        // same side of the geometric surface → diffuse (glass: glossy), else transmission
        const V3 nn = len2(sp.ng) > 0.0f ? sp.ng : sp.n;
        if (dot(wo, nn) * dot(wi, nn) >= 0.0f) (type == 2 ? split->glossy : split->diffuse) = f;
        else split->transmission = f;
    }
    return f;
}

PE_HD V3 bsdfEvalPdf(const TablesGPU* T, const MatGPU& m, V3 wo, V3 wi, const ShadePoint& sp, float& pdf,
                     LobeSplit3* split) {
    return bsdfEvalPdfT<-1>(T, m, wo, wi, sp, pdf, split);
}

template <int MT>
PE_HD bool bsdfSampleT(const TablesGPU* T, const MatGPU& m, V3 wo, const ShadePoint& sp, float uc, V2 u,
                       BsdfSample& out) {
    switch (MT >= 0 ? MT : m.type) {
        case 0:
            return lambertSample(m, wo, sp.n, u, out);
        case 1:
            return disneySample(T, wo, disneyResolve(m, sp), uc, u, out);
        case 2:
            return glassSample(m, wo, sp, uc, u, out);
        case 3:
            return mirrorSample(m, wo, sp.n, out);
        default:
            return false;
    }
}

PE_HD bool bsdfSample(const TablesGPU* T, const MatGPU& m, V3 wo, const ShadePoint& sp, float uc, V2 u,
                      BsdfSample& out) {
    return bsdfSampleT<-1>(T, m, wo, sp, uc, u, out);
}

} // namespace pe
