// pe_trace.cuh — ray/scene queries on the device: Owen-Sobol sampling, the camera ray of
// Renderer::tracePixel, BVH traversal (closest hit and any hit), the hit record of
// Triangle::fillHit and the robust ray-spawn rules of ray_spawn.h.
//
// Rounding: this file is compiled with -fmad=false and IEEE division / square root, and every
// expression keeps the reference's operand order, so the slab test, Möller–Trumbore and the hit
// record produce the reference CPU path's floats bit for bit.
#pragma once

#include <limits>

#include "pe_wave.h"

#include "pe_math.h"
#include "pe_scene.h"

namespace pe {

// ---- Owen-scrambled Sobol (src/samplers/sobol_sampler.cpp:111-146) --------------------------
struct Sobol {
    uint32_t pixelHash;
    uint32_t revIndex;
    uint32_t dim;
};
__device__ __forceinline__ uint32_t revSobol1(const TablesGPU* T, uint32_t index) {
    return __ldg(&T->sobolTab[0][index & 0xFFu]) ^ __ldg(&T->sobolTab[1][(index >> 8) & 0xFFu]) ^
           __ldg(&T->sobolTab[2][(index >> 16) & 0xFFu]) ^ __ldg(&T->sobolTab[3][index >> 24]);
}
__device__ __forceinline__ float get1D(Sobol& s) {
    const uint32_t seed = hashMix(s.pixelHash, s.dim++);
    const uint32_t index = rev32(lkPermute(s.revIndex, seed));
    return unitFloat24(rev32(lkPermute(index, hashMix(seed, 0u))));
}
__device__ __forceinline__ V2 get2D(const TablesGPU* T, Sobol& s) {
    const uint32_t seed = hashMix(s.pixelHash, s.dim++);
    const uint32_t index = rev32(lkPermute(s.revIndex, seed));
    const uint32_t x = rev32(lkPermute(index, hashMix(seed, 0u)));
    const uint32_t y = rev32(lkPermute(revSobol1(T, index), hashMix(seed, 1u)));
    return mk2(unitFloat24(x), unitFloat24(y));
}

// ---- camera ray (renderer.cpp:139-160, pixel_filter.cpp:84-91, perspective_camera.cpp:36-40) --
__device__ __forceinline__ float filterSample1D(const float* cdf, float filterWidth, float u) {
    if (cdf[0] < 0.0f) return (u - 0.5f) * filterWidth;
    // std::upper_bound over 513 entries
    int lo = 0, count = kFilterBins + 1;
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
    const int i = iclamp(lo - 1, 0, kFilterBins - 1);
    const float c0 = cdf[i], c1 = cdf[i + 1];
    const float t = c1 > c0 ? (u - c0) / (c1 - c0) : 0.5f;
    const float radius = 0.5f * filterWidth;
    return -radius + (static_cast<float>(i) + sclamp(t, 0.0f, 1.0f)) * (filterWidth / kFilterBins);
}
// Camera::generateRay(u, v, lens, time) with a shutter-close pose and 0 < time (camera.h:58-90):
// the two descriptions mixed linearly, a round lens of the mixed radius.
static __device__ __noinline__ void cameraRayMoving(const CamDev& c, float sx, float sy, V2 lens, float t, V3& o, V3& d) {
    const float b = 1.0f - t;
    auto mix3 = [&](V3 p, V3 q) { return p * b + q * t; };
    const V3 ll = mix3(c.lowerLeft, c.lowerLeft1), horiz = mix3(c.horizontal, c.horizontal1),
             vert = mix3(c.vertical, c.vertical1);
    if (c.orthographic) {
        o = ll + horiz * sx + vert * sy;
        d = normalize(mix3(c.forward, c.forward1));
        return;
    }
    const V3 pos = mix3(c.position, c.position1);
    const float radius = c.lensRadius * b + c.lensRadius1 * t;
    o = pos;
    if (radius > 0.0f) {
        const V3 cu = normalize(mix3(c.u, c.u1)), cv = normalize(mix3(c.v, c.v1));
        const V2 l = sampleDiskConcentric(lens);
        const V2 lp = mk2(l.x * radius, l.y * radius);
        o = pos + cu * lp.x + cv * lp.y;
    }
    const V3 target = ll + horiz * sx + vert * sy;
    d = normalize(target - o);
}

// Primary ray of pixel (x, y): consumes Sobol dimensions 0 (filter) and 1 (lens), and with motion
// blur 2 (the shutter time, renderer.cpp:152-153), returned in `time` (0 without).
__device__ __forceinline__ void cameraRay(const TablesGPU* T, const float* filterCdf, const CamDev& c, float filterWidth,
                                          int x, int y, int w, int h, Sobol& s, V3& o, V3& d, bool motion = false,
                                          float* time = nullptr) {
    const V2 u = get2D(T, s);
    const float ox = filterSample1D(filterCdf, filterWidth, u.x);
    const float oy = filterSample1D(filterCdf, filterWidth, u.y);
    const float sx = (static_cast<float>(x) + 0.5f + ox) / static_cast<float>(w);
    const float sy = 1.0f - (static_cast<float>(y) + 0.5f + oy) / static_cast<float>(h);
    const V2 lens = get2D(T, s); // lens sample (consumed by every camera)
    if (motion) {
        const float t = sclamp(get1D(s), 0.0f, 1.0f);
        if (time) *time = t;
        if (c.hasEnd && t > 0.0f) {
            cameraRayMoving(c, sx, sy, lens, t, o, d);
            return;
        }
    } else if (time) {
        *time = 0.0f;
    }
    const V3 target = c.lowerLeft + sx * c.horizontal + sy * c.vertical;
    if (c.orthographic) {
        // OrthographicCamera::generateRay (orthographic_camera.cpp:24-27)
        o = target;
        d = c.forward;
    } else if (c.lensRadius > 0.0f) {
        // ThinLensCamera::generateRay (thin_lens_camera.cpp:51-64): the focus-plane point seen
        // from a point of the aperture (disk, or polygon of `blades` sides, :37-49)
        V2 l;
        if (c.blades >= 3) {
            const float n = static_cast<float>(c.blades);
            const float scaled = smin(lens.x * n, n - 1e-4f);
            const float k = floorf(scaled);
            const float ux = scaled - k;
            const float a0 = c.bladeRotation + kTwoPi * k / n;
            const float a1 = a0 + kTwoPi / n;
            const float su0 = sqrtf(ux);
            const float bx = 1.0f - su0, by = lens.y * su0; // uniformSampleTriangle
            l = mk2(cosf(a0) * bx + cosf(a1) * by, sinf(a0) * bx + sinf(a1) * by);
        } else {
            l = sampleDiskConcentric(lens);
        }
        const V2 lp = mk2(l.x * c.lensRadius, l.y * c.lensRadius);
        o = c.position + c.u * lp.x + c.v * lp.y;
        d = normalize(target - o);
    } else {
        o = c.position;
        d = normalize(target - c.position);
    }
}

// ---- BVH traversal -------------------------------------------------------------------------
// Slab test of BVH::hitBox (bvh.cpp:269-283), std::max/min argument order kept so NaNs resolve
// exactly as there.
__device__ __forceinline__ bool slab(float lox, float hix, float loy, float hiy, float loz, float hiz, V3 o, V3 inv,
                                     float tMin, float tMax, float& tNear) {
    float tx0 = (lox - o.x) * inv.x, tx1 = (hix - o.x) * inv.x;
    if (tx0 > tx1) { const float t = tx0; tx0 = tx1; tx1 = t; }
    float ty0 = (loy - o.y) * inv.y, ty1 = (hiy - o.y) * inv.y;
    if (ty0 > ty1) { const float t = ty0; ty0 = ty1; ty1 = t; }
    float tz0 = (loz - o.z) * inv.z, tz1 = (hiz - o.z) * inv.z;
    if (tz0 > tz1) { const float t = tz0; tz0 = tz1; tz1 = t; }
    const float t0 = smax(smax(tMin, tx0), smax(ty0, tz0));
    const float t1 = smin(smin(tMax, tx1), smin(ty1, tz1)) * 1.0000004f;
    tNear = t0;
    return t0 <= t1;
}

// Lean Möller–Trumbore of BVH::hitTriangleLean (bvh.cpp:302-316).
__device__ __forceinline__ bool triLean(const float4 a, const float4 b, const float4 c, V3 o, V3 d, float tMin,
                                        float tMax, float& t, float& uu, float& vv) {
    const V3 v0 = mk(a.x, a.y, a.z), e1 = mk(b.x, b.y, b.z), e2 = mk(c.x, c.y, c.z);
    const V3 h = cross(d, e2);
    const float A = dot(e1, h);
    if (A * A <= a.w) return false;
    const float f = 1.0f / A;
    const V3 s = o - v0;
    const float u = f * dot(s, h);
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    const V3 q = cross(s, e1);
    const float v = f * dot(d, q);
    if (!(v >= 0.0f && u + v <= 1.0f)) return false;
    t = f * dot(e2, q);
    uu = u;
    vv = v;
    return t >= tMin && t <= tMax;
}

// Sphere::intersect's root choice (src/geometry/sphere.cpp:12-40) with solveQuadratic
// (src/core/math/utils.h:64-88): the nearer root inside [tMin, tMax], else the farther one.
__device__ __forceinline__ bool sphereLean(const float4 a, V3 o, V3 d, float tMin, float tMax, float& t) {
    const V3 oc = o - mk(a.x, a.y, a.z);
    const float qa = dot(d, d);
    const float qb = 2.0f * dot(oc, d);
    const float qc = dot(oc, oc) - a.w * a.w;
    float t0, t1;
    if (fabsf(qa) < 1e-6f) {
        if (fabsf(qb) < 1e-6f) return false;
        t0 = t1 = -qc / qb;
    } else {
        const float disc = qb * qb - 4.0f * qa * qc;
        if (disc < 0.0f) return false;
        const float sq = sqrtf(disc);
        const float q = -0.5f * (qb + (qb < 0.0f ? -sq : sq));
        t0 = q / qa;
        t1 = qc / q;
        if (t0 > t1) {
            const float x = t0;
            t0 = t1;
            t1 = x;
        }
    }
    float th = t0;
    if (th < tMin || th > tMax) {
        th = t1;
        if (th < tMin || th > tMax) return false;
    }
    t = th;
    return true;
}

struct Hit {
    float t, u, v;
    int32_t prim; // leaf-order primitive index, -1 = miss
    uint32_t meta; // visibility mask | material type << 8 of the hit triangle
};

__device__ __forceinline__ void leafRange(int ref, int& first, int& count) {
    const uint32_t v = ~static_cast<uint32_t>(ref);
    first = static_cast<int>(v >> 8);
    count = static_cast<int>(v & 0xFFu) + 1;
}

// Transform::transformPoint / transformVector (transform.cpp:15-40) with a row-major 4×4, in
// global memory (an instance's own pose) or a thread's local array (a pose between).
__device__ __forceinline__ V3 xfPointD(const float4* m, V3 p) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2], r3 = m[3];
    const float x = r0.x * p.x + r0.y * p.y + r0.z * p.z + r0.w;
    const float y = r1.x * p.x + r1.y * p.y + r1.z * p.z + r1.w;
    const float z = r2.x * p.x + r2.y * p.y + r2.z * p.z + r2.w;
    const float w = r3.x * p.x + r3.y * p.y + r3.z * p.z + r3.w;
    if (w != 1.0f && w != 0.0f) {
        const float iw = 1.0f / w;
        return mk(x * iw, y * iw, z * iw);
    }
    return mk(x, y, z);
}
__device__ __forceinline__ V3 xfVectorD(const float4* m, V3 v) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2];
    return mk(r0.x * v.x + r0.y * v.y + r0.z * v.z, r1.x * v.x + r1.y * v.y + r1.z * v.z,
              r2.x * v.x + r2.y * v.y + r2.z * v.z);
}
// A closest hit inside mesh instance `inst` at its BLAS-local record `local` (negative, never -1).
__device__ __forceinline__ int32_t instanceHitCode(int inst, int local) {
    return static_cast<int32_t>(0x80000000u | (static_cast<uint32_t>(inst) << 21) | static_cast<uint32_t>(local));
}
__device__ __forceinline__ bool isInstanceHit(int32_t prim) { return prim < -1; }
// A miss: -1 only (instance hits are negative too).
__device__ __forceinline__ bool isMiss(int32_t prim) { return prim == -1; }
__device__ __forceinline__ int instanceOfHit(int32_t prim) { return static_cast<int>((static_cast<uint32_t>(prim) >> 21) & 0x3FFu); }
__device__ __forceinline__ int localOfHit(int32_t prim) { return static_cast<int>(static_cast<uint32_t>(prim) & 0x1FFFFFu); }

template <bool COUNT, int LEVEL>
__device__ void walkClosest(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float& tMax,
                            Hit& best, uint32_t& nodeVisits, uint32_t& triTests, float time);
template <bool COUNT, int SD, int LEVEL>
__device__ void walkClosestWide(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float& tMax,
                                Hit& best, uint32_t& nodeVisits, uint32_t& triTests, uint2* sstack, float time);
template <bool COUNT, int LEVEL>
__device__ bool walkAny(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float tMax,
                        uint32_t& nodeVisits, uint32_t& triTests, float time);
template <bool COUNT, int LEVEL, int AW = 0>
__device__ bool walkAnyWide(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float tMax,
                            uint32_t& nodeVisits, uint32_t& triTests, float time);

// MeshInstance::transformAt (mesh_instance.cpp:31-34): the instance's matrices at shutter time
// `time` — its own (no motion, or time ≤ 0), the shutter-close pose (time ≥ 1), or
// interpolateTransform's pose between, written to `buf` (local-to-world rows, then the inverse).
static __device__ __noinline__ void instancePoseBetween(const MotionTRS& M, float a, float4* buf, float& uvScale) {
    float m[16], inv[16];
    motionPoseAt(M, a, m, inv);
    for (int r = 0; r < 4; ++r) {
        buf[r] = make_float4(m[4 * r], m[4 * r + 1], m[4 * r + 2], m[4 * r + 3]);
        buf[4 + r] = make_float4(inv[4 * r], inv[4 * r + 1], inv[4 * r + 2], inv[4 * r + 3]);
    }
    uvScale = uvScaleOf(m);
}
__device__ __forceinline__ void instancePose(const SceneGPU& S, const InstGPU& I, float time, float4* buf,
                                             const float4*& l2w, const float4*& w2l, float& uvScale) {
    l2w = I.l2w;
    w2l = I.w2l;
    uvScale = I.uvScale;
    if (I.motion < 0) return;
    const float a = sclamp(time, 0.0f, 1.0f);
    if (a <= 0.0f) return;
    const InstMotionGPU& M = S.motions[I.motion];
    if (a >= 1.0f) {
        l2w = M.l2w1;
        w2l = M.w2l1;
        uvScale = M.uvScale1;
        return;
    }
    instancePoseBetween(M.trs, a, buf, uvScale);
    l2w = buf;
    w2l = buf + 4;
}

// MeshInstance::intersect (mesh_instance.cpp:104-115): the ray carried into the instance's space
// by its world-to-local matrix at the ray's time (direction not renormalised, so t is shared), its
// BLAS walked with every visibility bit; a hit shortens the world ray as it shortens the local one.
template <bool COUNT, bool WIDE>
__device__ __noinline__ void instanceClosest(const SceneGPU& S, int inst, uint32_t meta, V3 o, V3 d, float tMin,
                                             float& tMax, Hit& best, uint32_t& nodeVisits, uint32_t& triTests,
                                             float time) {
    const InstGPU& I = S.instances[inst];
    float4 buf[8];
    const float4 *l2w, *w2l;
    float uvScale;
    instancePose(S, I, time, buf, l2w, w2l, uvScale);
    const V3 lo = xfPointD(w2l, o), ld = xfVectorD(w2l, d);
    const V3 linv = mk(1.0f / ld.x, 1.0f / ld.y, 1.0f / ld.z);
    Hit h;
    h.prim = -1;
    h.meta = 0;
    h.t = tMax;
    h.u = h.v = 0.0f;
    float tm = tMax;
    if (WIDE)
        walkClosestWide<COUNT, 0, 1>(S, I.rootWide, lo, ld, linv, 0x1Fu, tMin, tm, h, nodeVisits, triTests, nullptr, 0.0f);
    else
        walkClosest<COUNT, 1>(S, I.rootBinary, lo, ld, linv, 0x1Fu, tMin, tm, h, nodeVisits, triTests, 0.0f);
    if (h.prim < 0) return;
    tMax = tm;
    best.t = h.t;
    best.u = h.u;
    best.v = h.v;
    best.prim = instanceHitCode(inst, h.prim - I.recBase);
    best.meta = meta;
}

template <bool COUNT, bool WIDE>
__device__ __noinline__ bool instanceAny(const SceneGPU& S, int inst, V3 o, V3 d, float tMin, float tMax,
                                         uint32_t& nodeVisits, uint32_t& triTests, float time) {
    const InstGPU& I = S.instances[inst];
    float4 buf[8];
    const float4 *l2w, *w2l;
    float uvScale;
    instancePose(S, I, time, buf, l2w, w2l, uvScale);
    const V3 lo = xfPointD(w2l, o), ld = xfVectorD(w2l, d);
    const V3 linv = mk(1.0f / ld.x, 1.0f / ld.y, 1.0f / ld.z);
    return WIDE ? walkAnyWide<COUNT, 1>(S, I.rootWide, lo, ld, linv, 0x1Fu, tMin, tMax, nodeVisits, triTests, 0.0f)
                : walkAny<COUNT, 1>(S, I.rootBinary, lo, ld, linv, 0x1Fu, tMin, tMax, nodeVisits, triTests, 0.0f);
}

// The primitives of one leaf, in order: triangles (lean Möller–Trumbore), spheres and, at the top
// level, mesh instances; the last one with t <= tMax wins a tie, as in BVH::intersect.
template <bool COUNT, int LEVEL, bool WIDE>
__device__ __forceinline__ void testLeafClosest(const SceneGPU& S, int first, int count, V3 o, V3 d, uint32_t mask,
                                                float tMin, float& tMax, Hit& best, uint32_t& nodeVisits,
                                                uint32_t& triTests, float time) {
    for (int k = 0; k < count; ++k) {
        const int pi = first + k;
        const float4 a = __ldg(&S.tris[3 * pi + 0]);
        const float4 b = __ldg(&S.tris[3 * pi + 1]);
        const uint32_t meta = __float_as_uint(b.w);
        if ((meta & mask) == 0u) continue;
        if (LEVEL == 0 && (meta & PRIM_INSTANCE)) {
            instanceClosest<COUNT, WIDE>(S, __float_as_int(a.x), meta, o, d, tMin, tMax, best, nodeVisits, triTests, time);
            continue;
        }
        if (COUNT) ++triTests;
        float t, u = 0.0f, v = 0.0f;
        if (meta & PRIM_SPHERE) {
            if (!sphereLean(a, o, d, tMin, tMax, t)) continue;
        } else if (!triLean(a, b, __ldg(&S.tris[3 * pi + 2]), o, d, tMin, tMax, t, u, v)) {
            continue;
        }
        tMax = t;
        best.t = t;
        best.u = u;
        best.v = v;
        best.prim = pi;
        best.meta = meta;
    }
}

template <bool COUNT, int LEVEL, bool WIDE>
__device__ __forceinline__ bool testLeafAny(const SceneGPU& S, int first, int count, V3 o, V3 d, uint32_t mask,
                                            float tMin, float tMax, uint32_t& nodeVisits, uint32_t& triTests,
                                            float time) {
    for (int k = 0; k < count; ++k) {
        const int pi = first + k;
        const float4 a = __ldg(&S.tris[3 * pi + 0]);
        const float4 b = __ldg(&S.tris[3 * pi + 1]);
        const uint32_t meta = __float_as_uint(b.w);
        if ((meta & mask) == 0u) continue;
        if (LEVEL == 0 && (meta & PRIM_INSTANCE)) {
            if (instanceAny<COUNT, WIDE>(S, __float_as_int(a.x), o, d, tMin, tMax, nodeVisits, triTests, time)) return true;
            continue;
        }
        if (COUNT) ++triTests;
        float t, u, v;
        if (meta & PRIM_SPHERE) {
            if (sphereLean(a, o, d, tMin, tMax, t)) return true;
        } else if (triLean(a, b, __ldg(&S.tris[3 * pi + 2]), o, d, tMin, tMax, t, u, v)) {
            return true;
        }
    }
    return false;
}

// The root of the top-level tree as a walk's first reference: node 0, or the leaf it is.
__device__ __forceinline__ int rootRef(const SceneGPU& S) {
    return S.rootIsLeaf ? static_cast<int>(~((static_cast<uint32_t>(S.rootFirst) << 8) | static_cast<uint32_t>(S.rootCount - 1)))
                        : 0;
}

// BVH::intersect (bvh.cpp:322-401) from reference `cur`: near child first, far child pushed with
// its entry distance and skipped on pop when farther than the current hit.
template <bool COUNT, int LEVEL>
__device__ void walkClosest(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float& tMax,
                            Hit& best, uint32_t& nodeVisits, uint32_t& triTests, float time) {
    int stackRef[kMaxStack];
    float stackT[kMaxStack];
    int sp = 0;
    // while-while form: descend through interior nodes until a leaf (or nothing) is next, test the
    // leaf, pop.  A ray's own sequence of node and triangle tests is the reference's; the loop
    // shape only lets the lanes of a warp spend more of their steps in the same branch.
    for (;;) {
        while (cur >= 0) {
            if (COUNT) ++nodeVisits;
            const float4 n0 = __ldg(&S.nodes[4 * cur + 0]);
            const float4 n1 = __ldg(&S.nodes[4 * cur + 1]);
            const float4 n2 = __ldg(&S.nodes[4 * cur + 2]);
            const float4 n3 = __ldg(&S.nodes[4 * cur + 3]);
            float t0, t1;
            const bool h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tMin, tMax, t0);
            const bool h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tMin, tMax, t1);
            const int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                const bool farFirst = t1 < t0;
                stackRef[sp] = farFirst ? c0 : c1;
                stackT[sp] = farFirst ? t0 : t1;
                ++sp;
                cur = farFirst ? c1 : c0;
            } else if (h0) {
                cur = c0;
            } else if (h1) {
                cur = c1;
            } else {
                // pop: entries farther than the current hit are skipped
                bool found = false;
                while (sp > 0) {
                    --sp;
                    if (stackT[sp] <= tMax) {
                        cur = stackRef[sp];
                        found = true;
                        break;
                    }
                }
                if (!found) return;
            }
        }
        int first, count;
        leafRange(cur, first, count);
        testLeafClosest<COUNT, LEVEL, false>(S, first, count, o, d, mask, tMin, tMax, best, nodeVisits, triTests, time);
        bool found = false;
        while (sp > 0) {
            --sp;
            if (stackT[sp] <= tMax) {
                cur = stackRef[sp];
                found = true;
                break;
            }
        }
        if (!found) return;
    }
}

// Closest hit over the binary tree in the reference's visiting order; the last triangle with
// t <= tMax wins ties, as in BVH::intersect.
template <bool COUNT>
__device__ Hit traceClosest(const SceneGPU& S, V3 o, V3 d, uint32_t mask, float tMin, float tMax, uint32_t& nodeVisits,
                            uint32_t& triTests, float time = 0.0f) {
    Hit best;
    best.prim = -1;
    best.meta = 0;
    best.t = tMax;
    best.u = best.v = 0.0f;
    const V3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float tn;
    if (S.nTris == 0) return best;
    if (!slab(S.rootMin[0], S.rootMax[0], S.rootMin[1], S.rootMax[1], S.rootMin[2], S.rootMax[2], o, inv, tMin, tMax, tn))
        return best;
    walkClosest<COUNT, 0>(S, rootRef(S), o, d, inv, mask, tMin, tMax, best, nodeVisits, triTests, time);
    return best;
}

// BVH::intersectAny (bvh.cpp:404-446) from reference `cur`.
template <bool COUNT, int LEVEL>
__device__ bool walkAny(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float tMax,
                        uint32_t& nodeVisits, uint32_t& triTests, float time) {
    int stackRef[kMaxStack];
    int sp = 0;
    for (;;) {
        while (cur >= 0) {
            if (COUNT) ++nodeVisits;
            const float4 n0 = __ldg(&S.nodes[4 * cur + 0]);
            const float4 n1 = __ldg(&S.nodes[4 * cur + 1]);
            const float4 n2 = __ldg(&S.nodes[4 * cur + 2]);
            const float4 n3 = __ldg(&S.nodes[4 * cur + 3]);
            float t0, t1;
            const bool h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tMin, tMax, t0);
            const bool h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tMin, tMax, t1);
            const int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                const bool farFirst = t1 < t0;
                stackRef[sp++] = farFirst ? c0 : c1;
                cur = farFirst ? c1 : c0;
            } else if (h0) {
                cur = c0;
            } else if (h1) {
                cur = c1;
            } else {
                if (sp == 0) return false;
                cur = stackRef[--sp];
            }
        }
        int first, count;
        leafRange(cur, first, count);
        if (testLeafAny<COUNT, LEVEL, false>(S, first, count, o, d, mask, tMin, tMax, nodeVisits, triTests, time)) return true;
        if (sp == 0) return false;
        cur = stackRef[--sp];
    }
}

// BVH::intersectAny (bvh.cpp:404-446): true when any primitive in [tMin, tMax] passes the mask.
// The answer does not depend on visiting order; near child first for early exit.
template <bool COUNT>
__device__ bool traceAny(const SceneGPU& S, V3 o, V3 d, uint32_t mask, float tMin, float tMax, uint32_t& nodeVisits,
                         uint32_t& triTests, float time = 0.0f) {
    const V3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float tn;
    if (S.nTris == 0) return false;
    if (!slab(S.rootMin[0], S.rootMax[0], S.rootMin[1], S.rootMax[1], S.rootMin[2], S.rootMax[2], o, inv, tMin, tMax, tn))
        return false;
    return walkAny<COUNT, 0>(S, rootRef(S), o, d, inv, mask, tMin, tMax, nodeVisits, triTests, time);
}

// ---- 4-wide traversal ----------------------------------------------------------------------
// The kernels traverse the 4-wide collapse of the binary tree (pe_host.cpp collapseWide): one
// 128-byte node per step tests four child boxes with the same slab arithmetic, so a ray makes
// about half the dependent node fetches of the binary walk.  Closest hit: children hit are
// visited nearest entry first (ties by child order), the others pushed with their entry
// distance and skipped on pop when farther than the current hit, as in the binary walk.  Every
// triangle that can hold the closest hit is tested with the same arithmetic, so the hit
// distance is the binary walk's; only when two triangles give the bit-identical distance (a ray
// through a shared edge or vertex) may the other of them win, because the last one tested wins.
constexpr float kInf = std::numeric_limits<float>::infinity();

struct WideNode {
    float4 lx, hx, ly, hy, lz, hz;
    int4 child;
    int count;
};
__device__ __forceinline__ WideNode loadWide(const float4* w, int i) {
    WideNode n;
    const float4* p = w + 8 * static_cast<size_t>(i);
    n.lx = __ldg(p + 0);
    n.hx = __ldg(p + 1);
    n.ly = __ldg(p + 2);
    n.hy = __ldg(p + 3);
    n.lz = __ldg(p + 4);
    n.hz = __ldg(p + 5);
    const float4 c = __ldg(p + 6);
    n.child = make_int4(__float_as_int(c.x), __float_as_int(c.y), __float_as_int(c.z), __float_as_int(c.w));
    n.count = __float_as_int(__ldg(reinterpret_cast<const float*>(p + 7)));
    return n;
}
// Entry distances of the four children (+inf where a child is absent or missed).
__device__ __forceinline__ void wideSlabs(const WideNode& n, V3 o, V3 inv, float tMin, float tMax, float t[4]) {
    float tn;
    t[0] = slab(n.lx.x, n.hx.x, n.ly.x, n.hy.x, n.lz.x, n.hz.x, o, inv, tMin, tMax, tn) ? tn : kInf;
    t[1] = slab(n.lx.y, n.hx.y, n.ly.y, n.hy.y, n.lz.y, n.hz.y, o, inv, tMin, tMax, tn) ? tn : kInf;
    t[2] = n.count > 2 && slab(n.lx.z, n.hx.z, n.ly.z, n.hy.z, n.lz.z, n.hz.z, o, inv, tMin, tMax, tn) ? tn : kInf;
    t[3] = n.count > 3 && slab(n.lx.w, n.hx.w, n.ly.w, n.hy.w, n.lz.w, n.hz.w, o, inv, tMin, tMax, tn) ? tn : kInf;
}
// Compare-exchange on (distance, child order): a total order, so equal distances keep child order.
__device__ __forceinline__ void cmpx(float& ta, int& ra, int& ka, float& tb, int& rb, int& kb) {
    if (ta > tb || (ta == tb && ka > kb)) {
        const float t = ta; ta = tb; tb = t;
        const int r = ra; ra = rb; rb = r;
        const int k = ka; ka = kb; kb = k;
    }
}

// A traversal stack whose top K entries live in registers (shifted on every push and pop, so
// every index is static) and the rest in the thread's local memory: a walk pushes and pops mostly
// within a few entries of the top, so most of its stack traffic never reaches memory.
template <typename T, int K, int N>
struct WindowStack {
    T top[K];
    T rest[N - K];
    int n = 0;
    __device__ __forceinline__ void push(T e) {
        if (n >= K) rest[n - K] = top[K - 1];
#pragma unroll
        for (int i = K - 1; i > 0; --i) top[i] = top[i - 1];
        top[0] = e;
        ++n;
    }
    __device__ __forceinline__ T pop() {
        const T e = top[0];
#pragma unroll
        for (int i = 0; i < K - 1; ++i) top[i] = top[i + 1];
        --n;
        if (n >= K) top[K - 1] = rest[n - K];
        return e;
    }
    __device__ __forceinline__ bool empty() const { return n == 0; }
};

// The closest-hit walk's stack of (reference, entry distance) pairs.  SD > 0: its first SD entries
// in shared memory (`shared` points at the thread's column of a [SD][128] block array, stride 128),
// the rest in local memory; SD == 0: all in local memory; SD < 0: the top −SD entries in registers.
template <int SD, bool WINDOW = (SD < 0)>
struct TraceStack;
template <int SD>
struct TraceStack<SD, false> {
    uint2* shared;
    uint2 local[kWideStack - SD];
    int sp = 0;
    __device__ __forceinline__ void push(uint2 e) {
        if (SD > 0 && sp < SD) shared[sp * 128] = e;
        else local[sp - SD] = e;
        ++sp;
    }
    __device__ __forceinline__ uint2 pop() {
        --sp;
        return (SD > 0 && sp < SD) ? shared[sp * 128] : local[sp - SD];
    }
    __device__ __forceinline__ bool empty() const { return sp == 0; }
};
template <int SD>
struct TraceStack<SD, true> : WindowStack<uint2, -SD, kWideStack> {
    uint2* shared;
};

// The 4-wide walk from reference `cur`.  SD: stack entries kept in shared memory (`sstack`:
// this thread's column); 0 keeps all in local memory.
template <bool COUNT, int SD, int LEVEL>
__device__ void walkClosestWide(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float& tMax,
                                Hit& best, uint32_t& nodeVisits, uint32_t& triTests, uint2* sstack, float time) {
    TraceStack<SD> stack;
    stack.shared = sstack;
    for (;;) {
        while (cur >= 0) {
            if (COUNT) ++nodeVisits;
            const WideNode n = loadWide(S.wide, cur);
            float t[4];
            wideSlabs(n, o, inv, tMin, tMax, t);
            float t0 = t[0], t1 = t[1], t2 = t[2], t3 = t[3];
            int r0 = n.child.x, r1 = n.child.y, r2 = n.child.z, r3 = n.child.w;
            int k0 = 0, k1 = 1, k2 = 2, k3 = 3;
            cmpx(t0, r0, k0, t1, r1, k1);
            cmpx(t2, r2, k2, t3, r3, k3);
            cmpx(t0, r0, k0, t2, r2, k2);
            cmpx(t1, r1, k1, t3, r3, k3);
            cmpx(t1, r1, k1, t2, r2, k2);
            if (t0 == kInf) {
                bool found = false;
                while (!stack.empty()) {
                    const uint2 e = stack.pop();
                    if (__uint_as_float(e.y) <= tMax) {
                        cur = static_cast<int>(e.x);
                        found = true;
                        break;
                    }
                }
                if (!found) return;
                continue;
            }
            // farther children first onto the stack, so they pop nearest first
            if (t3 != kInf) stack.push(make_uint2(static_cast<uint32_t>(r3), __float_as_uint(t3)));
            if (t2 != kInf) stack.push(make_uint2(static_cast<uint32_t>(r2), __float_as_uint(t2)));
            if (t1 != kInf) stack.push(make_uint2(static_cast<uint32_t>(r1), __float_as_uint(t1)));
            cur = r0;
        }
        int first, count;
        leafRange(cur, first, count);
        testLeafClosest<COUNT, LEVEL, true>(S, first, count, o, d, mask, tMin, tMax, best, nodeVisits, triTests, time);
        bool found = false;
        while (!stack.empty()) {
            const uint2 e = stack.pop();
            if (__uint_as_float(e.y) <= tMax) {
                cur = static_cast<int>(e.x);
                found = true;
                break;
            }
        }
        if (!found) return;
    }
}

// The 4-wide walk with postponed leaves (speculative traversal after Aila and Laine, "Understanding
// the Efficiency of Ray Traversal on GPUs", 2009): a lane that reaches a leaf keeps it aside and
// goes on descending until every active lane of its warp holds one, then the warp tests its
// leaves together, so leaf tests and node steps stop interleaving across the lanes.  Leaves are
// tested in another order than the depth-first walk's and tMax shrinks later, so a few more nodes
// are visited; every leaf that can hold a closer hit is still tested, so the distance is the same.
template <bool COUNT, int SD, int LEVEL>
__device__ void walkClosestWideSpec(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin,
                                    float& tMax, Hit& best, uint32_t& nodeVisits, uint32_t& triTests, uint2* sstack,
                                    float time) {
    TraceStack<SD> stack;
    stack.shared = sstack;
    auto popNext = [&]() {
        while (!stack.empty()) {
            const uint2 e = stack.pop();
            if (__uint_as_float(e.y) <= tMax) {
                cur = static_cast<int>(e.x);
                return true;
            }
        }
        return false;
    };
    bool alive = true;       // `cur` holds a reference still to visit
    bool hasLeaf = false;    // a leaf is kept aside for the next test
    int leafRef = 0;
    while (alive || hasLeaf) {
        while (alive && (cur >= 0 || !hasLeaf)) {
            if (cur < 0) {
                // a leaf and none kept aside: keep it, take the next reference
                leafRef = cur;
                hasLeaf = true;
                alive = popNext();
            } else {
                if (COUNT) ++nodeVisits;
                const WideNode n = loadWide(S.wide, cur);
                float t[4];
                wideSlabs(n, o, inv, tMin, tMax, t);
                float t0 = t[0], t1 = t[1], t2 = t[2], t3 = t[3];
                int r0 = n.child.x, r1 = n.child.y, r2 = n.child.z, r3 = n.child.w;
                int k0 = 0, k1 = 1, k2 = 2, k3 = 3;
                cmpx(t0, r0, k0, t1, r1, k1);
                cmpx(t2, r2, k2, t3, r3, k3);
                cmpx(t0, r0, k0, t2, r2, k2);
                cmpx(t1, r1, k1, t3, r3, k3);
                cmpx(t1, r1, k1, t2, r2, k2);
                if (t0 == kInf) {
                    alive = popNext();
                } else {
                    if (t3 != kInf) stack.push(make_uint2(static_cast<uint32_t>(r3), __float_as_uint(t3)));
                    if (t2 != kInf) stack.push(make_uint2(static_cast<uint32_t>(r2), __float_as_uint(t2)));
                    if (t1 != kInf) stack.push(make_uint2(static_cast<uint32_t>(r1), __float_as_uint(t1)));
                    cur = r0;
                }
            }
            // every lane still walking holds a leaf: test them together
            if (!__any_sync(__activemask(), !hasLeaf)) break;
        }
        if (hasLeaf) {
            int first, count;
            leafRange(leafRef, first, count);
            testLeafClosest<COUNT, LEVEL, true>(S, first, count, o, d, mask, tMin, tMax, best, nodeVisits, triTests, time);
            hasLeaf = false;
            // the reference in hand may have become too far while the leaf was aside; it is an
            // interior node or a leaf, tested against tMax when it is visited or kept
        }
    }
}

template <bool COUNT, int SD = 0, bool SPEC = false>
__device__ Hit traceClosestWide(const SceneGPU& S, V3 o, V3 d, uint32_t mask, float tMin, float tMax,
                                uint32_t& nodeVisits, uint32_t& triTests, uint2* sstack = nullptr, float time = 0.0f) {
    Hit best;
    best.prim = -1;
    best.meta = 0;
    best.t = tMax;
    best.u = best.v = 0.0f;
    const V3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float tn;
    if (S.nTris == 0) return best;
    if (!slab(S.rootMin[0], S.rootMax[0], S.rootMin[1], S.rootMax[1], S.rootMin[2], S.rootMax[2], o, inv, tMin, tMax, tn))
        return best;
    if (SPEC)
        walkClosestWideSpec<COUNT, SD, 0>(S, rootRef(S), o, d, inv, mask, tMin, tMax, best, nodeVisits, triTests, sstack,
                                          time);
    else
        walkClosestWide<COUNT, SD, 0>(S, rootRef(S), o, d, inv, mask, tMin, tMax, best, nodeVisits, triTests, sstack, time);
    return best;
}

// Any hit over the 4-wide tree from reference `cur`: the answer does not depend on the order.
// AW > 0: the top AW stack entries in registers (WindowStack), else all in local memory.
template <bool COUNT, int LEVEL, int AW>
__device__ bool walkAnyWide(const SceneGPU& S, int cur, V3 o, V3 d, V3 inv, uint32_t mask, float tMin, float tMax,
                            uint32_t& nodeVisits, uint32_t& triTests, float time) {
    if constexpr (AW > 0) {
        WindowStack<int, AW, kWideStack> stack;
        for (;;) {
            while (cur >= 0) {
                if (COUNT) ++nodeVisits;
                const WideNode n = loadWide(S.wide, cur);
                float t[4];
                wideSlabs(n, o, inv, tMin, tMax, t);
                int next = 0;
                bool have = false;
                if (t[0] != kInf) { next = n.child.x; have = true; }
                if (t[1] != kInf) { if (!have) { next = n.child.y; have = true; } else stack.push(n.child.y); }
                if (t[2] != kInf) { if (!have) { next = n.child.z; have = true; } else stack.push(n.child.z); }
                if (t[3] != kInf) { if (!have) { next = n.child.w; have = true; } else stack.push(n.child.w); }
                if (!have) {
                    if (stack.empty()) return false;
                    cur = stack.pop();
                } else {
                    cur = next;
                }
            }
            int first, count;
            leafRange(cur, first, count);
            if (testLeafAny<COUNT, LEVEL, true>(S, first, count, o, d, mask, tMin, tMax, nodeVisits, triTests, time))
                return true;
            if (stack.empty()) return false;
            cur = stack.pop();
        }
    }
    int stackRef[kWideStack];
    int sp = 0;
    for (;;) {
        while (cur >= 0) {
            if (COUNT) ++nodeVisits;
            const WideNode n = loadWide(S.wide, cur);
            float t[4];
            wideSlabs(n, o, inv, tMin, tMax, t);
            // the first child hit is next, the other hits wait on the stack (a flag, not a
            // sentinel reference: the leaf of primitive 0 alone is encoded as ~0 = -1)
            int next = 0;
            bool have = false;
            if (t[0] != kInf) { next = n.child.x; have = true; }
            if (t[1] != kInf) { if (!have) { next = n.child.y; have = true; } else stackRef[sp++] = n.child.y; }
            if (t[2] != kInf) { if (!have) { next = n.child.z; have = true; } else stackRef[sp++] = n.child.z; }
            if (t[3] != kInf) { if (!have) { next = n.child.w; have = true; } else stackRef[sp++] = n.child.w; }
            if (!have) {
                if (sp == 0) return false;
                cur = stackRef[--sp];
            } else {
                cur = next;
            }
        }
        int first, count;
        leafRange(cur, first, count);
        if (testLeafAny<COUNT, LEVEL, true>(S, first, count, o, d, mask, tMin, tMax, nodeVisits, triTests, time)) return true;
        if (sp == 0) return false;
        cur = stackRef[--sp];
    }
}

template <bool COUNT, int AW = 0>
__device__ bool traceAnyWide(const SceneGPU& S, V3 o, V3 d, uint32_t mask, float tMin, float tMax, uint32_t& nodeVisits,
                             uint32_t& triTests, float time = 0.0f) {
    const V3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float tn;
    if (S.nTris == 0) return false;
    if (!slab(S.rootMin[0], S.rootMax[0], S.rootMin[1], S.rootMax[1], S.rootMin[2], S.rootMax[2], o, inv, tMin, tMax, tn))
        return false;
    return walkAnyWide<COUNT, 0, AW>(S, rootRef(S), o, d, inv, mask, tMin, tMax, nodeVisits, triTests, time);
}

// Shutter time of the path in `slot` (Ray::time): read only where the scene has moving instances.
__device__ __forceinline__ float pathTime(const SceneGPU& S, const Paths& P, int slot) {
    return (S.motions && P.time) ? P.time[slot] : 0.0f;
}

// ---- hit record (src/geometry/triangle.cpp:54-133) -----------------------------------------
struct Isect {
    V3 point, normal, ng, tangent, pError, pSmooth;
    float t;
    bool frontFace, hasSmooth;
    int32_t tri;    // global triangle index
    int32_t shape;
    int32_t material;
    V2 uv;          // interpolated vertex uv (0 without uvs)
    float uvDensity; // sqrt(|uv area| / world area) (scenes with mipmapped textures only)
};

__device__ __forceinline__ V3 ld3(const float4* a, int i) {
    const float4 v = __ldg(&a[i]);
    return mk(v.x, v.y, v.z);
}

// Sphere::intersect's record (src/geometry/sphere.cpp:40-90): the point projected back onto the
// sphere, its error bound, the outward normal faced to the ray, spherical uv and the ∂P/∂φ tangent.
static __device__ __noinline__ void fillSphereHit(const SceneGPU& S, const Hit& h, V3 rayO, V3 rayDir, int g, int shape,
                                                  Isect& is) {
    const float4 a = __ldg(&S.tris[3 * h.prim + 0]);
    const V3 c = mk(a.x, a.y, a.z);
    const float r = a.w;
    is.t = h.t;
    V3 local = (rayO + rayDir * h.t) - c;
    const float len = length(local);
    if (len > 0.0f) local = local * (r / len);
    is.point = c + local;
    const float iso = gammaN(32) * smax(r + maxComp(vabs(c)), 1e-20f);
    is.pError = (vabs(local) + vabs(c)) * gammaN(16) + mk(iso);
    is.hasSmooth = false;
    is.pSmooth = is.point;
    const V3 outward = local / r;
    is.ng = outward;
    is.frontFace = dot(rayDir, outward) < 0.0f;
    is.normal = is.frontFace ? outward : -outward;
    if (len2(is.ng) == 0.0f) is.ng = outward;
    const float theta = acosf(sclamp(outward.y, -1.0f, 1.0f));
    float phi = atan2f(-outward.z, outward.x) + kPi;
    if (phi < 0.0f) phi += kTwoPi;
    is.uv.x = phi / kTwoPi;
    is.uv.y = theta / kPi;
    is.uvDensity = 1.0f;
    V3 tangent = mk(outward.z, 0.0f, -outward.x);
    if (len2(tangent) == 0.0f) {
        const float sign = copysignf(1.0f, outward.z);
        const float ac = -1.0f / (sign + outward.z);
        const float bc = outward.x * outward.y * ac;
        tangent = mk(1.0f + sign * outward.x * outward.x * ac, sign * bc, -sign * outward.x);
    }
    is.tangent = normalize(tangent);
    is.tri = g;
    is.shape = shape;
    is.material = S.shapes[shape].material;
}

// Triangle::fillHit's record of leaf record h.prim, in the space its vertices are in; returns the
// triangle's vertex indices and (w) shape, which a mesh instance's triangle does not have.
static __device__ __forceinline__ int4 fillTriangleHit(const SceneGPU& S, const Hit& h, V3 rayDir, Isect& is);

// transformHitToWorld (mesh_instance.cpp:57-100): point and smooth point by the local-to-world
// matrix, both normals by its inverse transpose and renormalised (the shading normal faced to
// the world ray), the tangent carried and made orthogonal again, a world error bound from the
// matrix's absolute rows plus a relative and an absolute slack, the texel density rescaled.
static __device__ __noinline__ void instanceToWorld(const float4* l2w, const float4* w2l, float uvScale, V3 rayDir,
                                                    Isect& is) {
    const V3 localOutNg = is.ng;
    const V3 localOutNs = is.frontFace ? is.normal : -is.normal;
    is.point = xfPointD(l2w, is.point);
    is.pSmooth = is.hasSmooth ? xfPointD(l2w, is.pSmooth) : is.point;
    const float4 i0 = w2l[0], i1 = w2l[1], i2 = w2l[2];
    auto xfNormal = [&](V3 n) {
        return mk(i0.x * n.x + i1.x * n.y + i2.x * n.z, i0.y * n.x + i1.y * n.y + i2.y * n.z,
                  i0.z * n.x + i1.z * n.y + i2.z * n.z);
    };
    V3 ngW = xfNormal(localOutNg);
    if (len2(ngW) > 0.0f) ngW = normalize(ngW);
    V3 nsW = xfNormal(localOutNs);
    if (len2(nsW) > 0.0f) nsW = normalize(nsW);
    else nsW = ngW;
    is.ng = ngW;
    is.frontFace = dot(rayDir, nsW) < 0.0f;
    is.normal = is.frontFace ? nsW : -nsW;
    if (len2(is.ng) == 0.0f) is.ng = nsW;
    V3 tW = xfVectorD(l2w, is.tangent);
    tW = tW - is.normal * dot(is.normal, tW);
    if (len2(tW) > 1e-12f) {
        is.tangent = normalize(tW);
    } else {
        const V3 n = is.normal;
        const float sign = copysignf(1.0f, n.z);
        const float a = -1.0f / (sign + n.z);
        const float b = n.x * n.y * a;
        is.tangent = normalize(mk(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x));
    }
    const float4 m0 = l2w[0], m1 = l2w[1], m2 = l2w[2];
    const V3 r0 = mk(fabsf(m0.x), fabsf(m0.y), fabsf(m0.z)), r1 = mk(fabsf(m1.x), fabsf(m1.y), fabsf(m1.z)),
             r2 = mk(fabsf(m2.x), fabsf(m2.y), fabsf(m2.z));
    const V3 pAbs = vabs(is.point);
    is.pError = mk(dot(r0, is.pError), dot(r1, is.pError), dot(r2, is.pError)) + pAbs * 1e-5f + mk(1e-6f);
    if (is.uvDensity > 0.0f) is.uvDensity = is.uvDensity / uvScale;
}

static __device__ __noinline__ void fillHit(const SceneGPU& S, const Hit& h, V3 rayO, V3 rayDir, Isect& is,
                                            float time = 0.0f) {
    if (isInstanceHit(h.prim)) {
        // MeshInstance::shadeInstanceHit (mesh_instance.cpp:125-133): the triangle's record in the
        // instance's space at the ray's time, carried to world space
        const InstGPU& I = S.instances[instanceOfHit(h.prim)];
        float4 buf[8];
        const float4 *l2w, *w2l;
        float uvScale;
        instancePose(S, I, time, buf, l2w, w2l, uvScale);
        Hit hl = h;
        hl.prim = I.recBase + localOfHit(h.prim);
        fillTriangleHit(S, hl, xfVectorD(w2l, rayDir), is);
        instanceToWorld(l2w, w2l, uvScale, rayDir, is);
        is.shape = I.shape;
        is.material = I.material;
        return;
    }
    const float4 e2w = __ldg(&S.tris[3 * h.prim + 2]);
    const int g = static_cast<int>(__float_as_uint(e2w.w));
    if (__float_as_uint(__ldg(&S.tris[3 * h.prim + 1]).w) & PRIM_SPHERE) {
        fillSphereHit(S, h, rayO, rayDir, g, __ldg(&S.triVerts[g]).w, is);
        return;
    }
    const int4 tv = fillTriangleHit(S, h, rayDir, is);
    is.shape = tv.w;
    is.material = S.shapes[tv.w].material;
}

static __device__ __forceinline__ int4 fillTriangleHit(const SceneGPU& S, const Hit& h, V3 rayDir, Isect& is) {
    const float4 e2w = __ldg(&S.tris[3 * h.prim + 2]);
    const int g = static_cast<int>(__float_as_uint(e2w.w));
    const int4 tv = __ldg(&S.triVerts[g]);
    const V3 v0 = ld3(S.pos, tv.x), v1 = ld3(S.pos, tv.y), v2 = ld3(S.pos, tv.z);
    const V3 n0 = ld3(S.nrm, tv.x), n1 = ld3(S.nrm, tv.y), n2 = ld3(S.nrm, tv.z);
    const float2 uv0 = __ldg(&S.uv[tv.x]), uv1 = __ldg(&S.uv[tv.y]), uv2 = __ldg(&S.uv[tv.z]);
    const float u = h.u, v = h.v;
    const V3 edge1 = v1 - v0, edge2 = v2 - v0;
    is.t = h.t;
    const float w = 1.0f - u - v;
    const V3 a0 = v0 * w, a1 = v1 * u, a2 = v2 * v;
    is.point = a0 + a1 + a2;
    const float iso = gammaN(32) * smax(smax(smax(maxComp(vabs(v0)), maxComp(vabs(v1))), maxComp(vabs(v2))), 1e-20f);
    is.pError = (vabs(a0) + vabs(a1) + vabs(a2)) * gammaN(16) + mk(iso);
    const V3 geomNormal = normalize(cross(edge1, edge2));
    const bool hasN = len2(n0) > 0.0f && len2(n1) > 0.0f && len2(n2) > 0.0f;
    const V3 shading = hasN ? normalize(n0 * w + n1 * u + n2 * v) : geomNormal;
    is.ng = geomNormal;
    is.frontFace = dot(rayDir, shading) < 0.0f;
    is.normal = is.frontFace ? shading : -shading;
    if (len2(is.ng) == 0.0f) is.ng = shading;
    is.hasSmooth = false;
    is.pSmooth = is.point;
    if (hasN) {
        const V3 p = is.point;
        const V3 m0 = normalize(n0), m1 = normalize(n1), m2 = normalize(n2);
        const V3 lift = m0 * (w * smax(0.0f, dot(v0 - p, m0))) + m1 * (u * smax(0.0f, dot(v1 - p, m1))) +
                        m2 * (v * smax(0.0f, dot(v2 - p, m2)));
        if (len2(lift) > 0.0f) {
            is.pSmooth = p + lift;
            is.hasSmooth = true;
        }
    }
    is.uv.x = (uv0.x * w + uv1.x * u) + uv2.x * v;
    is.uv.y = (uv0.y * w + uv1.y * u) + uv2.y * v;
    const float d1x = uv1.x - uv0.x, d1y = uv1.y - uv0.y;
    const float d2x = uv2.x - uv0.x, d2y = uv2.y - uv0.y;
    const float r = d1x * d2y - d2x * d1y;
    is.uvDensity = 1.0f;
    if (S.hasMips) {
        // Triangle::fillHit's texel-density term (triangle.cpp:114-118)
        const float worldArea2 = length(cross(edge1, edge2));
        is.uvDensity = (worldArea2 > 1e-12f && fabsf(r) > 1e-12f) ? sqrtf(fabsf(r) / worldArea2) : 0.0f;
    }
    V3 tangent;
    if (fabsf(r) < 1e-6f) {
        const V3 n = is.normal;
        const float sign = copysignf(1.0f, n.z);
        const float ac = -1.0f / (sign + n.z);
        const float bc = n.x * n.y * ac;
        tangent = mk(1.0f + sign * n.x * n.x * ac, sign * bc, -sign * n.x);
    } else {
        const float invR = 1.0f / r;
        tangent = (edge1 * d2y - edge2 * d1y) * invR;
    }
    is.tangent = normalize(tangent);
    is.tri = g;
    return tv;
}

// ---- robust spawning (src/geometry/ray_spawn.h) --------------------------------------------
__device__ __forceinline__ V3 offsetRayOrigin(V3 p, V3 pError, V3 n, V3 w) {
    const float d = dot(vabs(n), pError);
    V3 off = n * d;
    if (dot(w, n) < 0.0f) off = -off;
    V3 po = p + off;
    po.x = off.x > 0.0f ? nextUp(po.x) : (off.x < 0.0f ? nextDown(po.x) : po.x);
    po.y = off.y > 0.0f ? nextUp(po.y) : (off.y < 0.0f ? nextDown(po.y) : po.y);
    po.z = off.z > 0.0f ? nextUp(po.z) : (off.z < 0.0f ? nextDown(po.z) : po.z);
    return po;
}
__device__ __forceinline__ V3 spawnNormal(const Isect& is) { return len2(is.ng) > 0.0f ? is.ng : is.normal; }
__device__ __forceinline__ V3 spawnOrigin(const Isect& is, V3 dir) {
    return offsetRayOrigin(is.point, is.pError, spawnNormal(is), dir);
}
__device__ __forceinline__ V3 shadowOrigin(const Isect& is, V3 toLight) {
    const V3 n = spawnNormal(is);
    V3 p = is.point;
    if (is.hasSmooth) {
        const V3 shadingOut = is.frontFace ? is.normal : -is.normal;
        const V3 ngOut = dot(n, shadingOut) >= 0.0f ? n : -n;
        const float NL = dot(shadingOut, toLight);
        if (NL > 0.0f) {
            const float kCutoff = 0.1f;
            const float NgL = dot(ngOut, toLight);
            const float amount = NL < kCutoff ? sclamp(2.0f - (NgL + NL) / kCutoff, 0.0f, 1.0f)
                                              : sclamp(1.0f - NgL / kCutoff, 0.0f, 1.0f);
            if (amount > 0.0f) p += (is.pSmooth - is.point) * amount;
        }
    }
    return offsetRayOrigin(p, is.pError, n, toLight);
}
// makeShadowRay (path_tracer.cpp:144-157) with spawnRayTo (ray_spawn.h:75-85).
__device__ __forceinline__ bool makeShadowRay(const Isect& is, V3 wi, float distance, V3& o, V3& d, float& tMax) {
    if (!(distance < kFltMax) || distance >= 1e29f) {
        o = shadowOrigin(is, wi);
        d = wi;
        tMax = 1e30f;
        return true;
    }
    const V3 target = is.point + wi * distance;
    const V3 toTarget = target - is.point;
    const float len = length(toTarget);
    if (!(len > 0.0f)) return false;
    const V3 origin = shadowOrigin(is, toTarget / len);
    const V3 dd = target - origin;
    const float dist = length(dd);
    const float slack = smax(dist * 1e-4f, 2e-6f * maxComp(vabs(target)));
    if (!(dist > slack)) return false;
    o = origin;
    d = dd / dist;
    tMax = dist - slack;
    return true;
}

} // namespace pe
