// pe_integrator.cuh — the wavefront form of PathTracer::Li (src/integrators/path_tracer.cpp:321-890).
//
// One path slot per (pixel, sample) of a wave.  A slot's state lives in HBM as SoA float4
// columns; each bounce runs three persistent kernels over compacted queues:
//   closest-hit  (queue of live rays)            → hit records
//   shade        (same queue) → next-ray queue + shadow queue (warp-aggregated appends)
//   any-hit      (shadow queue)                  → adds visible NEE terms to the slot's L
// The state machine below is Li's loop body split at its two scene queries.  Radiance terms are
// added to L in the reference's order (emission of vertex k, NEE of vertex k, emission of
// vertex k+1, ...), and each slot draws Sobol dimensions in the reference's order.
#pragma once

#include "pe_bsdf.h"
#include "pe_guide.cuh"
#include "pe_light.h"
#include "pe_medium.h"
#include "pe_trace.cuh"
#include "pe_wave.h"

namespace pe {

// Persistent-warp work distribution: lane 0 claims the next 32 items for its warp.
__device__ __forceinline__ int warpFetch(uint32_t* cursor) {
    int base = 0;
    if ((threadIdx.x & 31) == 0) base = static_cast<int>(atomicAdd(cursor, 32u));
    return __shfl_sync(0xffffffffu, base, 0);
}

__device__ __forceinline__ uint32_t packCounters(int depth, int diffuse, int pass, int skips) {
    return static_cast<uint32_t>(depth) | (static_cast<uint32_t>(diffuse) << 8) | (static_cast<uint32_t>(pass) << 16) |
           (static_cast<uint32_t>(skips) << 24);
}

// Warp-aggregated queue append: one atomicAdd per warp (ballot + popc).
__device__ __forceinline__ void queuePush(int32_t* queue, uint32_t* counter, bool want, int32_t value) {
    const unsigned mask = __ballot_sync(__activemask(), want);
    if (!want) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    const int rank = __popc(mask & ((1u << lane) - 1u));
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    queue[base + rank] = value;
}

// ---- generate: camera rays ------------------------------------------------------------------
// Wave path `path` (its segment, sample and pixel) starts in `slot`.
// ---- render passes (path_tracer.cpp:373-395) ---------------------------------------------------
__device__ __forceinline__ float4* passBlock(const Paths& P, int path) {
    return P.pass + static_cast<size_t>(path) * static_cast<size_t>(P.passStride);
}
__device__ __forceinline__ void passAdd(float4* q, V3 c) {
    float4 v = *q;
    v.x += c.x;
    v.y += c.y;
    v.z += c.z;
    *q = v;
}
// Shares of f's diffuse, glossy and transmission groups, per channel; 1, 0, 0 where the groups
// sum to zero (path_tracer.cpp:683-690, 803-811).
__device__ __forceinline__ void lobeShares(const LobeSplit3& sp, V3 out[3]) {
    const V3 sum = sp.diffuse + sp.glossy + sp.transmission;
    const V3* parts[3] = {&sp.diffuse, &sp.glossy, &sp.transmission};
    for (int k = 0; k < 3; ++k) {
        out[k].x = sum.x > 0.0f ? parts[k]->x / sum.x : (k == 0 ? 1.0f : 0.0f);
        out[k].y = sum.y > 0.0f ? parts[k]->y / sum.y : (k == 0 ? 1.0f : 0.0f);
        out[k].z = sum.z > 0.0f ? parts[k]->z / sum.z : (k == 0 ? 1.0f : 0.0f);
    }
}
// creditGroup: a term of light group `group` (ids outside the groups count for group 0).
__device__ __noinline__ void creditGroup(const SceneGPU& S, const Paths& P, int path, int group, V3 added) {
    if (S.nLightGroups <= 0 || isBlack(added)) return;
    const int g = (group >= 0 && group < S.nLightGroups) ? group : 0;
    if (g < PE_MAX_LIGHT_GROUPS) passAdd(passBlock(P, path) + PASS_GROUPS + g, added);
}
// creditPath: light reaching the path past its first surface, split by that surface's lobe
// shares into the direct (found by the first bounce) or indirect passes.
__device__ __noinline__ void creditPath(const Paths& P, int path, V3 added, bool direct) {
    float4* b = passBlock(P, path);
    for (int k = 0; k < 3; ++k) {
        const float4 share = b[PASS_LOBES + k];
        passAdd(b + 2 * k + (direct ? 0 : 1), added * mk(share.x, share.y, share.z));
    }
}
__device__ __forceinline__ int lightGroupOf(const SceneGPU& S, int light) {
    return light < 0 ? S.envGroup : (S.lightGroup ? S.lightGroup[light] : -1);
}
// A NEE term's passes: its light's group, and the direct passes by the vertex's own lobe shares
// at the first surface (shares non-null), else the first surface's shares as indirect light.
__device__ __noinline__ void creditNee(const SceneGPU& S, const Paths& P, int path, int light, V3 added,
                                       const float4* shares) {
    if (isBlack(added)) return;
    creditGroup(S, P, path, lightGroupOf(S, light), added);
    if (shares) {
        float4* b = passBlock(P, path);
        for (int k = 0; k < 3; ++k) passAdd(b + 2 * k, added * mk(shares[k].x, shares[k].y, shares[k].z));
    } else {
        creditPath(P, path, added, false);
    }
}

__device__ __forceinline__ void generatePath(const SceneGPU& S, const Paths& P, const Wave& W, int slot, int path) {
    const TablesGPU* T = S.tables;
    const WaveSeg& A = W.segs[segOfSlot(W, path)];
    const int local = path - A.slotFirst;
    const int sOff = local / A.nPix;
    const int pix = A.pixelFirst + (local - sOff * A.nPix);
    const int fp = A.pixList ? A.pixList[pix] : -1;
    const int x = fp >= 0 ? fp % A.width : A.tileX + pix % A.tileW;
    const int y = fp >= 0 ? fp / A.width : A.tileY + pix / A.tileW;
    Sobol sb;
    sb.pixelHash = pixelHashOf(A.seed, x, y);
    sb.revIndex = rev32(static_cast<uint32_t>(A.sampleFirst + sOff));
    sb.dim = 0;
    V3 o, d;
    float time;
    cameraRay(T, A.filterCdf, A.cam, A.filterWidth, x, y, A.width, A.height, sb, o, d, (A.flags & SEG_MOTION) != 0, &time);
    if (S.motions && P.time) P.time[slot] = time;
    P.rayO[slot] = make_float4(o.x, o.y, o.z, __uint_as_float(VIS_CAMERA));
    P.rayD[slot] = make_float4(d.x, d.y, d.z, 0.0f);
    P.thr[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.lastN[slot] = make_float4(0.0f, 1.0f, 0.0f, __uint_as_float(PF_SPECULAR_BOUNCE | PF_CAMERA_RAY | PF_FIRST_SEGMENT));
    P.lastP[slot] = make_float4(o.x, o.y, o.z, __uint_as_float(sb.dim));
    P.pickP[slot] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(sb.pixelHash));
    P.pickN[slot] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(packCounters(0, 0, 0, 0)));
    if (S.hasVolumes | S.hasSubsurface) P.med[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (P.guiding) {
        P.guideMark[slot] = 0u;
        if (slot % P.guideStride == 0) P.guideRec[static_cast<size_t>(slot) * 6 + 4] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (S.hasMips && P.cone) P.cone[slot] = make_float2(A.coneWidth, A.coneSpread);
    if (P.pass) {
        float4* b = passBlock(P, path);
        for (int k = 0; k < P.passStride; ++k) b[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        b[PASS_LOBES] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        b[PASS_HIT] = make_float4(o.x, o.y, o.z, 0.0f);
    }
    if (P.pathOf) P.pathOf[slot] = path;
}

// Hands an ended path's radiance to Lout (and counts it off its segment when those are tracked).
__device__ __forceinline__ void flushPath(const Paths& P, const Wave& W, int slot) {
    const int path = P.pathOf[slot];
    P.Lout[path] = P.L[slot];
    if (P.segLeft) {
        __threadfence(); // the radiance is visible before the segment's count says it is done
        atomicSub(&P.segLeft[segOfSlot(W, path)], 1u);
    }
}

// The wave's first `count` paths into slots [0, count), all queued.
__global__ void kGenerate(SceneGPU S, Paths P, Wave W, int count) {
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < count; slot += gridDim.x * blockDim.x) {
        generatePath(S, P, W, slot, slot);
        P.queueA[slot] = slot;
    }
}

// After a bounce of a regenerating wave: every slot freed this bounce hands its path's radiance
// to Lout (its NEE terms are in by now), and the first `fresh` of them take the wave's paths
// [nextPath, nextPath + fresh), appended to the next closest-hit queue after its `queued` entries.
__global__ void kRecycle(SceneGPU S, Paths P, Wave W, int freed, int fresh, int nextPath, int32_t* queue, int queued,
                         uint32_t* queueCount) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < freed; k += gridDim.x * blockDim.x) {
        const int slot = P.freeQ[k];
        flushPath(P, W, slot);
        if (k < fresh) {
            generatePath(S, P, W, slot, nextPath + k);
            queue[queued + k] = slot;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *queueCount = static_cast<uint32_t>(queued + fresh);
}

// The radiance of the paths the tail kernel finished, to Lout.
__global__ void kFlush(Paths P, Wave W, const int32_t* queue, const uint32_t* count) {
    const int n = static_cast<int>(*count);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flushPath(P, W, queue[i]);
}

// Continuous waves (the request server): freed slots form a stack (freeQ, its size in
// counters[CNT_FREE]).  kFlushFreed hands over the radiance of the `freed` slots pushed this
// bounce, above `base`; kInject then pops `fresh` slots for the wave's paths [nextPath, +fresh),
// appended to the next closest-hit queue after its `queued` entries.
__global__ void kFlushFreed(Paths P, Wave W, int base, int freed) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < freed; k += gridDim.x * blockDim.x)
        flushPath(P, W, P.freeQ[base + k]);
}

__global__ void kInject(SceneGPU S, Paths P, Wave W, int top, int fresh, int nextPath, int32_t* queue, int queued,
                        uint32_t* queueCount) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < fresh; k += gridDim.x * blockDim.x) {
        const int slot = P.freeQ[top - fresh + k];
        generatePath(S, P, W, slot, nextPath + k);
        if (P.born) P.born[slot] = P.iter;
        queue[queued + k] = slot;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *queueCount = static_cast<uint32_t>(queued + fresh);
        P.counters[CNT_FREE] = static_cast<uint32_t>(top - fresh);
    }
}

// Slots of a finished sweep back onto the free stack, above `top`.
__global__ void kReturnSlots(Paths P, const int32_t* slots, int n, int top) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) P.freeQ[top + k] = slots[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) P.counters[CNT_FREE] = static_cast<uint32_t>(top + n);
}

// Every slot free: the stack holds slots [0, n).
__global__ void kInitFree(Paths P, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) P.freeQ[k] = k;
    if (blockIdx.x == 0 && threadIdx.x == 0) P.counters[CNT_FREE] = static_cast<uint32_t>(n);
}

// ---- closest hit over a queue -----------------------------------------------------------------
// Closest hit for every queued ray; each ray is then binned by its shading key (miss or the
// hit material's type) so the shading kernel runs warps of one material kind.
// Closest-hit traversal variants the tuner chooses among (pe_tuning::closest_traversal).
// Closest-hit traversals: the binary tree in the reference's order; the 4-wide tree with its stack
// in local memory, its first 8 / 16 entries in shared memory, or its top 4 / 8 entries in registers.
// TRACE_WIDE_OCC8: the 4-wide walk capped at 64 registers, eight 128-thread blocks per SM; with
// the first 8 / 16 stack entries in shared memory as well (TRACE_WIDE_SMEM8_OCC8 / _SMEM16_OCC8).
enum TraceMode { TRACE_BINARY = 0, TRACE_WIDE = 1, TRACE_WIDE_SMEM8 = 2, TRACE_WIDE_SMEM16 = 3, TRACE_WIDE_REG4 = 4,
                 TRACE_WIDE_REG8 = 5, TRACE_WIDE_OCC8 = 6, TRACE_WIDE_SMEM8_OCC8 = 7, TRACE_WIDE_SMEM16_OCC8 = 8,
                 TRACE_WIDE_SPEC_OCC8 = 9, TRACE_MODES = 10 };
// TRACE_WIDE_SPEC_OCC8: the 64-register walk with postponed leaves (walkClosestWideSpec).
constexpr bool traceSpeculative(int mode) { return mode == TRACE_WIDE_SPEC_OCC8; }
constexpr int traceMinBlocks(int mode) { return mode >= TRACE_WIDE_OCC8 ? 8 : 1; }
constexpr int traceStackShared(int mode) {
    return (mode == TRACE_WIDE_SMEM8 || mode == TRACE_WIDE_SMEM8_OCC8) ? 8
         : (mode == TRACE_WIDE_SMEM16 || mode == TRACE_WIDE_SMEM16_OCC8) ? 16
         : mode == TRACE_WIDE_REG4 ? -4
         : mode == TRACE_WIDE_REG8 ? -8 : 0;
}

template <bool COUNT, int MODE = TRACE_WIDE>
__global__ void __launch_bounds__(128, traceMinBlocks(MODE)) kIntersect(SceneGPU S, Paths P, const int32_t* queue,
                                                                        const uint32_t* count, unsigned long long* stats) {
    constexpr int SD = traceStackShared(MODE);
    __shared__ uint2 sstack[SD > 0 ? SD * 128 : 1];
    const int n = static_cast<int>(*count);
    uint32_t nodes = 0, tris = 0;
    const int lane = threadIdx.x & 31;
    for (;;) {
        const int base = warpFetch(&P.counters[CNT_WORK_ISECT]);
        if (base >= n) break;
        const int i = base + lane;
        int key = -1, slot = -1;
        if (i < n) {
            slot = queue[i];
            const float4 ro = P.rayO[slot];
            const float4 rd = P.rayD[slot];
            const V3 o = mk(ro.x, ro.y, ro.z), d = mk(rd.x, rd.y, rd.z);
            const uint32_t vmask = __float_as_uint(ro.w);
            const float time = pathTime(S, P, slot);
            const Hit h = MODE == TRACE_BINARY ? traceClosest<COUNT>(S, o, d, vmask, 0.0f, 1e30f, nodes, tris, time)
                                               : traceClosestWide<COUNT, SD, traceSpeculative(MODE)>(
                                                     S, o, d, vmask, 0.0f, 1e30f, nodes, tris,
                                                                             sstack + threadIdx.x, time);
            P.hit[slot] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
            key = (__float_as_uint(ro.w) & RAY_WALK) ? kShadeKeys - 1
                  : (isMiss(h.prim) ? 0 : 1 + static_cast<int>((h.meta >> 8) & 0xFFu));
        }
        // warp-aggregated append into the key's segment: one atomic per distinct key per warp
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0) {
            const int leader = __ffs(peers) - 1;
            const int rank = __popc(peers & ((1u << lane) - 1u));
            uint32_t at = 0;
            if (lane == leader) at = atomicAdd(&P.counters[CNT_KEYS + key], static_cast<uint32_t>(__popc(peers)));
            at = __shfl_sync(peers, at, leader);
            P.sortQ[static_cast<size_t>(key) * P.capacity + at + rank] = slot;
        }
    }
    if (COUNT) {
        atomicAdd(&stats[0], static_cast<unsigned long long>(nodes));
        atomicAdd(&stats[1], static_cast<unsigned long long>(tris));
    }
}

// Surface coverage of a hit for a ray that may pass through cutouts (DisneyMaterial::opacity,
// disney.cpp:505-509: the opacity times the opacity map's red channel, a level-0 lookup).
__device__ __noinline__ float mappedOpacity(const SceneGPU& S, const MatGPU& m, const Isect& is) {
    ShadePoint sp;
    sp.uv = is.uv;
    sp.p = is.point;
    sp.n = is.normal;
    sp.ng = is.ng;
    const V2 uv = textureCoord(m, sp);
    return m.opacity * sclamp(texBilinear(S.textures[m.texOpacity], uv.x, uv.y, 0).x, 0.0f, 1.0f);
}
__device__ __forceinline__ float surfaceOpacity(const SceneGPU& S, const MatGPU& m, const Isect& is) {
    if (m.type != PE_MAT_DISNEY) return 1.0f;
    return m.texOpacity >= 0 ? mappedOpacity(S, m, is) : m.opacity;
}

// passesCutout (path_tracer.cpp:161-167): true = the ray goes on through this hit.
__device__ __forceinline__ bool passesCutout(const SceneGPU& S, const MatGPU& m, const Isect& is, Sobol& sb) {
    const float alpha = surfaceOpacity(S, m, is);
    if (alpha >= 1.0f) return false;
    if (alpha <= 0.0f) return true;
    return get1D(sb) >= alpha;
}

// Material::shadowTransmittance: thin-walled glass passes (1 − R_thin)·tint, a cutout Disney
// surface 1 − opacity, every other surface nothing.
__device__ __forceinline__ V3 surfaceShadowTransmittance(const SceneGPU& S, const MatGPU& m, const Isect& is, V3 dir) {
    if (m.type == PE_MAT_DIELECTRIC) return glassShadowTransmittance(m, is.ng, is.normal, dir);
    if (m.type == PE_MAT_DISNEY) return mk(1.0f - surfaceOpacity(S, m, is));
    return mk(0.0f);
}

// Scene::hasShadowLinkFor: light `light` (explicit, else -1) lets some blockers through.
__device__ __forceinline__ bool shadowLinkFor(const SceneGPU& S, int light) {
    return S.hasShadowLinks && light >= 0 && S.links[light].shadowMode != 0;
}

// shadowTransmittance (path_tracer.cpp:172-202).  Without shadow-transmitting materials or a
// shadow link for the light it is the any-hit test; otherwise the shadow ray walks from surface
// to surface (at most 64), passing the blockers the light's shadow link leaves out and
// multiplying the transmittance of thin-walled glass and cutouts, and stops black at any other
// surface.
template <bool COUNT>
__device__ V3 shadowVisibility(const SceneGPU& S, V3 o, V3 d, float tMax, int light, uint32_t& nodes, uint32_t& tris,
                              float time) {
    const bool link = shadowLinkFor(S, light);
    if (!S.hasShadowTransmitters && !link)
        return traceAnyWide<COUNT>(S, o, d, VIS_SHADOW, 0.0f, tMax, nodes, tris, time) ? mk(0.0f) : mk(1.0f);
    V3 T = mk(1.0f);
    V3 origin = o;
    float remaining = tMax;
    for (int i = 0; i < 64; ++i) {
        const Hit h = traceClosestWide<COUNT>(S, origin, d, VIS_SHADOW, 0.0f, remaining, nodes, tris, nullptr, time);
        if (isMiss(h.prim)) return T;
        Isect is;
        fillHit(S, h, origin, d, is, time);
        if (link && !linkAllows(S.links[light].shadowMode, S.links[light].shadowMask, S.shapes[is.shape].linkNode)) {
            origin = offsetRayOrigin(is.point, is.pError, len2(is.ng) > 0.0f ? is.ng : is.normal, d);
            remaining -= h.t;
            if (remaining <= 0.0f) return T;
            continue;
        }
        const MatGPU& m = S.materials[is.material];
        if (!(m.flags & MF_TRANSMITS_SHADOWS)) return mk(0.0f);
        T *= surfaceShadowTransmittance(S, m, is, d);
        if (isBlack(T)) return T;
        origin = offsetRayOrigin(is.point, is.pError, len2(is.ng) > 0.0f ? is.ng : is.normal, d);
        remaining -= h.t;
        if (remaining <= 0.0f) return T;
    }
    return mk(0.0f);
}

// A NEE sample's term: throughput × f·Li·vis·(cos·w / (lightPdf·n)), clamped when indirect
// (path_tracer.cpp:683-690).
__device__ __forceinline__ V3 neeTerm(V3 fLi, V3 vis, float scalar, V3 thr, bool indirect, float clampIndirect) {
    const V3 neeLocal = (fLi * vis) * scalar;
    V3 c = thr * neeLocal;
    if (indirect && clampIndirect > 0.0f) {
        const float m = smax3(c.x, c.y, c.z);
        if (m > clampIndirect) c = c * (clampIndirect / m);
    }
    return c;
}

// ---- any hit over the shadow queue ------------------------------------------------------------
// ANY: the scene has neither shadow-transmitting surfaces nor shadow links, so visibility is
// the plain any-hit query (and the transmittance walk is compiled out).
// AW: the any-hit walk's top AW stack entries in registers (0: all in local memory).
// MINB: at least this many 128-thread blocks per SM (8: a 64-register cap).
template <bool COUNT, bool ANY = false, int AW = 0, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) kShadow(SceneGPU S, Paths P, const uint32_t* count,
                                                    unsigned long long* stats) {
    const int n = static_cast<int>(*count);
    uint32_t nodes = 0, tris = 0;
    for (;;) {
        const int base = warpFetch(&P.counters[CNT_WORK_SHADOW]);
        if (base >= n) break;
        const int i = base + (threadIdx.x & 31);
        if (i >= n) continue;
        const int slot = P.shadowQ[i];
        const float4 so = P.shO[i];
        const float4 sd = P.shD[i];
        const int light = static_cast<int>(__float_as_uint(P.shC[i].w) >> 1) - 1;
        const float time = pathTime(S, P, slot);
        const V3 vis = ANY ? (traceAnyWide<COUNT, AW>(S, mk(so.x, so.y, so.z), mk(sd.x, sd.y, sd.z), VIS_SHADOW, 0.0f, so.w,
                                                  nodes, tris, time) ? mk(0.0f) : mk(1.0f))
                           : shadowVisibility<COUNT>(S, mk(so.x, so.y, so.z), mk(sd.x, sd.y, sd.z), so.w, light, nodes, tris,
                                                     time);
        if (isBlack(vis)) continue;
        const float4 sc = P.shC[i];
        const float4 st = P.shT[i];
        const V3 c = neeTerm(mk(sc.x, sc.y, sc.z), vis, sd.w, mk(st.x, st.y, st.z), (__float_as_uint(sc.w) & 1u) != 0, st.w);
        if (!isFinite3(c)) continue;
        float4 L = P.L[slot];
        L.x += c.x;
        L.y += c.y;
        L.z += c.z;
        P.L[slot] = L;
        if (P.pass) {
            const float4* shares = P.shPass + 3 * static_cast<size_t>(i);
            creditNee(S, P, pathOfSlot(P, slot), light, c, shares[0].w != 0.0f ? shares : nullptr);
        }
    }
    if (COUNT) {
        atomicAdd(&stats[2], static_cast<unsigned long long>(nodes));
        atomicAdd(&stats[3], static_cast<unsigned long long>(tris));
    }
}

// accumulate(): adds a finite term and returns it; a non-finite one is skipped and counts as
// black (path_tracer.cpp:355-359).
__device__ __forceinline__ V3 addL(float4& L, V3 c) {
    if (!isFinite3(c)) return mk(0.0f);
    L.x += c.x;
    L.y += c.y;
    L.z += c.z;
    return c;
}

// russianRoulette (path_tracer.cpp:131-137): false ends the path.
__device__ __forceinline__ bool russianRoulette(V3& thr, Sobol& sb) {
    const float m = smax3(thr.x, thr.y, thr.z);
    if (m >= 1.0f) return true;
    if (!(m > 0.0f) || get1D(sb) >= m) return false;
    thr /= m;
    return true;
}

enum SegmentOutcome { SEG_SURFACE = 0, SEG_SCATTERED = 1, SEG_END = 2 };

// Absorption and scattering over the segment a path just travelled inside the medium of the
// innermost volume boundary it entered (path_tracer.cpp:456-479).  SEG_SCATTERED sets up the
// next ray (origin newO, direction newD).
__device__ __noinline__ int mediumSegment(const TablesGPU* T, const MatGPU& mm, V3 segStart, V3 dir, bool hit, V3 hitPoint,
                                          Sobol& sb, V3& thr, uint32_t& volCtr, V3& newO, V3& newD) {
    const float dirLen = length(dir);
    const float segment = hit ? length(hitPoint - segStart) : kFltMax;
    const V3 sA = m3f(mm.sigmaA), sS = m3f(mm.sigmaS);
    if (mm.flags & MF_MEDIUM_SCATTERS) {
        const float uc = get1D(sb);
        const float u = get1D(sb);
        float t = 0.0f;
        if (sampleFreeFlight(sA + sS, sS, segment, hit, thr, uc, u, thr, t)) {
            const uint32_t events = (volCtr & 0xFFFFu) + 1u;
            volCtr = (volCtr & 0xFFFF0000u) | events;
            if (events > static_cast<uint32_t>(kMaxMediumEvents) || !isFinite3(thr)) return SEG_END;
            const V3 d = dir / dirLen;
            newO = segStart + d * t;
            newD = sampleHG(d, mm.mediumG, get2D(T, sb));
            if (events > 8u && !russianRoulette(thr, sb)) return SEG_END;
            return SEG_SCATTERED;
        }
    } else if (hit) {
        thr *= expNeg(sA, segment);
    } else if (!isBlack(sA)) {
        return SEG_END; // open mesh: an infinitely long absorbing segment
    }
    if (isBlack(thr) || !isFinite3(thr)) return SEG_END;
    return SEG_SURFACE;
}

// ---- learned proposal in the shading step ------------------------------------------------------
// Vertices the proposal may serve: non-delta surfaces that are neither volume boundaries nor
// shadow transmitters (the reference's useGuiding condition, path_tracer.cpp:623-626).
__device__ __forceinline__ bool guidable(const MatGPU& m) {
    return (m.flags & (MF_DELTA | MF_VOLUME_BOUNDARY | MF_TRANSMITS_SHADOWS)) == 0;
}

__device__ __noinline__ void slotLobes(const Paths& P, int slot, Lobes& L) {
    float o[kNetUsedOut];
    for (int j = 0; j < kNetUsedOut / 4; ++j) {
        const float4 v = P.guideOut[static_cast<size_t>(slot) * 10 + j];
        o[4 * j + 0] = v.x;
        o[4 * j + 1] = v.y;
        o[4 * j + 2] = v.z;
        o[4 * j + 3] = v.w;
    }
    decodeLobes(o, L);
}

__device__ __noinline__ float guidePdf(const Paths& P, int slot, V3 w) {
    Lobes L;
    slotLobes(P, slot, L);
    return lobesPdf(L, w);
}

// Training record of a path's first guidable vertex; its radiance along wi is what the path adds
// from here on (kGuideCollect).  False when the path has one already.
__device__ __noinline__ bool guideRecord(const Paths& P, int slot, V3 p, V3 n, V3 wo, V3 wi, V3 thrBefore) {
    float4* rec = P.guideRec + static_cast<size_t>(slot) * 6;
    if (rec[4].w != 0.0f) return false;
    rec[0] = make_float4(p.x, p.y, p.z, 0.0f);
    rec[1] = make_float4(n.x, n.y, n.z, 0.0f);
    rec[2] = make_float4(wo.x, wo.y, wo.z, 0.0f);
    rec[3] = make_float4(wi.x, wi.y, wi.z, 0.0f);
    rec[4] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    rec[5] = make_float4(thrBefore.x, thrBefore.y, thrBefore.z, 0.0f);
    return true;
}

// One-sample MIS of the proposal and the BSDF, 50/50 (path_tracer.cpp:703-735 with the
// learned mixture in place of the SD-tree): the branch number picks the strategy, the
// proposal draws a lobe from the rest of it and a direction from one get2D.
__device__ __noinline__ bool guidedSample(const TablesGPU* T, const MatGPU& mat, V3 wo, const ShadePoint& sp, const Paths& P,
                                          int slot, Sobol& sb, BsdfSample& bs) {
    Lobes L;
    slotLobes(P, slot, L);
    const float uBranch = get1D(sb);
    if (uBranch < 0.5f) {
        const V3 gwi = lobesSample(L, uBranch * 2.0f, get2D(T, sb));
        const float gPdf = lobesPdf(L, gwi);
        if (!(gPdf > 0.0f)) return false;
        float bPdf = 0.0f;
        const V3 f = bsdfEvalPdf(T, mat, wo, gwi, sp, bPdf, nullptr);
        const float mixPdf = 0.5f * gPdf + 0.5f * bPdf;
        if (isBlack(f) || !(mixPdf > 0.0f)) return false;
        bs.wi = gwi;
        bs.f = f;
        bs.pdf = mixPdf;
        bs.delta = false;
        bs.passThrough = false;
        bs.subsurface = false;
        bs.weight = mk(0.0f);
        return true;
    }
    const float uc = get1D(sb);
    const V2 u2 = get2D(T, sb);
    if (!bsdfSample(T, mat, wo, sp, uc, u2, bs)) return false;
    if (bs.subsurface) bs.weight = bs.weight * 2.0f;
    else if (bs.delta || bs.passThrough) bs.pdf *= 0.5f;
    else if (bs.pdf > 0.0f) bs.pdf = 0.5f * bs.pdf + 0.5f * lobesPdf(L, bs.wi);
    return true;
}

// The same one-sample MIS with the SD-tree's sampling quadtree rooted at `root`
// (path_tracer.cpp:703-735): a direction from one get2D on the guide branch, the BSDF's
// get1D + get2D on the other.
__device__ __noinline__ bool sdGuidedSample(const TablesGPU* T, const MatGPU& mat, V3 wo, const ShadePoint& sp,
                                            const SdQuad* tree, int root, Sobol& sb, BsdfSample& bs) {
    const float uBranch = get1D(sb);
    if (uBranch < 0.5f) {
        float gPdf = 0.0f;
        const V3 gwi = sdTreeSample(tree, root, get2D(T, sb), gPdf);
        if (!(gPdf > 0.0f)) return false;
        float bPdf = 0.0f;
        const V3 f = bsdfEvalPdf(T, mat, wo, gwi, sp, bPdf, nullptr);
        const float mixPdf = 0.5f * gPdf + 0.5f * bPdf;
        if (isBlack(f) || !(mixPdf > 0.0f)) return false;
        bs.wi = gwi;
        bs.f = f;
        bs.pdf = mixPdf;
        bs.delta = false;
        bs.passThrough = false;
        bs.subsurface = false;
        bs.weight = mk(0.0f);
        return true;
    }
    const float uc = get1D(sb);
    const V2 u2 = get2D(T, sb);
    if (!bsdfSample(T, mat, wo, sp, uc, u2, bs)) return false;
    if (bs.subsurface) bs.weight = bs.weight * 2.0f;
    else if (bs.delta || bs.passThrough) bs.pdf *= 0.5f;
    else if (bs.pdf > 0.0f) bs.pdf = 0.5f * bs.pdf + 0.5f * sdTreePdf(tree, root, bs.wi);
    return true;
}

// ---- surface effects of Li that cast rays of their own ------------------------------------------
// Contact ambient occlusion (approxAo, path_tracer.cpp:27-45): `samples` cosine rays of at most
// 0.35 over the shading normal; the path's throughput is scaled by lerp(1, visibility, strength).
__device__ __noinline__ float approxAo(const SceneGPU& S, const Isect& is, Sobol& sb, float strength, int samples,
                                       float time) {
    if (strength <= 0.0f || samples <= 0) return 1.0f;
    const TablesGPU* T = S.tables;
    const Frame frame = frameFromNormal(is.normal);
    float occ = 0.0f;
    uint32_t n0 = 0, n1 = 0;
    for (int i = 0; i < samples; ++i) {
        const V3 local = sampleCosineHemisphere(get2D(T, sb));
        const V3 dir = normalize(toWorld(frame, local));
        if (traceAnyWide<false>(S, spawnOrigin(is, dir), dir, VIS_SHADOW, 0.0f, 0.35f, n0, n1, time)) occ += 1.0f;
    }
    const float visibility = 1.0f - (occ / static_cast<float>(samples));
    return lerpf(1.0f, visibility, strength);
}

// Rounded edges (roundedEdgeNormal, path_tracer.cpp:209-255): six points on a disk of `radius`
// around the hit, each probed along one of the frame's axes (normal ½, tangents ¼ each) from both
// sides with rays of 2·radius; the outward normals of hits on the same shape within 1.5·radius,
// weighted by their projection on the probe axis, average with a quarter of the own normal.
__device__ __noinline__ V3 roundedEdgeNormal(const SceneGPU& S, const Isect& is, float radius, Sobol& sb, float time) {
    const TablesGPU* T = S.tables;
    const V3 N = is.normal;
    const Frame f = frameFromNormal(N);
    V3 sum = N * 0.25f;
    uint32_t n0 = 0, n1 = 0;
    for (int i = 0; i < 6; ++i) {
        const float ua = get1D(sb);
        const V2 dd = sampleDiskConcentric(get2D(T, sb));
        const V2 d = mk2(dd.x * radius, dd.y * radius);
        V3 axis, s, t;
        if (ua < 0.5f) {
            axis = f.n; s = f.s; t = f.t;
        } else if (ua < 0.75f) {
            axis = f.s; s = f.t; t = f.n;
        } else {
            axis = f.t; s = f.n; t = f.s;
        }
        for (int k = 0; k < 2; ++k) {
            const float sign = k == 0 ? 1.0f : -1.0f;
            const V3 origin = is.point + s * d.x + t * d.y + axis * (sign * radius);
            const V3 rdir = axis * -sign;
            const Hit h = traceClosestWide<false>(S, origin, rdir, VIS_ALL, 0.0f, 2.0f * radius, n0, n1, nullptr, time);
            if (isMiss(h.prim)) continue;
            Isect hit;
            fillHit(S, h, origin, rdir, hit, time);
            if (hit.shape != is.shape) continue;
            if (len2(hit.point - is.point) > 2.25f * radius * radius) continue;
            const V3 outward = hit.frontFace ? hit.normal : -hit.normal;
            sum += outward * fabsf(dot(outward, axis));
        }
    }
    V3 n = normalize(sum);
    const V3 outwardN = is.frontFace ? N : -N;
    if (dot(n, outwardN) < 0.0f) n = -n;
    return is.frontFace ? n : -n;
}

// Shadow catcher (path_tracer.cpp:515-563): a camera ray that hits the catcher sees the
// background `bg` times the share `ratio` of the direct light, over 4 × shadowSamples NEE
// samples, that reaches the hit point.
__device__ __noinline__ V3 shadowCatcher(const SceneGPU& S, const Isect& is, V3 dir, int shadowSamples, Sobol& sb,
                                         float& ratioOut, float time) {
    const TablesGPU* T = S.tables;
    V3 bg = mk(0.0f);
    if (S.bgMode == PE_BG_COLOR) bg = m3f(S.bgColor);
    else if (S.bgMode == PE_BG_ENVIRONMENT && S.env.present) bg = envEval(S.env, dir);
    float visible = 0.0f, total = 0.0f;
    if (S.lightCount > 0) {
        LightCtx picker;
        lightPrepare(S, is.point, is.normal, picker);
        const int n = 4 * shadowSamples;
        uint32_t n0 = 0, n1 = 0;
        for (int k = 0; k < n; ++k) {
            float pmf = 0.0f;
            const int li = lightCtxSample(S, picker, get1D(sb), pmf);
            if (li < 0 || !(pmf > 0.0f)) {
                (void)get2D(T, sb);
                continue;
            }
            if (li < S.nLights && S.hasLightLinks &&
                !linkAllows(S.links[li].mode, S.links[li].mask, S.shapes[is.shape].linkNode)) {
                (void)get2D(T, sb);
                continue;
            }
            const V2 u = get2D(T, sb);
            const LightSample ls = li < S.nLights ? sampleLight(S.lights[li], is.point, u) : envSampleFull(S.env, S.envFull, u);
            const float cosT = dot(ls.wi, is.normal);
            if (!lsValid(ls) || cosT <= 0.0f) continue;
            const float c = luminance(ls.Li) * cosT / (pmf * ls.pdf);
            if (!(c > 0.0f) || !pe::finitef(c)) continue;
            total += c;
            V3 so, sd;
            float stMax;
            if (makeShadowRay(is, ls.wi, ls.distance, so, sd, stMax))
                visible += c * luminance(shadowVisibility<false>(S, so, sd, stMax, li < S.nLights ? li : -1, n0, n1, time));
        }
    }
    ratioOut = total > 0.0f ? sclamp(visible / total, 0.0f, 1.0f) : 1.0f;
    return bg;
}

// ---- shade: Li's loop body between two closest-hit queries ------------------------------------
// One path's step: reads the slot's state and hit record, adds the radiance found to L and
// writes back the state for its next closest-hit query.  A path is in one of three states at
// each query: an ordinary ray (medium segment, then the surface or the sky), a step of a random
// subsurface walk (PF_WALK), whose exit point is shaded at once as the walk's white-Lambert exit
// vertex, or a ray scattered inside a medium (an ordinary ray with specularBounce set).  NEE
// shadow rays go to the any-hit queue, or with INLINE_SHADOW are traced here and their terms
// added to L at once, in the same order.  Returns whether the path goes on.
//
// KEY selects a specialised instantiation: -1 the full shader; otherwise a lean one for waves
// whose scene has SceneGPU::leanShading and that neither guide nor record, with every feature
// those waves cannot reach compiled out (so the code fits in registers); KEY >= 0 also fixes the
// shading key (0 a miss, 1 + material type a surface hit), -2 leaves it to the hit.
template <bool INLINE_SHADOW, bool COUNT, bool OUT, int KEY = -1>
__device__ __forceinline__ bool shadeSlot(const SceneGPU& S, const Paths& P, const WaveSeg& A, int slot, int path,
                                          uint32_t& shNodes, uint32_t& shTris, uint32_t& shRays) {
    constexpr bool LEAN = KEY != -1;
    constexpr int MT = KEY >= 1 ? KEY - 1 : -1; // the material type a surface key fixes
    const TablesGPU* T = S.tables;
    const bool volumetric = !LEAN && (S.hasVolumes | S.hasSubsurface) != 0;
    bool cont = false;
    float4 ro = P.rayO[slot];
    float4 rd = P.rayD[slot];
    float4 th = P.thr[slot];
    float4 L = P.L[slot];
    float4 ln = P.lastN[slot];
    float4 lp = P.lastP[slot];
    float4 pp = P.pickP[slot];
    float4 pn = P.pickN[slot];
    const float4 hr = P.hit[slot];
    float4 md = volumetric ? P.med[slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    MediaStack media;
    media.lo = __float_as_uint(md.x);
    media.hi = __float_as_uint(md.y);
    media.n = __float_as_int(md.w);
    uint32_t volCtr = __float_as_uint(md.z);
    float lambda = th.w; // 0 = RGB path; > 0 = single-wavelength path after a dispersive hit
    uint32_t flags = __float_as_uint(ln.w);
    if (!LEAN && (flags & PF_GUIDE_SNAP)) {
        // radiance so far, the previous vertex's NEE included: the training record's baseline
        if (P.sdMode & SD_RECORD) {
            const uint32_t n = P.sdCount[slot];
            if (n > 0)
                P.sdRec[(static_cast<size_t>(slot) * kSdRecords + n - 1) * 4 + 3] = make_float4(L.x, L.y, L.z, 2.0f);
        } else {
            P.guideRec[static_cast<size_t>(slot) * 6 + 4] = make_float4(L.x, L.y, L.z, 2.0f);
        }
        flags &= ~PF_GUIDE_SNAP;
    }
    uint32_t ctr = __float_as_uint(pn.w);
    int depth = ctr & 0xFF, diffuseBounces = (ctr >> 8) & 0xFF, passThroughs = (ctr >> 16) & 0xFF,
        skips = (ctr >> 24) & 0xFF;
    Sobol sb;
    sb.pixelHash = __float_as_uint(pp.w);
    {
        const int sOff = (path - A.slotFirst) / A.nPix;
        sb.revIndex = rev32(static_cast<uint32_t>(A.sampleFirst + sOff));
    }
    sb.dim = __float_as_uint(lp.w);
    V3 thr = mk(th.x, th.y, th.z);
    const V3 dir = mk(rd.x, rd.y, rd.z);
    const V3 rayO = mk(ro.x, ro.y, ro.z);
    const float lastBsdfPdf = rd.w;
    const bool specularBounce = flags & PF_SPECULAR_BOUNCE;
    bool cameraRay = flags & PF_CAMERA_RAY;
    const int shadowSamples = A.shadowSamples;
    const int explicitLights = S.nLights;
    const int prim = __float_as_int(hr.w);
    const bool hit = KEY == 0 ? false : (KEY > 0 ? true : !isMiss(prim));
    const float time = pathTime(S, P, slot);
    // ray cone (path_tracer.cpp:428-454, 777-783, 853-857): only scenes with mipmapped textures
    const bool cones = !LEAN && S.hasMips && P.cone;
    float2 cone = cones ? P.cone[slot] : make_float2(0.0f, 0.0f);
    Isect is;
    bool done = false;
    bool vertex = false; // a surface vertex to shade (NEE + BSDF sampling) below
    bool exitVertex = false; // ... the exit vertex of a subsurface walk
    V3 wo = -dir;
    if (!LEAN && (flags & PF_WALK)) {
        // one step of the random walk (path_tracer.cpp:263-303)
        const V3 sigT = mk(lp.x, lp.y, lp.z), alb = mk(ln.x, ln.y, ln.z);
        const V3 sigS = alb * sigT;
        uint32_t step = volCtr >> 16;
        const float uc = get1D(sb);
        const float uf = get1D(sb);
        float t = 0.0f;
        const bool scattered = sampleFreeFlight(sigT, sigS, hit ? hr.x : kFltMax, hit, thr * alb, uc, uf, thr, t);
        if (!isFinite3(thr) || isBlack(thr)) {
            done = true;
        } else if (!scattered) {
            if (!hit) {
                done = true; // escaped through open geometry
            } else {
                Hit h;
                h.t = hr.x;
                h.u = hr.y;
                h.v = hr.z;
                h.prim = prim;
                fillHit(S, h, rayO, dir, is, time);
                // exit vertex: outward normal, white Lambert; the depth does not grow
                is.normal = -is.normal;
                is.material = S.exitMaterial;
                flags &= ~PF_WALK;
                wo = is.normal;
                exitVertex = true;
                if (depth >= A.maxDepth) done = true;
                else vertex = true;
            }
        } else {
            const V3 no = rayO + dir * t;
            const V3 nd = sampleHG(dir, pp.x, get2D(T, sb));
            if ((step >= 8u && !russianRoulette(thr, sb)) || ++step >= static_cast<uint32_t>(kMaxWalkSteps)) {
                done = true;
            } else {
                ro = make_float4(no.x, no.y, no.z, ro.w);
                rd = make_float4(nd.x, nd.y, nd.z, rd.w);
                volCtr = (volCtr & 0xFFFFu) | (step << 16);
                cont = true;
            }
        }
    } else {
        if (hit) {
            Hit h;
            h.t = hr.x;
            h.u = hr.y;
            h.v = hr.z;
            h.prim = prim;
            fillHit(S, h, rayO, dir, is, time);
            // Camera-invisible light quads (for camera rays) and cutouts are passed through;
            // the vertex does not count (path_tracer.cpp:426-439).
            if (skips < 64 && ((cameraRay && (S.shapes[is.shape].flags & SF_CAMERA_INVISIBLE)) ||
                               (!LEAN && passesCutout(S, S.materials[is.material], is, sb)))) {
                const V3 no = offsetRayOrigin(is.point, is.pError, is.ng, dir);
                ro = make_float4(no.x, no.y, no.z, ro.w);
                if (cones) cone.x = cone.x + cone.y * smax(0.0f, is.t);
                ++skips;
                cont = true;
                done = true;
            }
        }
        if (!done) {
            // AOVs of the camera path's first surface past the skipped ones (path_tracer.cpp:440-443;
            // tracePixel, renderer.cpp:177-203): albedo, normal and coverage, or the background
            // data passes of the first hit (tracePixel, renderer.cpp:162-176)
            if ((flags & PF_FIRST_SEGMENT) && (OUT && P.pass) && hit) {
                float4* b = passBlock(P, path);
                const float4 o = b[PASS_HIT];
                b[PASS_HIT] = make_float4(is.point.x, is.point.y, is.point.z, length(is.point - mk(o.x, o.y, o.z)));
                const float4 oc = S.idColor[is.shape];
                b[PASS_OBJECT] = make_float4(oc.x, oc.y, oc.z, 1.0f);
                b[PASS_MATERIAL] = S.idColor[S.nShapes + is.material];
                // Cryptomatte ids ride in the w of the id colours (renderer.cpp:170-175)
                b[PASS_CRYPTO] = make_float4(oc.w, b[PASS_MATERIAL].w, 0.0f, 0.0f);
            }
            if ((flags & PF_FIRST_SEGMENT) && OUT && P.aovA) {
                const int path = pathOfSlot(P, slot);
                if (hit) {
                    const V3 a = clamp3(m3f(S.materials[is.material].base), 0.0f, 1.0f);
                    P.aovA[path] = make_float4(a.x, a.y, a.z, 1.0f);
                    P.aovN[path] = make_float4(is.normal.x, is.normal.y, is.normal.z, 0.0f);
                } else {
                    V3 a = mk(0.0f);
                    if (S.bgMode == PE_BG_COLOR) a = m3f(S.bgColor);
                    else if (S.env.present) a = envEval(S.env, dir);
                    a = clamp3(a, 0.0f, 1.0f);
                    P.aovA[path] = make_float4(a.x, a.y, a.z, 0.0f);
                    P.aovN[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                }
            }
            flags &= ~PF_FIRST_SEGMENT;
            // inside an object: absorption and, when the medium scatters, free flight
            const int top = volumetric ? media.top() : -1;
            if (top >= 0 && (S.materials[top].flags & MF_HAS_MEDIUM)) {
                V3 no, nd;
                const int r = mediumSegment(T, S.materials[top], rayO, dir, hit, is.point, sb, thr, volCtr, no, nd);
                if (r == SEG_END) {
                    done = true;
                } else if (r == SEG_SCATTERED) {
                    // the next query starts at the scattering point; no NEE inside, so
                    // emission found next takes full weight
                    ro = make_float4(no.x, no.y, no.z, __uint_as_float(VIS_DIFFUSE));
                    rd = make_float4(nd.x, nd.y, nd.z, rd.w);
                    flags = (flags | PF_SPECULAR_BOUNCE) & ~PF_CAMERA_RAY;
                    if (cones) cone = make_float2(0.0f, 0.0f); // a new ray without a cone (path_tracer.cpp:465)
                    cont = true;
                    done = true;
                }
            }
        }
        if (!done) {
            if (!hit) {
                // environment / background (path_tracer.cpp:482-514)
                if (depth == 0 && S.bgMode != PE_BG_ENVIRONMENT) {
                    if (S.bgMode == PE_BG_COLOR) {
                        const V3 added = addL(L, thr * m3f(S.bgColor));
                        if ((OUT && P.pass)) {
                            passAdd(passBlock(P, path) + PASS_BACKGROUND, added);
                            creditGroup(S, P, path, S.envGroup, added);
                        }
                    } else if (passThroughs > 0 && OUT && P.aovA) {
                        // straight through thin glass to a transparent background: coverage is
                        // what the glass held back
                        P.aovA[pathOfSlot(P, slot)].w = smax(0.0f, 1.0f - luminance(thr));
                    }
                } else if (S.env.present) {
                    const V3 Le = envEval(S.env, dir);
                    float weight = 1.0f;
                    if (!specularBounce) {
                        float pmf = 0.0f;
                        if (flags & PF_PICKER_VALID) {
                            LightCtx c;
                            lightPrepare(S, mk(pp.x, pp.y, pp.z), mk(pn.x, pn.y, pn.z), c);
                            pmf = lightCtxPmf(S, c, explicitLights);
                        }
                        const float lightPdf = pmf * envPdf(S.env, dir);
                        weight = powerHeuristic(1, lastBsdfPdf, shadowSamples, lightPdf);
                    }
                    V3 c = thr * (Le * weight);
                    if (diffuseBounces >= 2 && A.clampIndirect > 0.0f) {
                        const float m = smax3(c.x, c.y, c.z);
                        if (m > A.clampIndirect) c = c * (A.clampIndirect / m);
                    }
                    const V3 added = addL(L, c);
                    if ((OUT && P.pass)) {
                        if (depth == 0) passAdd(passBlock(P, path) + PASS_BACKGROUND, added);
                        else creditPath(P, path, added, depth == 1);
                        creditGroup(S, P, path, S.envGroup, added);
                    }
                }
                done = true;
            } else if (!LEAN && cameraRay && is.shape == S.catcherShape) {
                // the shadow catcher ends the camera path with the shadowed background
                float ratio = 1.0f;
                const V3 bg = shadowCatcher(S, is, dir, shadowSamples, sb, ratio, time);
                const V3 added = addL(L, thr * bg * ratio);
                if ((OUT && P.pass)) {
                    passAdd(passBlock(P, path) + PASS_BACKGROUND, added);
                    creditGroup(S, P, path, S.envGroup, added);
                }
                if (depth == 0 && OUT && P.aovA) {
                    // the catcher's AOVs: the background it shows, its shadow as coverage
                    const V3 a = clamp3(bg, 0.0f, 1.0f);
                    P.aovA[pathOfSlot(P, slot)] =
                        make_float4(a.x, a.y, a.z, S.bgMode == PE_BG_TRANSPARENT ? 1.0f - ratio : 1.0f);
                }
                done = true;
            } else {
                const MatGPU& mat = S.materials[is.material];
                // emission with MIS against the previous vertex's NEE (path_tracer.cpp:565-593)
                if (mat.flags & MF_EMISSIVE) {
                    const ShapeInfo& sh = S.shapes[is.shape];
                    int li = -1;
                    if (sh.emitter >= 0)
                        li = (sh.flags & SF_AREA_TRIANGLE) ? sh.emitter : sh.emitter + (is.tri - static_cast<int>(sh.firstTri));
                    // Light linking: the previous receiver must be linked to this light
                    // (path_tracer.cpp:571-572; camera rays always see it)
                    const bool linked = depth == 0 || li < 0 || LEAN || !S.hasLightLinks ||
                                        linkAllows(S.links[li].mode, S.links[li].mask,
                                                   static_cast<int>((flags >> kPrevNodeShift) & 0xFFu));
                    float weight = 1.0f;
                    if (linked && !specularBounce) {
                        float lightPdf = 0.0f;
                        if (li >= 0) {
                            float pmf = 0.0f;
                            if (flags & PF_PICKER_VALID) {
                                LightCtx c;
                                lightPrepare(S, mk(pp.x, pp.y, pp.z), mk(pn.x, pn.y, pn.z), c);
                                pmf = lightCtxPmf(S, c, li);
                            }
                            lightPdf = pmf * lightPdfHit(S.lights[li], mk(lp.x, lp.y, lp.z), is.point);
                        }
                        if (lightPdf > 0.0f && lastBsdfPdf > 0.0f)
                            weight = powerHeuristic(1, lastBsdfPdf, shadowSamples, lightPdf);
                    }
                    if (linked) {
                        V3 c = thr * (m3f(mat.emission) * weight);
                        if (diffuseBounces >= 2 && A.clampIndirect > 0.0f) {
                            const float m = smax3(c.x, c.y, c.z);
                            if (m > A.clampIndirect) c = c * (A.clampIndirect / m);
                        }
                        const V3 added = addL(L, c);
                        if ((OUT && P.pass)) {
                            if (depth == 0) passAdd(passBlock(P, path) + PASS_EMISSION, added);
                            else creditPath(P, path, added, depth == 1);
                            creditGroup(S, P, path, li >= 0 ? lightGroupOf(S, li) : 0, added);
                        }
                    }
                }
                if (depth >= A.maxDepth) done = true;
                else vertex = true;
            }
        }
    }
    if (vertex) {
        const MatGPU& mat = S.materials[is.material];
        // dispersion: the first wavelength-dependent surface fixes one λ for the path
        if (!LEAN && lambda == 0.0f && (mat.flags & MF_DISPERSIVE)) {
            V3 w;
            lambda = sampleWavelength(T, get1D(sb), w);
            thr *= w;
        }
        // rounded edges on the first three vertices (not a walk's exit vertex), then contact AO at
        // the camera hit (path_tracer.cpp:612-621)
        if (!LEAN && depth <= 2 && mat.roundEdge > 0.0f && !exitVertex) {
            const V3 n = roundedEdgeNormal(S, is, mat.roundEdge, sb, time);
            if (dot(n, wo) > 0.02f) is.normal = n;
        }
        if (!LEAN && A.aoStrength > 0.0f && depth == 0) thr *= approxAo(S, is, sb, A.aoStrength, shadowSamples, time);
        ShadePoint sp;
        sp.uv = is.uv;
        sp.textures = S.textures;
        sp.uvDensity = is.uvDensity;
        sp.footprint = 0.0f;
        if (cones && !exitVertex && (cone.x > 0.0f || cone.y > 0.0f)) {
            const V3 nGeom = len2(is.ng) > 0.0f ? is.ng : is.normal;
            const float cosInc = smax(0.15f, fabsf(dot(-dir, nGeom)));
            sp.footprint = (cone.x + cone.y * smax(0.0f, is.t)) / cosInc;
        }
        sp.p = is.point;
        sp.n = is.normal;
        sp.ng = is.ng;
        sp.tangent = is.tangent;
        sp.frontFace = is.frontFace;
        sp.wavelength = lambda;
        const bool isSpecular = (mat.flags & MF_DELTA) != 0;
        // this bounce's proposal, when the inference kernel left one for the slot
        const bool useGuide = !LEAN && P.guiding == 2 && guidable(mat) && P.guideMark[slot] != 0u;
        if (useGuide) P.guideMark[slot] = 0u;
        // or the SD-tree's sampling quadtree of the vertex's spatial leaf (path_tracer.cpp:627-629)
        int sdRoot = -1;
        if (!LEAN && (P.sdMode & SD_SAMPLE) && !useGuide && guidable(mat)) {
            const int leaf = sdLeafWithData(P.sd, is.point);
            if (leaf >= 0) sdRoot = P.sd.leaves[leaf].sampRoot;
        }
        // next-event estimation (path_tracer.cpp:631-698)
        if (S.lightCount > 0 && !isSpecular) {
            LightCtx picker;
            lightPrepare(S, is.point, is.normal, picker);
            flags |= PF_PICKER_VALID;
            pp = make_float4(is.point.x, is.point.y, is.point.z, pp.w);
            pn.x = is.normal.x;
            pn.y = is.normal.y;
            pn.z = is.normal.z;
            for (int s = 0; s < shadowSamples; ++s) {
                float lightPmf = 0.0f;
                const int lightIndex = lightCtxSample(S, picker, get1D(sb), lightPmf);
                if (lightIndex < 0 || !(lightPmf > 0.0f)) {
                    (void)get2D(T, sb);
                    continue;
                }
                const bool fromEnv = lightIndex >= explicitLights;
                if (!LEAN && !fromEnv && S.hasLightLinks &&
                    !linkAllows(S.links[lightIndex].mode, S.links[lightIndex].mask, S.shapes[is.shape].linkNode)) {
                    (void)get2D(T, sb);
                    continue;
                }
                const V2 ul = get2D(T, sb);
                const LightSample ls = fromEnv ? envSample(S.env, ul) : sampleLight(S.lights[lightIndex], is.point, ul);
                if (!lsValid(ls)) continue;
                V3 so, sd;
                float stMax;
                if (!makeShadowRay(is, ls.wi, ls.distance, so, sd, stMax)) continue;
                float bsdfPdf = 0.0f;
                LobeSplit3 split;
                const bool firstShares = (OUT && P.pass) && depth == 0;
                const V3 f = bsdfEvalPdfT<MT>(T, mat, wo, ls.wi, sp, bsdfPdf, firstShares ? &split : nullptr);
                const float cosTheta = fabsf(dot(ls.wi, is.normal));
                if (isBlack(f) || !(cosTheta > 0.0f)) continue;
                const float lightPdf = lightPmf * ls.pdf;
                const float contPdf = useGuide     ? 0.5f * bsdfPdf + 0.5f * guidePdf(P, slot, ls.wi)
                                      : sdRoot >= 0 ? 0.5f * bsdfPdf + 0.5f * sdTreePdf(P.sd.samp, sdRoot, ls.wi)
                                                    : bsdfPdf;
                const float weight = powerHeuristic(shadowSamples, lightPdf, 1, contPdf);
                const float scalar = cosTheta * weight / (lightPdf * static_cast<float>(shadowSamples));
                const V3 fLi = f * ls.Li;
                if (INLINE_SHADOW) {
                    // the any-hit query now; its term follows this vertex's emission in L
                    ++shRays;
                    const V3 vis = shadowVisibility<COUNT>(S, so, sd, stMax, fromEnv ? -1 : lightIndex, shNodes, shTris, time);
                    if (!isBlack(vis)) {
                        const V3 c = neeTerm(fLi, vis, scalar, thr, diffuseBounces >= 1, A.clampIndirect);
                        if (isFinite3(c)) {
                            L.x += c.x;
                            L.y += c.y;
                            L.z += c.z;
                            if ((OUT && P.pass)) {
                                float4 shares[3];
                                if (firstShares) {
                                    V3 sh[3];
                                    lobeShares(split, sh);
                                    for (int k = 0; k < 3; ++k) shares[k] = make_float4(sh[k].x, sh[k].y, sh[k].z, 1.0f);
                                }
                                creditNee(S, P, path, fromEnv ? -1 : lightIndex, c, firstShares ? shares : nullptr);
                            }
                        }
                    }
                } else {
                    // shadow queue append (one record per sample)
                    const uint32_t pos = atomicAdd(&P.counters[CNT_SHADOW], 1u);
                    P.shadowQ[pos] = slot;
                    P.shO[pos] = make_float4(so.x, so.y, so.z, stMax);
                    P.shD[pos] = make_float4(sd.x, sd.y, sd.z, scalar);
                    // flags: bit 0 indirect, bits 1.. the light index + 1 (0: the environment)
                    const uint32_t lightBits = static_cast<uint32_t>(fromEnv ? 0 : lightIndex + 1) << 1;
                    P.shC[pos] = make_float4(fLi.x, fLi.y, fLi.z, __uint_as_float((diffuseBounces >= 1 ? 1u : 0u) | lightBits));
                    P.shT[pos] = make_float4(thr.x, thr.y, thr.z, A.clampIndirect);
                    if ((OUT && P.pass)) {
                        float4* q = P.shPass + 3 * static_cast<size_t>(pos);
                        if (firstShares) {
                            V3 sh[3];
                            lobeShares(split, sh);
                            for (int k = 0; k < 3; ++k) q[k] = make_float4(sh[k].x, sh[k].y, sh[k].z, 1.0f);
                        } else {
                            q[0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        }
                    }
                }
            }
        }
        // BSDF (and proposal) sampling (path_tracer.cpp:700-743)
        BsdfSample bs;
        bool sampled;
        if (useGuide) {
            sampled = guidedSample(T, mat, wo, sp, P, slot, sb, bs);
        } else if (sdRoot >= 0) {
            sampled = sdGuidedSample(T, mat, wo, sp, P.sd.samp, sdRoot, sb, bs);
        } else {
            const float uc = get1D(sb);
            const V2 u2 = get2D(T, sb);
            sampled = bsdfSampleT<MT>(T, mat, wo, sp, uc, u2, bs);
        }
        if (!sampled) {
            done = true;
        } else if (!LEAN && bs.subsurface) {
            // random-walk entry (path_tracer.cpp:745-761): the walk's coefficients ride
            // in the columns it does not need (lastP, lastN, pickP.x)
            V3 sigT, alb;
            float g = 0.0f;
            const DisneyParams dp = disneyResolve(mat, sp);
            if (!disneySubsurfaceCoeffs(mat, dp, sigT, alb, g)) {
                done = true;
            } else {
                thr *= bs.weight;
                const V3 d = normalize(bs.wi);
                const V3 no = spawnOrigin(is, d);
                ro = make_float4(no.x, no.y, no.z, __uint_as_float(VIS_ALL | RAY_WALK));
                rd = make_float4(d.x, d.y, d.z, rd.w);
                lp = make_float4(sigT.x, sigT.y, sigT.z, 0.0f);
                ln = make_float4(alb.x, alb.y, alb.z, 0.0f);
                pp.x = g;
                volCtr &= 0xFFFFu; // walk step 0
                flags = (flags | PF_WALK) & ~PF_CAMERA_RAY;
                cont = true;
            }
        } else if (bs.pdf <= 0.0f || isBlack(bs.f)) {
            done = true;
        } else if (bs.passThrough) {
            thr *= bs.f * (fabsf(dot(bs.wi, is.normal)) / bs.pdf);
            if (!isFinite3(thr) || ++passThroughs > 64) {
                done = true;
            } else {
                const V3 no = spawnOrigin(is, bs.wi);
                ro = make_float4(no.x, no.y, no.z, ro.w);
                rd = make_float4(bs.wi.x, bs.wi.y, bs.wi.z, rd.w);
                if (cones) cone.x = cone.x + cone.y * smax(0.0f, is.t);
                skips = 0;
                cont = true;
            }
        } else {
            const V3 wi = bs.wi;
            const bool refracted = dot(wo, is.ng) * dot(wi, is.ng) < 0.0f;
            if ((OUT && P.pass) && depth == 0) {
                // the first surface's lobe shares: all later light splits by them (path_tracer.cpp:797-812)
                V3 sh[3];
                if (bs.delta) {
                    sh[0] = mk(0.0f);
                    sh[1] = mk(refracted ? 0.0f : 1.0f);
                    sh[2] = mk(refracted ? 1.0f : 0.0f);
                } else {
                    LobeSplit3 split;
                    float unusedPdf = 0.0f;
                    (void)bsdfEvalPdfT<MT>(T, mat, wo, wi, sp, unusedPdf, &split);
                    lobeShares(split, sh);
                }
                float4* b = passBlock(P, path);
                for (int k = 0; k < 3; ++k) b[PASS_LOBES + k] = make_float4(sh[k].x, sh[k].y, sh[k].z, 0.0f);
            }
            const float cosTheta = fabsf(dot(wi, is.normal));
            const V3 thrBefore = thr;
            thr *= bs.f * (cosTheta / bs.pdf);
            if (!LEAN && P.guiding && !bs.delta && slot % P.guideStride == 0 && guidable(mat) && isFinite3(thr) &&
                guideRecord(P, slot, is.point, is.normal, wo, wi, thrBefore))
                flags |= PF_GUIDE_SNAP;
            if (!isFinite3(thr)) {
                done = true;
            } else {
                flags = bs.delta ? (flags | PF_SPECULAR_BOUNCE) : (flags & ~PF_SPECULAR_BOUNCE);
                // this vertex is the next emission hit's receiver (path_tracer.cpp:832)
                flags = (flags & ~kPrevNodeMask) | (static_cast<uint32_t>(S.shapes[is.shape].linkNode) << kPrevNodeShift);
                if (!bs.delta) ++diffuseBounces;
                cameraRay = cameraRay && bs.delta && dot(wi, is.normal) < 0.0f;
                flags = cameraRay ? (flags | PF_CAMERA_RAY) : (flags & ~PF_CAMERA_RAY);
                // crossing a volume boundary: enter the object's medium from outside,
                // leave it from inside
                if (!LEAN && (mat.flags & MF_VOLUME_BOUNDARY)) {
                    const float a = dot(wo, is.ng), b = dot(wi, is.ng);
                    if (a * b < 0.0f) {
                        if (a > 0.0f) media.enter(is.material);
                        else media.leave(is.material);
                    }
                }
                const uint32_t nextMask = refracted ? VIS_TRANSMISSION : (bs.delta ? VIS_GLOSSY : VIS_DIFFUSE);
                if (cones) {
                    cone.x = cone.x + cone.y * smax(0.0f, is.t);
                    cone.y = cone.y + (bs.delta ? 0.0f : 0.12f);
                }
                ln = make_float4(is.normal.x, is.normal.y, is.normal.z, 0.0f);
                lp = make_float4(is.point.x, is.point.y, is.point.z, 0.0f);
                const V3 no = spawnOrigin(is, wi);
                ro = make_float4(no.x, no.y, no.z, __uint_as_float(nextMask));
                rd = make_float4(wi.x, wi.y, wi.z, bs.pdf);
                ++depth;
                skips = 0;
                cont = true;
                if (depth > A.rrDepth && !russianRoulette(thr, sb)) {
                    cont = false;
                    done = true;
                }
                // SD-tree training vertex (path_tracer.cpp:823-827, recordable ones only): its
                // incident radiance is what L gains from here on over the throughput after the
                // bounce and the roulette
                if (!LEAN && cont && (P.sdMode & SD_RECORD) && !bs.delta && !(mat.flags & MF_VOLUME_BOUNDARY)) {
                    const uint32_t n = P.sdCount[slot];
                    if (n < static_cast<uint32_t>(kSdRecords)) {
                        float4* rec = P.sdRec + (static_cast<size_t>(slot) * kSdRecords + n) * 4;
                        rec[0] = make_float4(is.point.x, is.point.y, is.point.z, bs.pdf);
                        rec[1] = make_float4(wi.x, wi.y, wi.z, 0.0f);
                        rec[2] = make_float4(thr.x, thr.y, thr.z, 0.0f);
                        rec[3] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                        P.sdCount[slot] = n + 1;
                        flags |= PF_GUIDE_SNAP;
                    }
                }
            }
        }
    }
    // write back
    P.L[slot] = L;
    if (cont) {
        if (cones) P.cone[slot] = cone;
        P.rayO[slot] = ro;
        P.rayD[slot] = rd;
        P.thr[slot] = make_float4(thr.x, thr.y, thr.z, lambda);
        P.lastN[slot] = make_float4(ln.x, ln.y, ln.z, __uint_as_float(flags));
        P.lastP[slot] = make_float4(lp.x, lp.y, lp.z, __uint_as_float(sb.dim));
        P.pickP[slot] = pp;
        P.pickN[slot] = make_float4(pn.x, pn.y, pn.z, __uint_as_float(packCounters(depth, diffuseBounces, passThroughs, skips)));
        if (volumetric)
            P.med[slot] = make_float4(__uint_as_float(media.lo), __uint_as_float(media.hi), __uint_as_float(volCtr),
                                      __int_as_float(media.n));
    }
    return cont;
}

// Consumes the rays binned by shading key (segment by segment, so a warp mostly shades one
// material kind) and appends the continuing paths to nextQueue.
// OUT: the wave records AOVs or render passes (their code is compiled out of the plain kernel).
// INLINE: NEE shadow rays are traced here, each sample's term added in the sample loop's order
// (waves with shadowQuality > 1, whose several records per vertex the shadow queue does not hold).
template <bool OUT, bool INLINE = false>
__global__ void __launch_bounds__(128, 6) kShade(SceneGPU S, Paths P, Wave W, int32_t* nextQueue, uint32_t* nextCount) {
    uint32_t seg[kShadeKeys];
    int n = 0;
    for (int k = 0; k < kShadeKeys; ++k) {
        seg[k] = P.counters[CNT_KEYS + k];
        n += static_cast<int>(seg[k]);
    }
    const int lane = threadIdx.x & 31;
    uint32_t unused0 = 0, unused1 = 0, unused2 = 0;
    for (;;) {
        const int base = warpFetch(&P.counters[CNT_WORK_SHADE]);
        if (base >= n) break;
        const int i = base + lane;
        bool cont = false, sweepable = false;
        int slot = -1;
        if (i < n) {
            int k = 0;
            uint32_t j = static_cast<uint32_t>(i);
            while (k < kShadeKeys - 1 && j >= seg[k]) {
                j -= seg[k];
                ++k;
            }
            slot = P.sortQ[static_cast<size_t>(k) * P.capacity + j];
            const int path = pathOfSlot(P, slot);
            const WaveSeg& A = W.segs[segOfSlot(W, path)];
            cont = shadeSlot<INLINE, false, OUT>(S, P, A, slot, path, unused0, unused1, unused2);
            sweepable = (A.flags & SEG_SWEEP) != 0;
        }
        // a continuous wave sweeps its interactive paths that have lived sweepAge bounces into a
        // tail launch, so that their requests do not wait on one bounce per wavefront step
        const bool old = P.sweepAge > 0 && cont && sweepable && P.iter - P.born[slot] >= P.sweepAge;
        queuePush(nextQueue, nextCount, cont && !old, slot);
        if (P.sweepAge > 0) queuePush(P.sweepQ, &P.counters[CNT_SWEEP], old, slot);
        // a regenerating wave refills the slots of ended paths
        if (P.pathOf) queuePush(P.freeQ, &P.counters[CNT_FREE], !cont && slot >= 0, slot);
    }
}

// The lean shading kernel of one shading key: the rays of that key's bin only, shaded by the
// shadeSlot instantiation that carries the code of that key alone (waves of lean-shading scenes
// without guiding; one launch per key, each with the registers its key needs).
// MINB: at least this many 128-thread blocks per SM (__launch_bounds__), i.e. a register budget
// of 65536 / (128·MINB) per thread; 1 leaves the count to the compiler (pe_tuning::shade_budget).
template <bool OUT, int KEY, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) kShadeKey(SceneGPU S, Paths P, Wave W, int32_t* nextQueue, uint32_t* nextCount) {
    const int n = static_cast<int>(P.counters[CNT_KEYS + KEY]);
    const int32_t* bin = P.sortQ + static_cast<size_t>(KEY) * P.capacity;
    const int lane = threadIdx.x & 31;
    uint32_t unused0 = 0, unused1 = 0, unused2 = 0;
    for (;;) {
        const int base = warpFetch(&P.counters[CNT_WORK_KEYS + KEY]);
        if (base >= n) break;
        const int i = base + lane;
        bool cont = false, sweepable = false;
        int slot = -1;
        if (i < n) {
            slot = bin[i];
            const int path = pathOfSlot(P, slot);
            const WaveSeg& A = W.segs[segOfSlot(W, path)];
            cont = shadeSlot<false, false, OUT, KEY>(S, P, A, slot, path, unused0, unused1, unused2);
            sweepable = (A.flags & SEG_SWEEP) != 0;
        }
        // continuous waves sweep interactive paths that have lived sweepAge bounces, as kShade does
        const bool old = P.sweepAge > 0 && cont && sweepable && P.iter - P.born[slot] >= P.sweepAge;
        queuePush(nextQueue, nextCount, cont && !old, slot);
        if (P.sweepAge > 0) queuePush(P.sweepQ, &P.counters[CNT_SWEEP], old, slot);
        if (P.pathOf) queuePush(P.freeQ, &P.counters[CNT_FREE], !cont && slot >= 0, slot);
    }
}

// ---- tail: the last paths of a wave, each run to its end by one thread -------------------------
// Once a wave's live queue fits in one resident grid, per-bounce launches cost more than they
// save: each thread takes a path from the queue, alternates closest-hit queries with shadeSlot
// (shadow rays inline) until the path ends, then takes the next.  The arithmetic and the order of
// L's terms are the wavefront's, so the film is the same bit for bit.  This one-warp-per-block
// form serves the counting pass and waves with AOV or pass outputs; plain waves and the request
// server's sweeps and drains use kTailLockstep below.
constexpr int kTailBlock = 32;

template <bool COUNT, bool OUT>
__global__ void __launch_bounds__(kTailBlock) kTail(SceneGPU S, Paths P, Wave W, const int32_t* queue, const uint32_t* count,
                                             uint32_t* cursor, unsigned long long* stats) {
    const int n = static_cast<int>(*count);
    uint32_t nodes = 0, tris = 0, shNodes = 0, shTris = 0, rays = 0, shRays = 0;
    for (;;) {
        const int i = static_cast<int>(atomicAdd(cursor, 1u));
        if (i >= n) break;
        const int slot = queue[i];
        const int path = pathOfSlot(P, slot);
        const WaveSeg& A = W.segs[segOfSlot(W, path)];
        for (int q = 0;; ++q) {
            if (q >= kMaxPathQueries) {
                atomicAdd(&stats[7], 1ull);
                break;
            }
            const float4 ro = P.rayO[slot];
            const float4 rd = P.rayD[slot];
            const Hit h = traceClosestWide<COUNT>(S, mk(ro.x, ro.y, ro.z), mk(rd.x, rd.y, rd.z), __float_as_uint(ro.w), 0.0f,
                                              1e30f, nodes, tris, nullptr, pathTime(S, P, slot));
            ++rays;
            P.hit[slot] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
            if (!shadeSlot<true, COUNT, OUT>(S, P, A, slot, path, shNodes, shTris, shRays)) break;
        }
    }
    if (COUNT) {
        atomicAdd(&stats[0], static_cast<unsigned long long>(nodes));
        atomicAdd(&stats[1], static_cast<unsigned long long>(tris));
        atomicAdd(&stats[2], static_cast<unsigned long long>(shNodes));
        atomicAdd(&stats[3], static_cast<unsigned long long>(shTris));
    }
    atomicAdd(&stats[5], static_cast<unsigned long long>(rays));
    atomicAdd(&stats[6], static_cast<unsigned long long>(shRays));
}

// The tail in lockstep: the same per-path work as kTail<false, false, LEAN>, but the
// four warps of a 128-thread block meet at a barrier between each bounce's closest-hit query and
// its shading, so the warps sharing an SM run the same phase's code at once.  The loop body
// (traversal, every lean material's shading, the inline shadow ray) is far larger than an SM
// sub-partition's instruction cache; warps of 32-thread blocks, each at its own point of the
// loop, spend most of their stalls fetching instructions.  Threads whose paths have ended take
// the queue's next path at the top of the loop; the block leaves when none of its threads holds
// one.  Each path's queries and terms are kTail's, so the film is the same bit for bit.
constexpr int kTailLockstepBlock = 128;
template <bool LEAN>
__global__ void __launch_bounds__(kTailLockstepBlock) kTailLockstep(SceneGPU S, Paths P, Wave W, const int32_t* queue,
                                                                  const uint32_t* count, uint32_t* cursor,
                                                                  unsigned long long* stats) {
    const int n = static_cast<int>(*count);
    uint32_t nodes = 0, tris = 0, shNodes = 0, shTris = 0, rays = 0, shRays = 0;
    int slot = -1, path = 0, q = 0;
    const WaveSeg* A = nullptr;
    bool exhausted = false; // this thread found the queue taken
    for (;;) {
        if (slot < 0 && !exhausted) {
            const int i = static_cast<int>(atomicAdd(cursor, 1u));
            if (i < n) {
                slot = queue[i];
                path = pathOfSlot(P, slot);
                A = &W.segs[segOfSlot(W, path)];
                q = 0;
            } else {
                exhausted = true;
            }
        }
        if (!__syncthreads_or(slot >= 0)) break;
        if (slot >= 0) {
            const float4 ro = P.rayO[slot];
            const float4 rd = P.rayD[slot];
            const Hit h = traceClosestWide<false>(S, mk(ro.x, ro.y, ro.z), mk(rd.x, rd.y, rd.z), __float_as_uint(ro.w), 0.0f,
                                              1e30f, nodes, tris, nullptr, pathTime(S, P, slot));
            ++rays;
            P.hit[slot] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
        }
        __syncthreads();
        if (slot >= 0) {
            if (!shadeSlot<true, false, false, LEAN ? -2 : -1>(S, P, *A, slot, path, shNodes, shTris, shRays)) {
                slot = -1;
            } else if (++q >= kMaxPathQueries) {
                // as kTail: a path past the per-path query bound is ended and reported
                atomicAdd(&stats[7], 1ull);
                slot = -1;
            }
        }
    }
    atomicAdd(&stats[5], static_cast<unsigned long long>(rays));
    atomicAdd(&stats[6], static_cast<unsigned long long>(shRays));
}

// ---- film: Film::addSample in sample order per pixel (src/core/image/film.cpp:56-69) ----------
// The AOV films of one pixel (addAovs, renderer.cpp:219-224): albedo and alpha by addSample,
// the normal by addSampleSigned (film.cpp:73-85), in sample order.
__device__ __noinline__ void filmAovs(const Paths& P, const WaveSeg& A, int p, int pix) {
    const size_t n = static_cast<size_t>(A.width) * static_cast<size_t>(A.height);
    for (int f = 0; f < 3; ++f) {
        float* fsum = A.aov + static_cast<size_t>(f) * 5 * n;
        uint32_t* fcnt = reinterpret_cast<uint32_t*>(fsum + 3 * n);
        float* fsq = fsum + 4 * n;
        float r = fsum[3 * pix + 0], g = fsum[3 * pix + 1], b = fsum[3 * pix + 2], q = fsq[pix];
        uint32_t c = fcnt[pix];
        for (int s = 0; s < A.nSamples; ++s) {
            const int path = A.slotFirst + s * A.nPix + p;
            V3 v;
            if (f == 0) {
                const float4 a = P.aovA[path];
                v = mk(a.x, a.y, a.z);
            } else if (f == 1) {
                const float4 nn = P.aovN[path];
                v = mk(nn.x, nn.y, nn.z);
            } else {
                v = mk(P.aovA[path].w);
            }
            ++c;
            if (!(finitef(v.x) && finitef(v.y) && finitef(v.z))) continue;
            if (f != 1 && !(v.x >= 0.0f && v.y >= 0.0f && v.z >= 0.0f)) continue;
            r += v.x;
            g += v.y;
            b += v.z;
            if (f != 1) {
                const float lum = luminance(v);
                q += lum * lum;
            }
        }
        fsum[3 * pix + 0] = r;
        fsum[3 * pix + 1] = g;
        fsum[3 * pix + 2] = b;
        fsq[pix] = q;
        fcnt[pix] = c;
    }
}

// The render-pass films of one pixel (addPasses, renderer.cpp:206-217), in sample order: light
// passes, depth, ids and light groups by addSample, the position by addSampleSigned.
__device__ __noinline__ void filmPasses(const Paths& P, const WaveSeg& A, int p, int pix) {
    const size_t n = static_cast<size_t>(A.width) * static_cast<size_t>(A.height);
    const int nFilms = PFILM_GROUPS + (P.passStride - PASS_GROUPS);
    for (int f = 0; f < nFilms; ++f) {
        float* fsum = A.pass + static_cast<size_t>(f) * 5 * n;
        uint32_t* fcnt = reinterpret_cast<uint32_t*>(fsum + 3 * n);
        float* fsq = fsum + 4 * n;
        const int slotOf = f < PFILM_DEPTH ? f
                         : f == PFILM_DEPTH || f == PFILM_POSITION ? PASS_HIT
                         : f == PFILM_OBJECT ? PASS_OBJECT
                         : f == PFILM_MATERIAL ? PASS_MATERIAL
                                               : PASS_GROUPS + (f - PFILM_GROUPS);
        const bool isSigned = f == PFILM_POSITION;
        float r = fsum[3 * pix + 0], g = fsum[3 * pix + 1], b = fsum[3 * pix + 2], q = fsq[pix];
        uint32_t c = fcnt[pix];
        for (int s = 0; s < A.nSamples; ++s) {
            const float4* blk = passBlock(P, A.slotFirst + s * A.nPix + p);
            const float4 v4 = blk[slotOf];
            V3 v = mk(v4.x, v4.y, v4.z);
            if (f == PFILM_DEPTH || f == PFILM_POSITION) {
                const bool hit = blk[PASS_OBJECT].w != 0.0f;
                v = !hit ? mk(0.0f) : f == PFILM_DEPTH ? mk(v4.w) : v;
            }
            ++c;
            if (!(finitef(v.x) && finitef(v.y) && finitef(v.z))) continue;
            if (!isSigned && !(v.x >= 0.0f && v.y >= 0.0f && v.z >= 0.0f)) continue;
            r += v.x;
            g += v.y;
            b += v.z;
            if (!isSigned) {
                const float lum = luminance(v);
                q += lum * lum;
            }
        }
        fsum[3 * pix + 0] = r;
        fsum[3 * pix + 1] = g;
        fsum[3 * pix + 2] = b;
        fsq[pix] = q;
        fcnt[pix] = c;
    }
    if (A.cryptoObj) {
        // each sample's Cryptomatte ids; the host adds them to its CryptoFilms
        for (int s = 0; s < A.nSamples; ++s) {
            const float4 id = passBlock(P, A.slotFirst + s * A.nPix + p)[PASS_CRYPTO];
            const size_t o = static_cast<size_t>(A.sampleFirst + s - A.cryptoFirst) * n + static_cast<size_t>(pix);
            A.cryptoObj[o] = id.x;
            A.cryptoMat[o] = id.y;
        }
    }
}

__global__ void kFilm(Paths P, Wave W, unsigned long long* rejected) {
    unsigned long long rej = 0;
    for (int wp = blockIdx.x * blockDim.x + threadIdx.x; wp < W.nPix; wp += gridDim.x * blockDim.x) {
        const WaveSeg& A = W.segs[segOfPixel(W, wp)];
        const int p = wp - A.pixFirst;
        const int tp = A.pixelFirst + p;
        const int pix = A.pixList ? A.pixList[tp] : (A.tileY + tp / A.tileW) * A.width + A.tileX + tp % A.tileW;
        float* sum = A.sum;
        float sr = sum[3 * pix + 0], sg = sum[3 * pix + 1], sbb = sum[3 * pix + 2];
        float sq = A.sq[pix];
        uint32_t c = A.cnt[pix];
        for (int s = 0; s < A.nSamples; ++s) {
            const int path = A.slotFirst + s * A.nPix + p;
            const float4 L = P.Lout ? P.Lout[path] : P.L[path];
            ++c;
            const bool ok = finitef(L.x) && finitef(L.y) && finitef(L.z) && L.x >= 0.0f && L.y >= 0.0f && L.z >= 0.0f;
            if (!ok) {
                ++rej;
                continue;
            }
            sr += L.x;
            sg += L.y;
            sbb += L.z;
            const float lum = luminance(mk(L.x, L.y, L.z));
            sq += lum * lum;
        }
        sum[3 * pix + 0] = sr;
        sum[3 * pix + 1] = sg;
        sum[3 * pix + 2] = sbb;
        A.sq[pix] = sq;
        A.cnt[pix] = c;
        if (A.aov && P.aovA) filmAovs(P, A, p, pix);
        if (A.pass && P.pass) filmPasses(P, A, p, pix);
    }
    if (rej) atomicAdd(rejected, rej);
}

} // namespace pe
