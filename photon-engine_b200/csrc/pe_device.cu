// pe_device.cu — the CUDA device behind the pe_device_* C ABI: resident scene upload, the
// wavefront render loop (RenderDevice::render, src/engine/render_device.h:84-85) and the
// diagnostics the parity tests call.  Built for sm_100a only.
#include "pe_device_impl.h"
#include "pe_integrator.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using namespace pe;
using namespace pe_dev;

namespace pe_dev {

int32_t allocLane(WaveLane& ln, size_t slots) {
    freeList(ln.bufs);
    int32_t st = 0;
    Paths& P = ln.paths;
    float4** cols[] = {&P.rayO, &P.rayD, &P.thr, &P.L, &P.lastN, &P.lastP, &P.pickP, &P.pickN, &P.hit, &P.med};
    for (float4** c : cols)
        if ((st = devAlloc(ln.bufs, *c, slots))) return st;
    if ((st = devAlloc(ln.bufs, P.queueA, slots))) return st;
    if ((st = devAlloc(ln.bufs, P.queueB, slots))) return st;
    if ((st = devAlloc(ln.bufs, P.sortQ, slots * kShadeKeys))) return st;
    // shadow records: one per slot (shadow quality 1)
    if ((st = devAlloc(ln.bufs, P.shadowQ, slots))) return st;
    float4** scols[] = {&P.shO, &P.shD, &P.shC, &P.shT};
    for (float4** c : scols)
        if ((st = devAlloc(ln.bufs, *c, slots))) return st;
    if ((st = devAlloc(ln.bufs, P.counters, CNT_TOTAL))) return st;
    if ((st = devAlloc(ln.bufs, P.cone, slots))) return st;
    if ((st = devAlloc(ln.bufs, P.time, slots))) return st;
    // path regeneration: slot → path, freed slots, radiance of kStreamFactor × slots paths
    if ((st = devAlloc(ln.bufs, ln.pathOf, slots))) return st;
    if ((st = devAlloc(ln.bufs, ln.freeQ, slots))) return st;
    if ((st = devAlloc(ln.bufs, ln.Lout, slots * kStreamFactor))) return st;
    P.capacity = static_cast<uint32_t>(slots);
    return PE_OK;
}

// Per-slot buffers of `slots` paths (d->capacity: guided, AOV and pass waves size their own
// buffers by it); each lane's path state holds max(slots, d->waveSlots) slots, the regenerating
// waves' paths in flight.  Grows only.
int32_t ensureCapacity(pe_device* d, size_t slots) {
    const size_t cap = std::max(slots, d->capacity);
    const size_t lane = std::max(cap, d->waveSlots);
    if (cap == d->capacity && lane <= d->laneSlots) return PE_OK;
    d->capacity = 0;
    d->laneSlots = 0;
    for (WaveLane& ln : d->lanes) {
        const int32_t st = allocLane(ln, lane);
        if (st) return st;
    }
    d->capacity = cap;
    d->laneSlots = lane;
    return PE_OK;
}

// Device inverse-CDF table of a pixel filter.  `wave` stamps the slot so that a wave under
// construction never evicts a table that it or the previous wave (possibly still running on the
// other lane) reads.  Returns nullptr when no slot is free of both.
const float* filterTable(pe_device* d, int type, float width, uint64_t wave, cudaStream_t stream) {
    int pick = -1;
    for (int i = 0; i < kFilterSlots; ++i)
        if (d->filterSlots[i].type == type && d->filterSlots[i].width == width) {
            d->filterSlots[i].used = wave;
            return d->dFilters + static_cast<size_t>(i) * (kFilterBins + 1);
        }
    for (int i = 0; i < kFilterSlots && pick < 0; ++i)
        if (d->filterSlots[i].type < 0) pick = i; // never filled
    if (pick < 0)
        for (int i = 0; i < kFilterSlots; ++i) {
            if (d->filterSlots[i].used + 1 >= wave) continue; // this wave's or the wave still in flight
            if (pick < 0 || d->filterSlots[i].used < d->filterSlots[pick].used) pick = i;
        }
    if (pick < 0) return nullptr;
    float cdf[kFilterBins + 1];
    fillFilterCdf(type, width, cdf);
    // on the stream of the wave that reads it; no wave still in flight reads the evicted table
    if (cudaMemcpyAsync(d->dFilters + static_cast<size_t>(pick) * (kFilterBins + 1), cdf, sizeof(cdf),
                        cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return nullptr;
    d->filterSlots[pick] = FilterSlot{type, width, wave};
    return d->dFilters + static_cast<size_t>(pick) * (kFilterBins + 1);
}

int32_t ensureFilm(pe_device* d, int w, int h) {
    if (w == d->filmW && h == d->filmH && d->fSum) return PE_OK;
    cudaFree(d->fSum);
    cudaFree(d->fCnt);
    cudaFree(d->fSq);
    d->fSum = nullptr;
    d->fCnt = nullptr;
    d->fSq = nullptr;
    const size_t n = static_cast<size_t>(w) * static_cast<size_t>(h);
    PE_CUDA(cudaMalloc(&d->fSum, n * 3 * sizeof(float)));
    PE_CUDA(cudaMalloc(&d->fCnt, n * sizeof(uint32_t)));
    PE_CUDA(cudaMalloc(&d->fSq, n * sizeof(float)));
    PE_CUDA(cudaMemsetAsync(d->fSum, 0, n * 3 * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(d->fCnt, 0, n * sizeof(uint32_t), d->stream));
    PE_CUDA(cudaMemsetAsync(d->fSq, 0, n * sizeof(float), d->stream));
    d->filmW = w;
    d->filmH = h;
    return PE_OK;
}

int32_t checkSettings(const pe_camera* cam, const pe_settings* st) {
    if (!cam || !st) {
        setError("null camera or settings");
        return PE_ERR_INVALID;
    }
    if (st->width <= 0 || st->height <= 0 || st->width > 16384 || st->height > 16384) {
        setError("film size out of range (1..16384)");
        return PE_ERR_INVALID;
    }
    if (st->max_bounces < 0 || st->max_bounces > 255) {
        setError("max_bounces out of range (0..255)");
        return PE_ERR_LIMIT;
    }
    if (st->shadow_quality < 1 || st->shadow_quality > 64) {
        setError("shadow_quality out of range (1..64)");
        return PE_ERR_LIMIT;
    }
    if (!(cam->lens_radius >= 0.0f) || cam->blades < 0 || cam->blades > 64) {
        setError("camera lens radius must be >= 0 and blades in 0..64");
        return PE_ERR_INVALID;
    }
    if (!(st->ao_strength >= 0.0f) || !(st->ao_strength <= 1e30f)) {
        setError("ao_strength must be finite and >= 0");
        return PE_ERR_INVALID;
    }
    return PE_OK;
}

// A request's render settings as a wave segment (film, rectangle and ranges filled in later).
WaveSeg makeSeg(const pe_camera* cam, const pe_settings* st) {
    WaveSeg A{};
    A.cam.position = m3f(cam->position);
    A.cam.lowerLeft = m3f(cam->lower_left);
    A.cam.horizontal = m3f(cam->horizontal);
    A.cam.vertical = m3f(cam->vertical);
    A.cam.u = m3f(cam->u);
    A.cam.v = m3f(cam->v);
    A.cam.forward = m3f(cam->forward);
    A.cam.lensRadius = cam->orthographic ? 0.0f : (cam->lens_radius > 0.0f ? cam->lens_radius : 0.0f);
    A.cam.blades = cam->blades >= 3 ? cam->blades : 0;
    A.cam.bladeRotation = cam->blade_rotation;
    A.cam.orthographic = cam->orthographic ? 1 : 0;
    A.cam.hasEnd = cam->has_shutter_end ? 1 : 0;
    if (A.cam.hasEnd) {
        A.cam.position1 = m3f(cam->end_position);
        A.cam.lowerLeft1 = m3f(cam->end_lower_left);
        A.cam.horizontal1 = m3f(cam->end_horizontal);
        A.cam.vertical1 = m3f(cam->end_vertical);
        A.cam.u1 = m3f(cam->end_u);
        A.cam.v1 = m3f(cam->end_v);
        A.cam.forward1 = m3f(cam->end_forward);
        A.cam.lensRadius1 = cam->end_lens_radius;
    }
    A.flags = st->motion_blur ? SEG_MOTION : 0;
    A.width = st->width;
    A.height = st->height;
    A.seed = st->seed;
    A.filterWidth = sclamp(st->filter_width, 0.25f, 8.0f);
    A.maxDepth = st->max_bounces;
    A.rrDepth = st->rr_depth;
    A.shadowSamples = st->shadow_quality < 1 ? 1 : st->shadow_quality;
    A.clampIndirect = st->clamp_indirect > 0.0f ? st->clamp_indirect : 0.0f;
    A.aoStrength = st->ao_strength > 0.0f ? st->ao_strength : 0.0f;
    // Camera::pixelConeWidth / pixelConeSpread (camera.h:94-109): a pixel's width for the
    // orthographic camera, the angle a pixel subtends at the image plane's centre otherwise
    if (st->height > 0) {
        const float h = static_cast<float>(st->height);
        if (A.cam.orthographic) {
            A.coneWidth = length(A.cam.vertical) / h;
        } else {
            const V3 center = A.cam.lowerLeft + A.cam.horizontal * 0.5f + A.cam.vertical * 0.5f;
            const float dist = smax(1e-4f, length(center - A.cam.position));
            A.coneSpread = std::atan(length(A.cam.vertical) / (dist * h));
        }
    }
    return A;
}


// SceneGPU::leanShading of a scene: true when none of its materials and scene settings use a
// shading feature that the lean shading kernels compile out.
int32_t leanShadingOf(const SceneGPU& G, const std::vector<MatGPU>& mats) {
    if (G.hasVolumes || G.hasSubsurface || G.hasMips || G.hasLightLinks || G.hasShadowLinks || G.catcherShape >= 0)
        return 0;
    for (const MatGPU& m : mats) {
        if (m.roundEdge > 0.0f || (m.flags & (MF_DISPERSIVE | MF_VOLUME_BOUNDARY | MF_HAS_MEDIUM))) return 0;
        if (m.type == PE_MAT_DISNEY && (m.opacity < 1.0f || m.texOpacity >= 0)) return 0;
    }
    return 1;
}

// Scratch of pe_device_render_tile_noalloc: path-state columns, queues, shadow records and
// counters for kNoAllocSlots paths, carved out of one file-scope device array (8.5 MB).  Every
// GPU that loads this library holds the array until the process exits.
constexpr size_t kNoAllocSlots = size_t(1) << 15;
constexpr size_t kNoAllocColumn = kNoAllocSlots * sizeof(float4);   // 512 KiB, 256-aligned
constexpr size_t kNoAllocIndex = kNoAllocSlots * sizeof(int32_t);    // 128 KiB, 256-aligned
constexpr size_t kNoAllocBytes = 14 * kNoAllocColumn + (3 + kShadeKeys) * kNoAllocIndex + 256;
static __device__ __align__(256) unsigned char g_noAllocScratch[kNoAllocBytes];

// Path-state view of the scratch whose device address is `base`.
Paths noAllocPaths(unsigned char* base) {
    Paths P{};
    size_t off = 0;
    auto col = [&](float4*& c) { c = reinterpret_cast<float4*>(base + off); off += kNoAllocColumn; };
    auto idx = [&](int32_t*& c, size_t n) { c = reinterpret_cast<int32_t*>(base + off); off += n * kNoAllocIndex; };
    col(P.rayO); col(P.rayD); col(P.thr); col(P.L); col(P.lastN); col(P.lastP); col(P.pickP); col(P.pickN); col(P.hit);
    col(P.med);
    col(P.shO); col(P.shD); col(P.shC); col(P.shT);
    idx(P.queueA, 1); idx(P.queueB, 1); idx(P.shadowQ, 1); idx(P.sortQ, kShadeKeys);
    P.counters = reinterpret_cast<uint32_t*>(base + off);
    P.capacity = static_cast<uint32_t>(kNoAllocSlots);
    return P;
}

// The lean shading kernels of one bounce, one per shading key whose material type the scene
// uses (the miss key always); returns the number of launches.
int launchLeanShade(pe_device* d, const SceneGPU& S, const Paths& P, const Wave& W, int32_t* qOut, uint32_t* cOut,
                    cudaStream_t cs, bool out) {
    int n = 0;
    const int budget = d->shadeBudget;
    auto one = [&](auto kernel, int key) {
        if (key > 0 && !(S.materialTypes & (1 << (key - 1)))) return;
        kernel<<<d->blocksShadeKey[budget][key], 128, 0, cs>>>(S, P, W, qOut, cOut);
        ++n;
    };
    if (!out && budget == 2) {
        one(kShadeKey<false, 0, 5>, 0);
        one(kShadeKey<false, 1, 5>, 1);
        one(kShadeKey<false, 2, 5>, 2);
        one(kShadeKey<false, 3, 5>, 3);
        one(kShadeKey<false, 4, 5>, 4);
    } else if (!out && budget == 1) {
        one(kShadeKey<false, 0, 4>, 0);
        one(kShadeKey<false, 1, 4>, 1);
        one(kShadeKey<false, 2, 4>, 2);
        one(kShadeKey<false, 3, 4>, 3);
        one(kShadeKey<false, 4, 4>, 4);
    } else if (out) {
        one(kShadeKey<true, 0>, 0);
        one(kShadeKey<true, 1>, 1);
        one(kShadeKey<true, 2>, 2);
        one(kShadeKey<true, 3>, 3);
        one(kShadeKey<true, 4>, 4);
    } else {
        one(kShadeKey<false, 0>, 0);
        one(kShadeKey<false, 1>, 1);
        one(kShadeKey<false, 2>, 2);
        one(kShadeKey<false, 3>, 3);
        one(kShadeKey<false, 4>, 4);
    }
    return n;
}

int32_t timerEvent(pe_device* d, RenderTimer& tm, cudaEvent_t& e) {
    if (tm.evUsed >= d->evPool.size()) {
        cudaEvent_t ne;
        PE_CUDA(cudaEventCreate(&ne));
        d->evPool.push_back(ne);
    }
    e = d->evPool[tm.evUsed++];
    return PE_OK;
}

// Starts a render call's statistics and its device clock.
int32_t beginRender(pe_device* d) {
    std::memset(&d->stats, 0, sizeof(d->stats));
    PE_CUDA(cudaMemsetAsync(d->dStats, 0, 8 * sizeof(unsigned long long), d->stream));
    PE_CUDA(cudaEventRecord(d->evStart, d->stream));
    PE_CUDA(cudaStreamWaitEvent(d->lanes[1].stream, d->evStart, 0));
    d->filmLane = -1;
    return PE_OK;
}

// Ends it: waits for the stream, then reads the device counters and per-kernel times.
int32_t endRender(pe_device* d, const RenderTimer& tm) {
    pe_render_stats& stats = d->stats;
    // join the second lane into the device stream
    if (d->lanes[1].pending) {
        PE_CUDA(cudaStreamWaitEvent(d->stream, d->lanes[1].evDone, 0));
        d->lanes[1].pending = false;
    }
    d->lanes[0].pending = false;
    PE_CUDA(cudaEventRecord(d->evStop, d->stream));
    unsigned long long hs[8] = {};
    PE_CUDA(cudaMemcpyAsync(hs, d->dStats, sizeof(hs), cudaMemcpyDeviceToHost, d->stream));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    PE_CUDA(cudaGetLastError());
    float ms = 0.0f;
    PE_CUDA(cudaEventElapsedTime(&ms, d->evStart, d->evStop));
    stats.ms_total = ms;
    auto sum = [&](const std::vector<std::pair<size_t, size_t>>& v) {
        float acc = 0.0f;
        for (const auto& pr : v) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, d->evPool[pr.first], d->evPool[pr.second]);
            acc += t;
        }
        return acc;
    };
    stats.ms_intersect = sum(tm.isect);
    stats.ms_shade = sum(tm.shade);
    stats.ms_shadow = sum(tm.shadow);
    stats.ms_tail = sum(tm.tail);
    stats.node_visits = hs[0];
    stats.tri_tests = hs[1];
    stats.shadow_node_visits = hs[2];
    stats.shadow_tri_tests = hs[3];
    stats.rejected = hs[4];
    stats.closest_rays += hs[5];
    stats.shadow_rays += hs[6];
    stats.tail_closest_rays = hs[5];
    stats.tail_shadow_rays = hs[6];
    if (hs[7] != 0) {
        setError(std::to_string(hs[7]) + " paths exceeded the per-path query bound and were ended");
        return PE_ERR_DEVICE;
    }
    return PE_OK;
}

// A lane's pinned segment table may be rewritten only once its previous upload has run.
int32_t segsWritable(pe_device* d, int lane) {
    WaveLane& ln = d->lanes[lane];
    if (ln.segsInFlight) {
        PE_CUDA(cudaEventSynchronize(ln.evSegs));
        ln.segsInFlight = false;
    }
    return PE_OK;
}

static_assert(sizeof(pe_device::blocksIntersectMode) / sizeof(int) == TRACE_MODES, "a grid size per traversal mode");

// The tail in lockstep over `n` queued paths (count and cursor on the device).
void launchTailLockstep(pe_device* d, bool lean, const SceneGPU& S, const Paths& P, const Wave& W, const int32_t* queue,
                        const uint32_t* count, uint32_t* cursor, int64_t n, cudaStream_t cs) {
    const int grid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>(d->blocksTailLockstep[lean ? 1 : 0], (n + kTailLockstepBlock - 1) / kTailLockstepBlock)));
    if (lean) kTailLockstep<true><<<grid, kTailLockstepBlock, 0, cs>>>(S, P, W, queue, count, cursor, d->dStats);
    else kTailLockstep<false><<<grid, kTailLockstepBlock, 0, cs>>>(S, P, W, queue, count, cursor, d->dStats);
}

// The closest-hit kernel of the tuned traversal (pe_tuning::closest_traversal) over a queue.
void launchClosest(pe_device* d, const SceneGPU& S, const Paths& P, const int32_t* q, const uint32_t* c, cudaStream_t cs) {
    const int* g = d->blocksIntersectMode;
    unsigned long long* st = d->dStats;
    switch (d->closestMode) {
    case TRACE_BINARY: kIntersect<false, TRACE_BINARY><<<g[TRACE_BINARY], 128, 0, cs>>>(S, P, q, c, st); break;
    case TRACE_WIDE_SMEM8: kIntersect<false, TRACE_WIDE_SMEM8><<<g[TRACE_WIDE_SMEM8], 128, 0, cs>>>(S, P, q, c, st); break;
    case TRACE_WIDE_SMEM16: kIntersect<false, TRACE_WIDE_SMEM16><<<g[TRACE_WIDE_SMEM16], 128, 0, cs>>>(S, P, q, c, st); break;
    case TRACE_WIDE_REG4: kIntersect<false, TRACE_WIDE_REG4><<<g[TRACE_WIDE_REG4], 128, 0, cs>>>(S, P, q, c, st); break;
    case TRACE_WIDE_REG8: kIntersect<false, TRACE_WIDE_REG8><<<g[TRACE_WIDE_REG8], 128, 0, cs>>>(S, P, q, c, st); break;
    case TRACE_WIDE_OCC8: kIntersect<false, TRACE_WIDE_OCC8><<<g[TRACE_WIDE_OCC8], 128, 0, cs>>>(S, P, q, c, st); break;
    case TRACE_WIDE_SMEM8_OCC8:
        kIntersect<false, TRACE_WIDE_SMEM8_OCC8><<<g[TRACE_WIDE_SMEM8_OCC8], 128, 0, cs>>>(S, P, q, c, st);
        break;
    case TRACE_WIDE_SMEM16_OCC8:
        kIntersect<false, TRACE_WIDE_SMEM16_OCC8><<<g[TRACE_WIDE_SMEM16_OCC8], 128, 0, cs>>>(S, P, q, c, st);
        break;
    case TRACE_WIDE_SPEC_OCC8:
        kIntersect<false, TRACE_WIDE_SPEC_OCC8><<<g[TRACE_WIDE_SPEC_OCC8], 128, 0, cs>>>(S, P, q, c, st);
        break;
    default: kIntersect<false><<<d->blocksIntersect, 128, 0, cs>>>(S, P, q, c, st); break;
    }
}

// The plain any-hit shadow kernel of the tuned variant (pe_tuning::any_traversal).
void launchShadowAny(pe_device* d, const SceneGPU& S, const Paths& P, cudaStream_t cs) {
    uint32_t* n = &P.counters[CNT_SHADOW];
    unsigned long long* st = d->dStats;
    switch (d->anyMode) {
    case 1: kShadow<false, true, 4><<<d->blocksShadowAnyWindow, 128, 0, cs>>>(S, P, n, st); break;
    case 2: kShadow<false, true, 0, 8><<<d->blocksShadowAnyOcc8, 128, 0, cs>>>(S, P, n, st); break;
    default: kShadow<false, true><<<d->blocksShadowAny, 128, 0, cs>>>(S, P, n, st); break;
    }
}

// One wave on a lane over the nSegs segments in its segment table (nSlots paths, nPix film
// pixels): uploads the table, generates the camera rays, traces them bounce by bounce (closest
// hit → shade → any hit) until the live paths fit the tail kernel, which finishes them, and adds
// every sample to its segment's film in sample order, after the previous wave's film kernel.
// The host waits for each bounce's queue count, not for the tail or the film kernel.
int32_t runWave(pe_device* d, int lane, Paths& P, int nSegs, int nSlots, int nPix, RenderTimer& tm) {
    WaveLane& ln = d->lanes[lane];
    const cudaStream_t cs = ln.stream;
    (void)cudaGetLastError(); // launch errors below are this wave's, not an earlier call's
    const SceneGPU& S = d->scene;
    const int sm = d->prop.multiProcessorCount;
    pe_render_stats& stats = d->stats;
    int32_t rc = PE_OK;
    PE_CUDA(cudaMemcpyAsync(ln.dSegs, ln.hSegs, static_cast<size_t>(nSegs) * sizeof(WaveSeg), cudaMemcpyHostToDevice,
                            cs));
    PE_CUDA(cudaEventRecord(ln.evSegs, cs));
    ln.segsInFlight = true;
    const Wave W{ln.dSegs, nSegs, nSlots, nPix};
    // learned proposal: record training samples; sample with it once warm
    const GuideState& G = d->guide;
    P.guiding = (G.mode && P.guideQ) ? (G.step >= G.warmup ? 2 : 1) : 0;
    P.guideStride = 1;
    while (nSlots / P.guideStride > kGuideTrainRows) P.guideStride *= 2;
    // SD-tree guiding: the field as it stands, recording and sampling as the schedule says
    P.sdMode = (d->guideKind == 2 && P.sdRec) ? d->sd.waveMode : 0;
    P.sd = d->sd.field;
    // path regeneration: a wave of more paths than slots (unguided waves on a lane's own state,
    // wave_slots of them in flight); other waves on a lane's state use d->capacity slots, which
    // the guide, AOV and pass buffers are sized by
    const bool lanePaths = &P == &ln.paths;
    const bool regenOk = lanePaths && ln.Lout && !P.guiding && !P.sdMode && !d->aovTarget && !d->passTarget;
    const int64_t slotCap = static_cast<int64_t>(
        std::min<size_t>(P.capacity, regenOk ? d->waveSlots : (lanePaths ? d->capacity : P.capacity)));
    const bool regen = regenOk && nSlots > slotCap;
    P.pathOf = regen ? ln.pathOf : nullptr;
    P.freeQ = regen ? ln.freeQ : nullptr;
    P.Lout = regen ? ln.Lout : nullptr;
    P.segLeft = nullptr;
    P.aovA = (d->aovTarget && &P == &ln.paths) ? ln.aovA : nullptr;
    P.aovN = (d->aovTarget && &P == &ln.paths) ? ln.aovN : nullptr;
    const bool passes = d->passTarget && &P == &ln.paths;
    P.pass = passes ? ln.pass : nullptr;
    P.shPass = passes ? ln.shPass : nullptr;
    P.passStride = passes ? d->passStride : 0;
    P.born = nullptr;
    P.sweepQ = nullptr;
    P.sweepAge = 0;
    if (nSlots > (regen ? slotCap * kStreamFactor : slotCap)) {
        setError("wave of " + std::to_string(nSlots) + " paths exceeds its path state");
        return PE_ERR_LIMIT;
    }
    const int firstPaths = static_cast<int>(std::min<int64_t>(nSlots, slotCap));
    int nextPath = firstPaths;
    kGenerate<<<sm * 8, 256, 0, cs>>>(S, P, W, firstPaths);
    ++stats.kernel_launches;
    ++stats.waves;
    uint32_t live = static_cast<uint32_t>(firstPaths);
    PE_CUDA(cudaMemsetAsync(&P.counters[1], 0, (CNT_TOTAL - 1) * sizeof(uint32_t), cs));
    PE_CUDA(cudaMemcpyAsync(&P.counters[0], &live, sizeof(uint32_t), cudaMemcpyHostToDevice, cs));
    int32_t* qIn = P.queueA;
    int32_t* qOut = P.queueB;
    uint32_t* cIn = &P.counters[0];
    uint32_t* cOut = &P.counters[1];
    stats.paths += static_cast<uint64_t>(nSlots);
    // lean shading (one specialised kernel per shading key) for plain surface scenes that
    // neither guide nor record; shadows without transmitters or shadow links are plain any-hits
    bool noAo = true, inlineShadows = false;
    for (int k = 0; k < nSegs; ++k) {
        noAo = noAo && !(ln.hSegs[k].aoStrength > 0.0f);
        inlineShadows = inlineShadows || ln.hSegs[k].shadowSamples > 1;
    }
    const bool lean = S.leanShading && !P.guiding && !P.sdMode && noAo && !d->counting && !inlineShadows;
    const bool anyHitShadows = !S.hasShadowTransmitters && !S.hasShadowLinks;
    int64_t tailPaths = d->tailPaths < 0 ? static_cast<int64_t>(d->blocksTail) * kTailBlock : d->tailPaths;
    // the tail kernel runs no inference: keep guided bounces in the wavefront until few paths remain
    if (P.guiding == 2) tailPaths = std::min<int64_t>(tailPaths, kGuideTailPaths);
    for (int iter = 0; live > 0; ++iter) {
        if (static_cast<int64_t>(live) <= tailPaths && nextPath == nSlots) {
            // the rest of the wave: one thread per path until it ends
            const int grid = static_cast<int>(
                std::min<int64_t>(d->blocksTail, (static_cast<int64_t>(live) + kTailBlock - 1) / kTailBlock));
            cudaEvent_t t0 = nullptr, t1 = nullptr;
            if (tm.timing) {
                if ((rc = timerEvent(d, tm, t0)) || (rc = timerEvent(d, tm, t1))) return rc;
                PE_CUDA(cudaEventRecord(t0, cs));
            }
            const bool out = P.aovA || P.pass;
            if (lean && !d->counting && !out)
                launchTailLockstep(d, true, S, P, W, qIn, cIn, &P.counters[CNT_WORK_TAIL], live, cs);
            else if (d->counting && out)
                kTail<true, true><<<grid, kTailBlock, 0, cs>>>(S, P, W, qIn, cIn, &P.counters[CNT_WORK_TAIL], d->dStats);
            else if (d->counting)
                kTail<true, false><<<grid, kTailBlock, 0, cs>>>(S, P, W, qIn, cIn, &P.counters[CNT_WORK_TAIL], d->dStats);
            else if (out)
                kTail<false, true><<<grid, kTailBlock, 0, cs>>>(S, P, W, qIn, cIn, &P.counters[CNT_WORK_TAIL], d->dStats);
            else
                launchTailLockstep(d, false, S, P, W, qIn, cIn, &P.counters[CNT_WORK_TAIL], live, cs);
            if (tm.timing) {
                PE_CUDA(cudaEventRecord(t1, cs));
                tm.tail.push_back({tm.evUsed - 2, tm.evUsed - 1});
            }
            ++stats.kernel_launches;
            stats.tail_paths += live;
            if (regen) {
                kFlush<<<sm * 4, 256, 0, cs>>>(P, W, qIn, cIn);
                ++stats.kernel_launches;
            }
            break;
        }
        stats.closest_rays += live;
        cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
        if (tm.timing) {
            if ((rc = timerEvent(d, tm, e0)) || (rc = timerEvent(d, tm, e1)) || (rc = timerEvent(d, tm, e2)) ||
                (rc = timerEvent(d, tm, e3)))
                return rc;
            PE_CUDA(cudaEventRecord(e0, cs));
        }
        if (d->counting && d->closestMode == TRACE_BINARY)
            kIntersect<true, TRACE_BINARY><<<d->blocksIntersectMode[0], 128, 0, cs>>>(S, P, qIn, cIn, d->dStats);
        else if (d->counting)
            kIntersect<true><<<d->blocksIntersect, 128, 0, cs>>>(S, P, qIn, cIn, d->dStats);
        else
            launchClosest(d, S, P, qIn, cIn, cs);
        if (P.guiding == 2 && (rc = guideQueries(d, cs, P, W, qIn, cIn))) return rc;
        if (tm.timing) PE_CUDA(cudaEventRecord(e1, cs));
        if (lean)
            stats.kernel_launches += launchLeanShade(d, S, P, W, qOut, cOut, cs, P.aovA || P.pass);
        else if (inlineShadows && (P.aovA || P.pass))
            kShade<true, true><<<d->blocksShade, 128, 0, cs>>>(S, P, W, qOut, cOut);
        else if (inlineShadows)
            kShade<false, true><<<d->blocksShade, 128, 0, cs>>>(S, P, W, qOut, cOut);
        else if (P.aovA || P.pass)
            kShade<true><<<d->blocksShade, 128, 0, cs>>>(S, P, W, qOut, cOut);
        else
            kShade<false><<<d->blocksShade, 128, 0, cs>>>(S, P, W, qOut, cOut);
        if (tm.timing) PE_CUDA(cudaEventRecord(e2, cs));
        if (d->counting)
            kShadow<true><<<d->blocksShadow, 128, 0, cs>>>(S, P, &P.counters[CNT_SHADOW], d->dStats);
        else if (anyHitShadows)
            launchShadowAny(d, S, P, cs);
        else
            kShadow<false><<<d->blocksShadow, 128, 0, cs>>>(S, P, &P.counters[CNT_SHADOW], d->dStats);
        stats.kernel_launches += lean ? 2 : 3;
        ++stats.intersect_launches;
        if (tm.timing) {
            PE_CUDA(cudaEventRecord(e3, cs));
            tm.isect.push_back({tm.evUsed - 4, tm.evUsed - 3});
            tm.shade.push_back({tm.evUsed - 3, tm.evUsed - 2});
            tm.shadow.push_back({tm.evUsed - 2, tm.evUsed - 1});
        }
        PE_CUDA(cudaMemcpyAsync(ln.hCounters, P.counters, CNT_TOTAL * sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
        PE_CUDA(cudaStreamSynchronize(cs));
        stats.shadow_rays += ln.hCounters[CNT_SHADOW];
        live = cOut == &P.counters[1] ? ln.hCounters[1] : ln.hCounters[0];
        if (regen) {
            // ended paths hand over their radiance; their slots take the wave's next paths
            const int freed = static_cast<int>(ln.hCounters[CNT_FREE]);
            const int fresh = std::min(freed, nSlots - nextPath);
            if (freed > 0) {
                kRecycle<<<sm * 4, 256, 0, cs>>>(S, P, W, freed, fresh, nextPath, qOut, static_cast<int>(live), cOut);
                ++stats.kernel_launches;
                PE_CUDA(cudaMemsetAsync(&P.counters[CNT_FREE], 0, sizeof(uint32_t), cs));
            }
            nextPath += fresh;
            live += static_cast<uint32_t>(fresh);
        }
        if (iter > kMaxWavefrontIterations * (regen ? kStreamFactor + 1 : 1)) {
            setError("wavefront did not drain after " + std::to_string(kMaxWavefrontIterations) + " iterations");
            return PE_ERR_DEVICE;
        }
        // swap queues; reset the consumed queue's counter, the shadow counter, the work
        // cursors and the shading-key bins
        PE_CUDA(cudaMemsetAsync(cIn, 0, sizeof(uint32_t), cs));
        PE_CUDA(cudaMemsetAsync(&P.counters[CNT_SHADOW], 0, (CNT_KEYS + kShadeKeys - CNT_SHADOW) * sizeof(uint32_t),
                                cs));
        if (lean) PE_CUDA(cudaMemsetAsync(&P.counters[CNT_WORK_KEYS], 0, kShadeKeys * sizeof(uint32_t), cs));
        std::swap(qIn, qOut);
        std::swap(cIn, cOut);
    }
    // films accumulate in wave order: after the other lane's last film kernel
    if (d->filmLane >= 0 && d->filmLane != lane) PE_CUDA(cudaStreamWaitEvent(cs, d->evFilm, 0));
    kFilm<<<sm * 4, 256, 0, cs>>>(P, W, &d->dStats[4]);
    PE_CUDA(cudaEventRecord(d->evFilm, cs));
    d->filmLane = lane;
    ++stats.kernel_launches;
    if (P.guiding && (rc = guideLearn(d, cs, P, nSlots))) return rc;
    if ((P.sdMode & SD_RECORD) && (rc = sdRecord(d, cs, P, nSlots))) return rc;
    PE_CUDA(cudaEventRecord(ln.evDone, cs));
    ln.pending = true;
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

// ---- continuous waves (the request server) ----------------------------------------------------
// A lane whose wave never drains while work arrives: every bounce the slots of ended paths hand
// their radiance to Lout and return to a free stack, from which new requests' paths are injected.

int32_t loopBegin(pe_device* d, LaneLoop& L, uint32_t* segLeft) {
    WaveLane& ln = *L.ln;
    Paths& P = ln.paths;
    const cudaStream_t cs = ln.stream;
    (void)cudaGetLastError();
    P.guiding = 0;
    P.sdMode = 0;
    P.pathOf = ln.pathOf;
    P.freeQ = ln.freeQ;
    P.Lout = ln.Lout;
    P.segLeft = segLeft;
    P.aovA = nullptr;
    P.aovN = nullptr;
    P.pass = nullptr;
    P.shPass = nullptr;
    P.passStride = 0;
    P.born = L.born;
    P.sweepQ = nullptr;
    P.sweepAge = 0;
    P.iter = 0;
    for (int b = 0; b < LaneLoop::kSweepBufs; ++b) L.sweepN[b] = 0;
    L.sweeping = 0;
    L.qIn = P.queueA;
    L.qOut = P.queueB;
    L.cIn = &P.counters[0];
    L.cOut = &P.counters[1];
    L.live = 0;
    L.freeTop = static_cast<int>(P.capacity);
    L.nextPath = 0;
    L.pathCap = static_cast<int>(static_cast<int64_t>(P.capacity) * kStreamFactor);
    L.iter = 0;
    PE_CUDA(cudaMemsetAsync(P.counters, 0, CNT_TOTAL * sizeof(uint32_t), cs));
    kInitFree<<<d->prop.multiProcessorCount * 4, 256, 0, cs>>>(P, static_cast<int>(P.capacity));
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int32_t loopInject(pe_device* d, LaneLoop& L, const Wave& W, int fresh) {
    if (fresh <= 0) return PE_OK;
    WaveLane& ln = *L.ln;
    Paths& P = ln.paths;
    P.iter = L.iter;
    kInject<<<d->prop.multiProcessorCount * 4, 256, 0, ln.stream>>>(L.scene, P, W, L.freeTop, fresh, L.nextPath, L.qIn,
                                                                    static_cast<int>(L.live), L.cIn);
    PE_CUDA(cudaGetLastError());
    L.freeTop -= fresh;
    L.nextPath += fresh;
    L.live += static_cast<uint32_t>(fresh);
    return PE_OK;
}

int32_t loopBounce(pe_device* d, LaneLoop& L, const Wave& W, uint32_t* hSegLeft, const uint32_t* dSegLeft, int segFirst,
                   int segCount) {
    WaveLane& ln = *L.ln;
    Paths& P = ln.paths;
    const cudaStream_t cs = ln.stream;
    const SceneGPU& S = L.scene;
    // a free sweep buffer takes this bounce's old paths (none free: no sweep this bounce)
    int sweep = -1;
    if (L.sweepAge > 0 && (L.sweepLive <= 0 || static_cast<int64_t>(L.live) <= L.sweepLive))
        for (int b = 0; b < LaneLoop::kSweepBufs && sweep < 0; ++b)
            if (L.sweepN[b] == 0) sweep = b;
    P.sweepAge = sweep >= 0 ? L.sweepAge : 0;
    P.sweepQ = sweep >= 0 ? L.sweepBuf[sweep] : nullptr;
    P.iter = L.iter;
    // the tuned closest-hit and any-hit kernels, as a lone render uses
    launchClosest(d, S, P, L.qIn, L.cIn, cs);
    // lean-shading scenes shade with the per-key kernels, as a lone render does
    if (L.lean) launchLeanShade(d, S, P, W, L.qOut, L.cOut, cs, false);
    else kShade<false><<<d->blocksShade, 128, 0, cs>>>(S, P, W, L.qOut, L.cOut);
    if (!S.hasShadowTransmitters && !S.hasShadowLinks)
        launchShadowAny(d, S, P, cs);
    else
        kShadow<false><<<d->blocksShadow, 128, 0, cs>>>(S, P, &P.counters[CNT_SHADOW], d->dStats);
    PE_CUDA(cudaMemcpyAsync(ln.hCounters, P.counters, CNT_TOTAL * sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
    // segment counts as of the previous bounce's flushes (one bounce behind)
    if (segCount > 0)
        PE_CUDA(cudaMemcpyAsync(hSegLeft + segFirst, dSegLeft + segFirst, static_cast<size_t>(segCount) * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, cs));
    PE_CUDA(cudaStreamSynchronize(cs));
    L.live = L.cOut == &P.counters[1] ? ln.hCounters[1] : ln.hCounters[0];
    const int top = static_cast<int>(ln.hCounters[CNT_FREE]);
    const int freed = top - L.freeTop;
    if (freed > 0) {
        kFlushFreed<<<d->prop.multiProcessorCount * 4, 256, 0, cs>>>(P, W, L.freeTop, freed);
    }
    L.freeTop = top;
    const int swept = static_cast<int>(ln.hCounters[CNT_SWEEP]);
    if (sweep >= 0 && swept > 0) {
        // the swept paths run to their end on the side stream, then hand over their radiance
        PE_CUDA(cudaMemcpyAsync(&L.sweepCnt[sweep], &P.counters[CNT_SWEEP], sizeof(uint32_t), cudaMemcpyDeviceToDevice, cs));
        PE_CUDA(cudaMemsetAsync(&P.counters[CNT_SWEEP], 0, sizeof(uint32_t), cs));
        PE_CUDA(cudaEventRecord(L.evReady[sweep], cs));
        PE_CUDA(cudaStreamWaitEvent(L.side, L.evReady[sweep], 0));
        PE_CUDA(cudaMemsetAsync(&L.sweepCursor[sweep], 0, sizeof(uint32_t), L.side));
        launchTailLockstep(d, L.lean, S, P, W, L.sweepBuf[sweep], &L.sweepCnt[sweep], &L.sweepCursor[sweep],
                           static_cast<int64_t>(swept), L.side);
        kFlush<<<d->prop.multiProcessorCount * 4, 256, 0, L.side>>>(P, W, L.sweepBuf[sweep], &L.sweepCnt[sweep]);
        PE_CUDA(cudaEventRecord(L.evDone[sweep], L.side));
        L.sweepN[sweep] = swept;
        L.sweeping += swept;
    }
    PE_CUDA(cudaMemsetAsync(L.cIn, 0, sizeof(uint32_t), cs));
    PE_CUDA(cudaMemsetAsync(&P.counters[CNT_SHADOW], 0, (CNT_KEYS + kShadeKeys - CNT_SHADOW) * sizeof(uint32_t), cs));
    if (L.lean) PE_CUDA(cudaMemsetAsync(&P.counters[CNT_WORK_KEYS], 0, kShadeKeys * sizeof(uint32_t), cs));
    std::swap(L.qIn, L.qOut);
    std::swap(L.cIn, L.cOut);
    if (++L.iter > kMaxWavefrontIterations * 64) {
        setError("continuous wave exceeded its bounce bound");
        return PE_ERR_DEVICE;
    }
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int32_t loopTail(pe_device* d, LaneLoop& L, const Wave& W) {
    if (L.live == 0) return PE_OK;
    WaveLane& ln = *L.ln;
    Paths& P = ln.paths;
    const cudaStream_t cs = ln.stream;
    launchTailLockstep(d, L.lean, L.scene, P, W, L.qIn, L.cIn, &P.counters[CNT_WORK_TAIL], static_cast<int64_t>(L.live), cs);
    kFlush<<<d->prop.multiProcessorCount * 4, 256, 0, cs>>>(P, W, L.qIn, L.cIn);
    L.live = 0;
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int32_t loopReturn(pe_device* d, LaneLoop& L, bool wait) {
    if (L.sweeping == 0) return PE_OK;
    WaveLane& ln = *L.ln;
    for (int b = 0; b < LaneLoop::kSweepBufs; ++b) {
        if (L.sweepN[b] == 0) continue;
        const cudaError_t e = wait ? cudaEventSynchronize(L.evDone[b]) : cudaEventQuery(L.evDone[b]);
        if (e == cudaErrorNotReady) continue;
        if (e != cudaSuccess) {
            setError(std::string("sweep: ") + cudaMsg(e));
            return PE_ERR_CUDA;
        }
        kReturnSlots<<<d->prop.multiProcessorCount * 2, 256, 0, ln.stream>>>(ln.paths, L.sweepBuf[b], L.sweepN[b],
                                                                             L.freeTop);
        PE_CUDA(cudaGetLastError());
        L.freeTop += L.sweepN[b];
        L.sweeping -= L.sweepN[b];
        L.sweepN[b] = 0;
    }
    return PE_OK;
}

int32_t loopFilm(pe_device* d, LaneLoop& L, const WaveSeg* dSeg, int nPix) {
    WaveLane& ln = *L.ln;
    const Wave one{dSeg, 1, nPix, nPix};
    kFilm<<<std::max(1, std::min(d->prop.multiProcessorCount * 4, (nPix + 255) / 256)), 256, 0, ln.stream>>>(
        ln.paths, one, &d->dStats[4]);
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

// The wavefront render of samples [first, first+count) over `tile` into the film (sum, cnt, sq)
// on the device, with path state in `P` (room for `capacity` slots): waves of one segment each.
// With `timing` the closest-hit / shade / any-hit / tail launches are bracketed by events.
// With `pixList` the pixels rendered are the nList film pixels it names (tile: the whole frame).
int32_t renderWaves(pe_device* d, const pe_camera* cam, const pe_settings* st, int first, int count,
                    const volatile int32_t* cancel, float* sum, uint32_t* cnt, float* sq, Paths* scratch, size_t capacity,
                    bool timing, Tile tile, const int32_t* pixList = nullptr, size_t nList = 0) {
    const size_t npix = pixList ? nList : static_cast<size_t>(tile.w) * static_cast<size_t>(tile.h);
    if (npix == 0) return PE_OK;
    // unguided waves on the lanes' own state regenerate paths: kStreamFactor × the slots per wave
    const bool regenWaves = !scratch && !d->guide.mode && d->guideKind != 2 && !d->aovTarget && !d->passTarget;
    // regenerating waves keep pe_tuning::wave_slots paths in flight (the lanes hold that many)
    const size_t waveCap = regenWaves ? std::min(d->waveSlots, d->laneSlots) : capacity;
    const size_t pathCap = regenWaves ? waveCap * kStreamFactor : waveCap;
    const int pixChunk = static_cast<int>(std::min(npix, pathCap));
    const int samplesPerWave = static_cast<int>(std::max<size_t>(1, std::min<size_t>(static_cast<size_t>(count), pathCap / pixChunk)));
    WaveSeg base = makeSeg(cam, st);
    // uploaded on the device stream before evStart, which the second lane waits for
    base.filterCdf = filterTable(d, st->filter_type, st->filter_width, ++d->filterClock, d->stream);
    if (!base.filterCdf) {
        setError("pixel filter table upload failed");
        return PE_ERR_CUDA;
    }
    int32_t rc = beginRender(d);
    if (rc) return rc;
    base.tileX = tile.x0;
    base.tileY = tile.y0;
    base.tileW = tile.w;
    base.sum = sum;
    base.cnt = cnt;
    base.sq = sq;
    base.aov = scratch ? nullptr : d->aovTarget;
    base.pass = scratch ? nullptr : d->passTarget;
    base.pixList = pixList;
    base.cryptoObj = scratch ? nullptr : d->cryptoObj;
    base.cryptoMat = scratch ? nullptr : d->cryptoMat;
    base.cryptoFirst = d->cryptoFirst;
    RenderTimer tm;
    tm.timing = timing;
    bool cancelled = false;
    // SD-tree guiding trains over the first 32 samples in chunks of 2, 2, 4, 8, 16 with a
    // refinement after each, then samples from the frozen field (renderer.cpp:476-526)
    const bool sdGuided = d->guideKind == 2 && !scratch;
    if (sdGuided && (rc = sdBeginRender(d, first))) return rc;
    struct ModeReset {
        pe_device* d;
        ~ModeReset() { d->sd.waveMode = 0; }
    } modeReset{d};
    for (int cur = first; cur < first + count && !cancelled;) {
        const int chunkEnd = sdGuided ? sdChunkEnd(d, cur, first + count) : first + count;
        for (int s0 = cur; s0 < chunkEnd && !cancelled; s0 += samplesPerWave) {
            const int ns = std::min(samplesPerWave, chunkEnd - s0);
            for (size_t p0 = 0; p0 < npix; p0 += static_cast<size_t>(pixChunk)) {
                if (cancel && *cancel) {
                    cancelled = true;
                    break;
                }
                // alternate lanes (the no-allocation scratch has one; guided renders keep to lane 0
                // so that each wave's training step lands before the next wave's inference)
                const bool oneLane = scratch || d->guide.mode || sdGuided;
                const int lane = oneLane ? 0 : d->nextLane;
                if (!oneLane) d->nextLane ^= 1;
                Paths& P = scratch ? *scratch : d->lanes[lane].paths;
                if ((rc = segsWritable(d, lane))) return rc;
                WaveSeg& seg = d->lanes[lane].hSegs[0];
                seg = base;
                seg.pixelFirst = static_cast<int>(p0);
                seg.nPix = static_cast<int>(std::min<size_t>(static_cast<size_t>(pixChunk), npix - p0));
                seg.sampleFirst = s0;
                seg.nSamples = ns;
                seg.slotFirst = 0;
                seg.pixFirst = 0;
                if ((rc = runWave(d, lane, P, 1, seg.nPix * ns, seg.nPix, tm))) return rc;
            }
        }
        if (sdGuided && !cancelled && (rc = sdEndChunk(d, chunkEnd - cur))) return rc;
        cur = chunkEnd;
    }
    if ((rc = endRender(d, tm))) return rc;
    if (cancelled) {
        setError("render cancelled");
        return PE_ERR_CANCELLED;
    }
    return PE_OK;
}

// ---- adaptive sampling (renderer.cpp:442-467, 498-500) ------------------------------------------
// Film::relativeError (film.cpp:100-109): the relative standard error of the pixel's mean
// luminance; 1e30 below two samples.
__device__ __forceinline__ float pixelRelError(const float* sum, const uint32_t* cnt, const float* sq, int i) {
    const uint32_t n = cnt[i];
    if (n < 2) return 1e30f;
    const float nf = static_cast<float>(n);
    const float mean = (0.212671f * sum[3 * i + 0] + 0.715160f * sum[3 * i + 1] + 0.072169f * sum[3 * i + 2]) / nf;
    const float meanSq = sq[i] / nf;
    const float var = fmaxf(0.0f, meanSq - mean * mean) * nf / static_cast<float>(n - 1);
    return sqrtf(var / nf) / (fmaxf(mean, 0.0f) + 0.01f);
}

// Warp-aggregated append of the lanes whose `keep` is set (all 32 lanes of the warp call it).
__device__ __forceinline__ void appendPixel(int32_t* list, uint32_t* count, bool keep, int32_t pixel) {
    const unsigned mask = __ballot_sync(0xFFFFFFFFu, keep);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (keep) list[base + __popc(mask & ((1u << lane) - 1u))] = pixel;
}

// Pixels whose accumulated error is below the threshold.
__global__ void kAdaptiveClean(const float* sum, const uint32_t* cnt, const float* sq, int n, float threshold,
                               uint8_t* clean) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        clean[i] = pixelRelError(sum, cnt, sq, i) < threshold ? 1 : 0;
}

// The batch's pixels: all of them, or (with `clean`) those that are not clean together with all
// eight neighbours (edges clamped).  Blocks step over whole blocks of pixels, so every warp runs
// each iteration with all its lanes.
__global__ void kAdaptiveList(const uint8_t* clean, int w, int h, int32_t* list, uint32_t* count) {
    const int n = w * h;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int i = base + static_cast<int>(threadIdx.x);
        bool keep = i < n;
        if (keep && clean) {
            const int x = i % w, y = i / w;
            bool all = true;
            for (int dy = -1; dy <= 1 && all; ++dy)
                for (int dx = -1; dx <= 1 && all; ++dx) {
                    const int nx = min(max(x + dx, 0), w - 1), ny = min(max(y + dy, 0), h - 1);
                    all = clean[ny * w + nx] != 0;
                }
            keep = !all;
        }
        appendPixel(list, count, keep, i);
    }
}

// The listed pixels that go on after a check: those whose error is not yet below the threshold.
__global__ void kAdaptiveStop(const float* sum, const uint32_t* cnt, const float* sq, const int32_t* in, int nIn,
                              float threshold, int32_t* out, uint32_t* count) {
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < nIn; base += stride) {
        const int j = base + static_cast<int>(threadIdx.x);
        const int px = j < nIn ? in[j] : -1;
        appendPixel(out, count, px >= 0 && !(pixelRelError(sum, cnt, sq, px) < threshold), px);
    }
}

// Adaptive render of samples [first, first+count) into the device film, which holds the pixels'
// accumulated samples: pixels that are clean together with their neighbours skip the batch (once
// the film holds minAdaptiveSamples), and after every sample index that is a multiple of 8 (at
// least minAdaptiveSamples, before the batch's end) the pixels whose error fell below the
// threshold stop.  Renderer::renderSamples decides the same per pixel (renderer.cpp:442-467,
// 498-500), so every pixel takes the same samples and the film the same sums.
// With SD-tree guiding (renderer.cpp:413-526 runs both in one renderSamples) each check interval
// is further split at the field's refinements by renderWaves: a pixel's stops depend on its own
// samples only, and each refinement sees the samples of every pixel still rendering, as there.
int32_t renderAdaptive(pe_device* d, const pe_camera* cam, const pe_settings* st, int first, int count,
                       const volatile int32_t* cancel, uint64_t* traced) {
    const int w = st->width, h = st->height;
    const size_t n = static_cast<size_t>(w) * static_cast<size_t>(h);
    if (d->adaptPixels < n) {
        cudaFree(d->adaptList[0]);
        cudaFree(d->adaptList[1]);
        cudaFree(d->adaptClean);
        d->adaptList[0] = d->adaptList[1] = nullptr;
        d->adaptClean = nullptr;
        d->adaptPixels = 0;
        PE_CUDA(cudaMalloc(&d->adaptList[0], n * sizeof(int32_t)));
        PE_CUDA(cudaMalloc(&d->adaptList[1], n * sizeof(int32_t)));
        PE_CUDA(cudaMalloc(&d->adaptClean, n));
        d->adaptPixels = n;
    }
    if (!d->adaptCount) PE_CUDA(cudaMalloc(&d->adaptCount, 2 * sizeof(uint32_t)));
    const float threshold = std::max(1e-4f, st->noise_threshold);
    const int minSpp = std::max(2, st->min_adaptive_samples);
    const int threads = 256;
    auto gridFor = [&](size_t items) {
        return static_cast<int>(std::max<size_t>(1, std::min<size_t>((items + threads - 1) / threads, 148 * 16)));
    };
    cudaStream_t cs = d->stream;
    PE_CUDA(cudaMemsetAsync(d->adaptCount, 0, 2 * sizeof(uint32_t), cs));
    const bool skip = first >= minSpp;
    if (skip)
        kAdaptiveClean<<<gridFor(n), threads, 0, cs>>>(d->fSum, d->fCnt, d->fSq, static_cast<int>(n), threshold,
                                                       d->adaptClean);
    kAdaptiveList<<<gridFor(n), threads, 0, cs>>>(skip ? d->adaptClean : nullptr, w, h, d->adaptList[0], d->adaptCount);
    PE_CUDA(cudaGetLastError());
    uint32_t active = 0;
    PE_CUDA(cudaMemcpyAsync(&active, d->adaptCount, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
    PE_CUDA(cudaStreamSynchronize(cs));
    int cur = first, which = 0;
    const int end = first + count;
    uint64_t done = 0;
    while (cur < end && active > 0) {
        // the next check: the first multiple of 8 after cur that is at least minSpp, before the end
        int e = end;
        for (int k = (cur / 8 + 1) * 8; k < end; k += 8)
            if (k >= minSpp) {
                e = k;
                break;
            }
        const int32_t rc = renderWaves(d, cam, st, cur, e - cur, cancel, d->fSum, d->fCnt, d->fSq, nullptr, d->capacity,
                                       true, Tile{0, 0, w, h}, d->adaptList[which], active);
        if (rc != PE_OK) {
            if (traced) *traced = done;
            return rc;
        }
        done += static_cast<uint64_t>(active) * static_cast<uint64_t>(e - cur);
        cur = e;
        if (cur < end) {
            uint32_t* outCount = d->adaptCount + 1 - which;
            PE_CUDA(cudaMemsetAsync(outCount, 0, sizeof(uint32_t), cs));
            kAdaptiveStop<<<gridFor(active), threads, 0, cs>>>(d->fSum, d->fCnt, d->fSq, d->adaptList[which],
                                                               static_cast<int>(active), threshold,
                                                               d->adaptList[1 - which], outCount);
            PE_CUDA(cudaGetLastError());
            PE_CUDA(cudaMemcpyAsync(&active, outCount, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
            PE_CUDA(cudaStreamSynchronize(cs));
            which = 1 - which;
        }
    }
    if (traced) *traced = done;
    return PE_OK;
}

// WIDE: the traversal the render kernels use (4-wide tree); else the binary tree in the
// reference's visiting order.
template <bool WIDE>
__global__ void kTracePrimary(SceneGPU S, WaveSeg A, int nPix, int32_t* outShape, int32_t* outPrim, float* outT) {
    for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < nPix; pix += gridDim.x * blockDim.x) {
        const int x = pix % A.width, y = pix / A.width;
        Sobol sb;
        sb.pixelHash = pixelHashOf(A.seed, x, y);
        sb.revIndex = rev32(static_cast<uint32_t>(A.sampleFirst));
        sb.dim = 0;
        V3 o, d;
        cameraRay(S.tables, A.filterCdf, A.cam, A.filterWidth, x, y, A.width, A.height, sb, o, d);
        uint32_t a = 0, b = 0;
        const Hit h = WIDE ? traceClosestWide<false>(S, o, d, VIS_CAMERA, 0.0f, 1e30f, a, b)
                           : traceClosest<false>(S, o, d, VIS_CAMERA, 0.0f, 1e30f, a, b);
        if (isMiss(h.prim)) {
            outShape[pix] = -1;
            outPrim[pix] = -1;
            outT[pix] = 0.0f;
        } else {
            int rec = h.prim, shape;
            if (isInstanceHit(h.prim)) {
                const InstGPU& I = S.instances[instanceOfHit(h.prim)];
                rec = I.recBase + localOfHit(h.prim);
                shape = I.shape;
            }
            const float4 e2w = __ldg(&S.tris[3 * rec + 2]);
            const int g = static_cast<int>(__float_as_uint(e2w.w));
            if (!isInstanceHit(h.prim)) shape = __ldg(&S.triVerts[g]).w;
            outShape[pix] = shape;
            outPrim[pix] = g - static_cast<int>(S.shapes[shape].firstTri);
            outT[pix] = h.t;
        }
    }
}

// Ray queries of pe_device_trace_rays: closest hit (binary tree in the reference's visiting
// order, or the 4-wide tree) or any hit (4-wide), at a shutter time.
template <int MODE>
__global__ void kTraceRays(SceneGPU S, const float* o, const float* dir, const float* tMax, int n, uint32_t mask,
                           float time, int32_t* outShape, int32_t* outPrim, float* outT) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V3 ro = mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), rd = mk(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        uint32_t a = 0, b = 0;
        if (MODE == 2) {
            outShape[i] = traceAnyWide<false>(S, ro, rd, mask, 0.0f, tMax[i], a, b, time) ? 1 : 0;
            outPrim[i] = -1;
            outT[i] = 0.0f;
            continue;
        }
        const Hit h = MODE == 1 ? traceClosestWide<false>(S, ro, rd, mask, 0.0f, tMax[i], a, b, nullptr, time)
                                : traceClosest<false>(S, ro, rd, mask, 0.0f, tMax[i], a, b, time);
        if (isMiss(h.prim)) {
            outShape[i] = -1;
            outPrim[i] = -1;
            outT[i] = 0.0f;
            continue;
        }
        int rec = h.prim, shape = -1;
        if (isInstanceHit(h.prim)) {
            const InstGPU& I = S.instances[instanceOfHit(h.prim)];
            rec = I.recBase + localOfHit(h.prim);
            shape = I.shape;
        }
        const int g = static_cast<int>(__float_as_uint(__ldg(&S.tris[3 * rec + 2]).w));
        if (!isInstanceHit(h.prim)) shape = __ldg(&S.triVerts[g]).w;
        outShape[i] = shape;
        outPrim[i] = g - static_cast<int>(S.shapes[shape].firstTri);
        outT[i] = h.t;
    }
}

__global__ void kSobol(const TablesGPU* T, uint64_t seed, const int32_t* px, const int32_t* py, const int32_t* idx, int n,
                       int nd, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Sobol sb;
        sb.pixelHash = pixelHashOf(seed, px[i], py[i]);
        sb.revIndex = rev32(static_cast<uint32_t>(idx[i]));
        sb.dim = 0;
        for (int k = 0; k < nd; ++k) {
            const V2 v = get2D(T, sb);
            out[(static_cast<size_t>(i) * nd + k) * 2 + 0] = v.x;
            out[(static_cast<size_t>(i) * nd + k) * 2 + 1] = v.y;
        }
    }
}

__global__ void kBsdfProbe(SceneGPU S, int material, const pe_bsdf_query* q, int n, pe_bsdf_result* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const MatGPU& m = S.materials[material];
        ShadePoint sp;
        sp.uv = mk2(0.0f, 0.0f);
        sp.textures = nullptr;
        sp.p = m3f(q[i].point);
        sp.n = m3f(q[i].normal);
        sp.ng = m3f(q[i].ng);
        sp.tangent = m3f(q[i].tangent);
        sp.frontFace = q[i].front_face != 0;
        sp.wavelength = q[i].wavelength;
        pe_bsdf_result r;
        memset(&r, 0, sizeof(r));
        float pdf = 0.0f;
        const V3 f = bsdfEvalPdf(S.tables, m, m3f(q[i].wo), m3f(q[i].wi), sp, pdf, nullptr);
        r.f[0] = f.x;
        r.f[1] = f.y;
        r.f[2] = f.z;
        r.pdf = pdf;
        BsdfSample bs;
        bs.wi = mk(0.0f);
        bs.f = mk(0.0f);
        bs.pdf = 0.0f;
        bs.delta = bs.passThrough = bs.subsurface = false;
        bs.weight = mk(0.0f);
        r.sampled = bsdfSample(S.tables, m, m3f(q[i].wo), sp, q[i].uc, mk2(q[i].u[0], q[i].u[1]), bs) ? 1 : 0;
        r.wi[0] = bs.wi.x;
        r.wi[1] = bs.wi.y;
        r.wi[2] = bs.wi.z;
        r.sf[0] = bs.f.x;
        r.sf[1] = bs.f.y;
        r.sf[2] = bs.f.z;
        r.spdf = bs.pdf;
        r.delta = bs.delta;
        r.pass_through = bs.passThrough;
        r.subsurface = bs.subsurface;
        r.weight[0] = bs.weight.x;
        r.weight[1] = bs.weight.y;
        r.weight[2] = bs.weight.z;
        out[i] = r;
    }
}

} // namespace pe_dev

namespace pe_dev {

int32_t uploadScene(pe_device* d, const pe_scene* s, SceneGPU& G, std::vector<DevBuf>& bufs) {
    G = SceneGPU{};
    const HostBuild& B = s->build;
    int32_t rc = 0;
    if ((rc = upload(d, bufs, G.nodes, B.nodes)) || (rc = upload(d, bufs, G.wide, B.wide)) ||
        (rc = upload(d, bufs, G.instances, B.instances)) ||
        (rc = upload(d, bufs, G.tris, B.tris)) ||
        (rc = upload(d, bufs, G.triVerts, B.triVerts)) || (rc = upload(d, bufs, G.pos, B.pos)) ||
        (rc = upload(d, bufs, G.nrm, B.nrm)) || (rc = upload(d, bufs, G.uv, B.uv)) ||
        (rc = upload(d, bufs, G.shapes, B.shapes)) || (rc = upload(d, bufs, G.materials, B.materials)) ||
        (rc = upload(d, bufs, G.lights, B.lights)) || (rc = upload(d, bufs, G.lightNodes, B.lightNodes)) ||
        (rc = upload(d, bufs, G.topSlot, B.topSlot)) || (rc = upload(d, bufs, G.trail, B.trail)) ||
        (rc = upload(d, bufs, G.trailDepth, B.trailDepth)))
        return rc;
    G.rootIsLeaf = B.rootIsLeaf;
    G.rootFirst = B.rootFirst;
    G.rootCount = B.rootCount;
    G.nNodes = static_cast<int32_t>(B.nodes.size() / 4);
    for (int i = 0; i < 3; ++i) {
        G.rootMin[i] = B.rootMin[i];
        G.rootMax[i] = B.rootMax[i];
    }
    G.nTris = static_cast<uint32_t>(B.triVerts.size());
    G.nShapes = static_cast<int32_t>(B.shapes.size());
    G.nLights = static_cast<int32_t>(B.lights.size());
    G.lightMode = B.lightMode;
    G.lightCount = B.lightCount;
    G.nInfinite = static_cast<int32_t>(B.infinite.size());
    for (size_t i = 0; i < B.infinite.size() && i < static_cast<size_t>(kMaxInfinite); ++i) G.infinite[i] = B.infinite[i];
    G.nLightNodes = static_cast<int32_t>(B.lightNodes.size());
    // environment (the MIS-compensated distribution drives sampling and pdfLi)
    const HostEnv& e = s->env;
    EnvGPU& E = G.env;
    E.present = e.present ? 1 : 0;
    E.width = e.width;
    E.height = e.height;
    E.hasImage = e.hasImage ? 1 : 0;
    E.rotation = e.rotation;
    E.intensity = e.intensity;
    E.meanLuminance = e.meanLuminance;
    E.sunPdfWeight = e.sunPdfWeight;
    E.sunDir[0] = e.sunDir.x;
    E.sunDir[1] = e.sunDir.y;
    E.sunDir[2] = e.sunDir.z;
    E.sunCosMax = e.sunCosMax;
    E.sunRadiance[0] = e.sunRadiance.x;
    E.sunRadiance[1] = e.sunRadiance.y;
    E.sunRadiance[2] = e.sunRadiance.z;
    E.funcInt = e.misInt;
    E.valid = e.misValid ? 1 : 0;
    if ((rc = upload(d, bufs, E.image, e.image)) || (rc = upload(d, bufs, E.func, e.misFunc)) ||
        (rc = upload(d, bufs, E.marginalCdf, e.misMarg)) || (rc = upload(d, bufs, E.condCdf, e.misCond)))
        return rc;
    // the shadow catcher samples the environment without MIS compensation (sampleLiFull)
    G.envFull = E;
    if (B.catcherShape >= 0) {
        EnvGPU& F = G.envFull;
        F.funcInt = e.fullInt;
        F.valid = e.fullValid ? 1 : 0;
        if ((rc = upload(d, bufs, F.func, e.fullFunc)) || (rc = upload(d, bufs, F.marginalCdf, e.fullMarg)) ||
            (rc = upload(d, bufs, F.condCdf, e.fullCond)))
            return rc;
    }
    G.tables = d->dTables;
    G.bgMode = s->bgMode;
    for (int i = 0; i < 3; ++i) G.bgColor[i] = s->bgColor[i];
    G.hasShadowTransmitters = B.hasShadowTransmitters ? 1 : 0;
    G.hasVolumes = B.hasVolumes ? 1 : 0;
    G.hasSubsurface = B.hasSubsurface ? 1 : 0;
    G.exitMaterial = B.exitMaterial;
    G.catcherShape = B.catcherShape;
    G.hasLightLinks = B.hasLightLinks;
    G.hasShadowLinks = B.hasShadowLinks;
    if (!B.links.empty() && (rc = upload(d, bufs, G.links, B.links))) return rc;
    // image textures: the texels of each, then the table of them
    G.textures = nullptr;
    G.hasMips = 0;
    if (!s->textures.empty()) {
        std::vector<TexGPU> tex(s->textures.size());
        G.hasMips = 0;
        for (size_t i = 0; i < s->textures.size(); ++i) {
            const pe_scene::Texture& src = s->textures[i];
            std::vector<float> all = src.texels;
            std::memset(&tex[i], 0, sizeof(TexGPU));
            tex[i].width = src.width;
            tex[i].height = src.height;
            tex[i].levels = 1;
            tex[i].levelW[0] = src.width;
            tex[i].levelH[0] = src.height;
            for (size_t l = 0; l < src.mips.size() && l + 1 < static_cast<size_t>(kMaxMipLevels); ++l) {
                const int k = static_cast<int>(l) + 1;
                tex[i].levelOffset[k] = static_cast<int32_t>(all.size());
                tex[i].levelW[k] = src.mipW[l];
                tex[i].levelH[k] = src.mipH[l];
                all.insert(all.end(), src.mips[l].begin(), src.mips[l].end());
                tex[i].levels = k + 1;
            }
            if (tex[i].levels > 1) G.hasMips = 1;
            const float* texels = nullptr;
            if ((rc = upload(d, bufs, texels, all))) return rc;
            tex[i].texels = texels;
        }
        if ((rc = upload(d, bufs, G.textures, tex))) return rc;
    }
    G.nTextures = static_cast<int32_t>(s->textures.size());
    G.nInstances = static_cast<int32_t>(B.instances.size());
    // moving instances: null without, which also keeps the kernels from reading path times
    if (!B.motions.empty() && (rc = upload(d, bufs, G.motions, B.motions))) return rc;
    G.leanShading = leanShadingOf(G, B.materials);
    G.materialTypes = 0;
    for (const MatGPU& m : B.materials) G.materialTypes |= 1 << m.type;
    G.nLightGroups = static_cast<int32_t>(B.groupNames.size());
    G.envGroup = B.envGroup;
    if (!B.lightGroup.empty() && (rc = upload(d, bufs, G.lightGroup, B.lightGroup))) return rc;
    if ((rc = upload(d, bufs, G.idColor, B.idColor))) return rc;
    d->lightGroups = G.nLightGroups;
    PE_CUDA(cudaStreamSynchronize(d->stream));
    return PE_OK;
}


} // namespace pe_dev

extern "C" {


int32_t pe_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

pe_device* pe_device_create(int32_t ordinal, char* err, size_t errLen) {
    auto fail = [&](const std::string& m) -> pe_device* {
        setError(m);
        if (err && errLen > 0) {
            std::strncpy(err, m.c_str(), errLen - 1);
            err[errLen - 1] = '\0';
        }
        return nullptr;
    };
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaMsg(e) : "count 0"));
    if (ordinal < 0 || ordinal >= n) return fail("CUDA ordinal out of range");
    pe_device* d = new (std::nothrow) pe_device();
    if (!d) return fail("host out of memory");
    d->ordinal = ordinal;
    if ((e = cudaSetDevice(ordinal)) != cudaSuccess) {
        delete d;
        return fail(std::string("cudaSetDevice: ") + cudaMsg(e));
    }
    cudaGetDeviceProperties(&d->prop, ordinal);
    if (d->prop.major < 10) {
        const std::string msg = "device " + std::string(d->prop.name) + " is not sm_100 class; this build targets sm_100a only";
        delete d;
        return fail(msg);
    }
    if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&d->evStart) != cudaSuccess || cudaEventCreate(&d->evStop) != cudaSuccess ||
        cudaEventCreate(&d->evT0) != cudaSuccess || cudaEventCreate(&d->evT1) != cudaSuccess ||
        cudaMalloc(&d->dTables, sizeof(TablesGPU)) != cudaSuccess ||
        cudaMalloc(&d->dStats, 8 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&d->dFilters, static_cast<size_t>(kFilterSlots) * (kFilterBins + 1) * sizeof(float)) != cudaSuccess ||
        cudaEventCreateWithFlags(&d->evFilm, cudaEventDisableTiming) != cudaSuccess) {
        pe_device_destroy(d);
        return fail("device initialisation failed");
    }
    for (int l = 0; l < 2; ++l) {
        WaveLane& ln = d->lanes[l];
        if ((l == 0 ? (ln.stream = d->stream, cudaSuccess) : cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking)) !=
                cudaSuccess ||
            cudaMalloc(&ln.dSegs, kMaxSegs * sizeof(WaveSeg)) != cudaSuccess ||
            cudaMallocHost(&ln.hSegs, kMaxSegs * sizeof(WaveSeg)) != cudaSuccess ||
            cudaMallocHost(&ln.hCounters, 32 * sizeof(uint32_t)) != cudaSuccess ||
            cudaEventCreateWithFlags(&ln.evSegs, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&ln.evDone) != cudaSuccess) {
            pe_device_destroy(d);
            return fail("device initialisation failed");
        }
    }
    d->hTables = staticTables();
    cudaMemcpy(d->dTables, &d->hTables, sizeof(TablesGPU), cudaMemcpyHostToDevice);
    int b = 0;
    const int sm = d->prop.multiProcessorCount;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kIntersect<false>, 128, 0);
    d->blocksIntersect = sm * std::max(1, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kShade<false>, 128, 0);
    d->blocksShade = sm * std::max(1, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kShadow<false>, 128, 0);
    d->blocksShadow = sm * std::max(1, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kTail<true, false>, kTailBlock, 0);
    d->blocksTail = sm * std::max(1, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kTailLockstep<false>, kTailLockstepBlock, 0);
    d->blocksTailLockstep[0] = sm * std::max(1, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kTailLockstep<true>, kTailLockstepBlock, 0);
    d->blocksTailLockstep[1] = sm * std::max(1, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kShadow<false, true>, 128, 0);
    d->blocksShadowAny = sm * std::max(1, b);
    auto occ = [&](auto kernel, int threads) {
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0);
        return sm * std::max(1, nb);
    };
    d->blocksShadeKey[0][0] = occ(kShadeKey<false, 0>, 128);
    d->blocksShadeKey[0][1] = occ(kShadeKey<false, 1>, 128);
    d->blocksShadeKey[0][2] = occ(kShadeKey<false, 2>, 128);
    d->blocksShadeKey[0][3] = occ(kShadeKey<false, 3>, 128);
    d->blocksShadeKey[0][4] = occ(kShadeKey<false, 4>, 128);
    d->blocksShadeKey[1][0] = occ(kShadeKey<false, 0, 4>, 128);
    d->blocksShadeKey[1][1] = occ(kShadeKey<false, 1, 4>, 128);
    d->blocksShadeKey[1][2] = occ(kShadeKey<false, 2, 4>, 128);
    d->blocksShadeKey[1][3] = occ(kShadeKey<false, 3, 4>, 128);
    d->blocksShadeKey[1][4] = occ(kShadeKey<false, 4, 4>, 128);
    d->blocksShadeKey[2][0] = occ(kShadeKey<false, 0, 5>, 128);
    d->blocksShadeKey[2][1] = occ(kShadeKey<false, 1, 5>, 128);
    d->blocksShadeKey[2][2] = occ(kShadeKey<false, 2, 5>, 128);
    d->blocksShadeKey[2][3] = occ(kShadeKey<false, 3, 5>, 128);
    d->blocksShadeKey[2][4] = occ(kShadeKey<false, 4, 5>, 128);
    d->blocksIntersectMode[TRACE_BINARY] = occ(kIntersect<false, TRACE_BINARY>, 128);
    d->blocksIntersectMode[TRACE_WIDE] = occ(kIntersect<false, TRACE_WIDE>, 128);
    d->blocksIntersectMode[TRACE_WIDE_SMEM8] = occ(kIntersect<false, TRACE_WIDE_SMEM8>, 128);
    d->blocksIntersectMode[TRACE_WIDE_SMEM16] = occ(kIntersect<false, TRACE_WIDE_SMEM16>, 128);
    d->blocksIntersectMode[TRACE_WIDE_REG4] = occ(kIntersect<false, TRACE_WIDE_REG4>, 128);
    d->blocksIntersectMode[TRACE_WIDE_REG8] = occ(kIntersect<false, TRACE_WIDE_REG8>, 128);
    d->blocksShadowAnyWindow = occ(kShadow<false, true, 4>, 128);
    d->blocksIntersectMode[TRACE_WIDE_OCC8] = occ(kIntersect<false, TRACE_WIDE_OCC8>, 128);
    d->blocksIntersectMode[TRACE_WIDE_SMEM8_OCC8] = occ(kIntersect<false, TRACE_WIDE_SMEM8_OCC8>, 128);
    d->blocksIntersectMode[TRACE_WIDE_SMEM16_OCC8] = occ(kIntersect<false, TRACE_WIDE_SMEM16_OCC8>, 128);
    d->blocksIntersectMode[TRACE_WIDE_SPEC_OCC8] = occ(kIntersect<false, TRACE_WIDE_SPEC_OCC8>, 128);
    d->blocksShadowAnyOcc8 = occ(kShadow<false, true, 0, 8>, 128);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
        pe_device_destroy(d);
        return fail(std::string("kernel image not loadable on this device: ") + cudaMsg(le));
    }
    // Device address of the no-allocation scratch on this device, taken once here with the
    // device current (a host-side use of the array's name would not be a device address).
    const cudaError_t se = cudaGetSymbolAddress(reinterpret_cast<void**>(&d->noAllocBase), g_noAllocScratch);
    if (se != cudaSuccess) {
        d->noAllocBase = nullptr;
        d->noAllocError = std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaMsg(se);
        cudaGetLastError();
    }
    return d;
}

void pe_device_destroy(pe_device* d) {
    if (!d) return;
    cudaSetDevice(d->ordinal);
    if (d->stream) cudaStreamSynchronize(d->stream);
    if (d->lanes[1].stream) cudaStreamSynchronize(d->lanes[1].stream);
    freeList(d->sceneBufs);
    for (int l = 0; l < 2; ++l) {
        WaveLane& ln = d->lanes[l];
        freeList(ln.bufs);
        freeList(ln.aovBufs);
        freeList(ln.passBufs);
        cudaFree(ln.dSegs);
        if (ln.hSegs) cudaFreeHost(ln.hSegs);
        if (ln.hCounters) cudaFreeHost(ln.hCounters);
        if (ln.evSegs) cudaEventDestroy(ln.evSegs);
        if (ln.evDone) cudaEventDestroy(ln.evDone);
        if (l == 1 && ln.stream) cudaStreamDestroy(ln.stream);
    }
    if (d->evFilm) cudaEventDestroy(d->evFilm);
    cudaFree(d->aovFilm);
    cudaFree(d->passFilm);
    cudaFree(d->adaptList[0]);
    cudaFree(d->adaptList[1]);
    cudaFree(d->adaptClean);
    cudaFree(d->adaptCount);
    cudaFree(d->fSum);
    cudaFree(d->fCnt);
    cudaFree(d->fSq);
    cudaFree(d->dTables);
    cudaFree(d->dStats);
    cudaFree(d->dFilters);
    if (d->stage) cudaFreeHost(d->stage);
    for (cudaEvent_t e : d->evPool) cudaEventDestroy(e);
    if (d->evStart) cudaEventDestroy(d->evStart);
    if (d->evT0) cudaEventDestroy(d->evT0);
    if (d->evT1) cudaEventDestroy(d->evT1);
    if (d->evStop) cudaEventDestroy(d->evStop);
    if (d->stream) cudaStreamDestroy(d->stream);
    delete d;
}

int32_t pe_device_info_get(pe_device* d, pe_device_info* out) {
    if (!d || !out) {
        setError("pe_device_info_get: null argument");
        return PE_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    std::strncpy(out->name, d->prop.name, sizeof(out->name) - 1);
    out->memory_bytes = d->prop.totalGlobalMem;
    out->compute_major = d->prop.major;
    out->compute_minor = d->prop.minor;
    out->sm_count = d->prop.multiProcessorCount;
    out->usable = 1;
    cudaDeviceGetPCIBusId(out->pci_bus_id, sizeof(out->pci_bus_id), d->ordinal);
    return PE_OK;
}

int32_t pe_device_set_scene(pe_device* d, const pe_scene* s) {
    if (!d || !s) {
        setError("pe_device_set_scene: null argument");
        return PE_ERR_INVALID;
    }
    if (!s->built) {
        setError("pe_device_set_scene: scene not built (call pe_scene_build)");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    freeList(d->sceneBufs);
    d->hasScene = false;
    SceneGPU G{};
    const int32_t rc = uploadScene(d, s, G, d->sceneBufs);
    if (rc) return rc;
    d->scene = G;
    d->hasScene = true;
    d->sceneSrc = s;
    d->sceneVersion = s->version;
    d->sceneMaterials = s->build.materials.size();
    d->sceneLightNodes = s->build.lightNodes.size();
    ++d->sceneSerial;
    return PE_OK;
}

// RenderDevice::updateScene(scene, SceneUpdateKind::Lights): the lights, their emissive quads'
// materials and the light sampler of the scene already set are copied again, when the sampler
// keeps its shape (same node count and mode); else PE_ERR_LIMIT and the caller sets the scene.
int32_t pe_device_update_lights(pe_device* d, const pe_scene* s) {
    if (!d || !s) {
        setError("pe_device_update_lights: null argument");
        return PE_ERR_INVALID;
    }
    const HostBuild& B = s->build;
    if (!d->hasScene || d->sceneSrc != s || d->sceneVersion != s->version || !s->built ||
        B.materials.size() != d->sceneMaterials || B.lights.size() != static_cast<size_t>(d->scene.nLights)) {
        setError("pe_device_update_lights: the device holds another build of the scene (call pe_device_set_scene)");
        return PE_ERR_INVALID;
    }
    if (B.lightNodes.size() != d->sceneLightNodes || B.lightMode != d->scene.lightMode ||
        B.infinite.size() > static_cast<size_t>(kMaxInfinite)) {
        setError("pe_device_update_lights: the light sampler changed shape (call pe_device_set_scene)");
        return PE_ERR_LIMIT;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    PE_CUDA(cudaStreamSynchronize(d->lanes[1].stream));
    SceneGPU& G = d->scene;
    auto put = [&](const void* dst, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, d->stream) : cudaSuccess;
    };
    PE_CUDA(put(G.lights, B.lights.data(), B.lights.size() * sizeof(LightGPU)));
    PE_CUDA(put(G.materials, B.materials.data(), B.materials.size() * sizeof(MatGPU)));
    if (G.lightNodes) PE_CUDA(put(G.lightNodes, B.lightNodes.data(), B.lightNodes.size() * sizeof(LightNodeGPU)));
    if (G.topSlot) PE_CUDA(put(G.topSlot, B.topSlot.data(), B.topSlot.size() * sizeof(int16_t)));
    if (G.trail) PE_CUDA(put(G.trail, B.trail.data(), B.trail.size() * sizeof(unsigned long long)));
    if (G.trailDepth) PE_CUDA(put(G.trailDepth, B.trailDepth.data(), B.trailDepth.size() * sizeof(uint8_t)));
    G.nInfinite = static_cast<int32_t>(B.infinite.size());
    for (size_t i = 0; i < B.infinite.size(); ++i) G.infinite[i] = B.infinite[i];
    PE_CUDA(cudaStreamSynchronize(d->stream));
    ++d->sceneSerial;
    return PE_OK;
}

// RenderDevice::updateScene(scene, SceneUpdateKind::Materials) (render_device.h:77-79): the
// material table of the scene already set is copied again; its geometry, BVH, lights and
// textures stay on the device.
int32_t pe_device_update_materials(pe_device* d, const pe_scene* s) {
    if (!d || !s) {
        setError("pe_device_update_materials: null argument");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene || d->sceneSrc != s || d->sceneVersion != s->version || !s->built ||
        s->build.materials.size() != d->sceneMaterials) {
        setError("pe_device_update_materials: the device holds another build of the scene (call pe_device_set_scene)");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    PE_CUDA(cudaStreamSynchronize(d->lanes[1].stream));
    PE_CUDA(cudaMemcpyAsync(const_cast<MatGPU*>(d->scene.materials), s->build.materials.data(),
                            s->build.materials.size() * sizeof(MatGPU), cudaMemcpyHostToDevice, d->stream));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    d->scene.leanShading = leanShadingOf(d->scene, s->build.materials);
    ++d->sceneSerial;
    return PE_OK;
}

// SceneUpdateKind::Transforms: the top-level tree refitted on the host (pe_scene_refit) and only
// its nodes, the instance table and the root box sent; BLASes stay as they are on the device.
int32_t pe_device_update_transforms(pe_device* d, pe_scene* s) {
    if (!d || !s) {
        setError("pe_device_update_transforms: null argument");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene || d->sceneSrc != s || d->sceneVersion != s->version || !s->built) {
        setError("pe_device_update_transforms: the device holds another build of the scene (call pe_device_set_scene)");
        return PE_ERR_INVALID;
    }
    int32_t rc = pe_scene_refit(s);
    if (rc) return rc;
    const HostBuild& B = s->build;
    PE_CUDA(cudaSetDevice(d->ordinal));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    PE_CUDA(cudaStreamSynchronize(d->lanes[1].stream));
    if (B.tlasInterior > 0)
        PE_CUDA(cudaMemcpyAsync(const_cast<float4*>(d->scene.nodes), B.nodes.data(),
                                static_cast<size_t>(B.tlasInterior) * 4 * sizeof(float4), cudaMemcpyHostToDevice, d->stream));
    if (!B.tlasWideKids.empty())
        PE_CUDA(cudaMemcpyAsync(const_cast<float4*>(d->scene.wide), B.wide.data(),
                                B.tlasWideKids.size() * 8 * sizeof(float4), cudaMemcpyHostToDevice, d->stream));
    if (!B.instances.empty())
        PE_CUDA(cudaMemcpyAsync(const_cast<InstGPU*>(d->scene.instances), B.instances.data(),
                                B.instances.size() * sizeof(InstGPU), cudaMemcpyHostToDevice, d->stream));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    for (int k = 0; k < 3; ++k) {
        d->scene.rootMin[k] = B.rootMin[k];
        d->scene.rootMax[k] = B.rootMax[k];
    }
    ++d->sceneSerial;
    return PE_OK;
}

int32_t pe_device_has_scene(pe_device* d) { return d && d->hasScene ? 1 : 0; }

int32_t pe_device_render_resident(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                                  const volatile int32_t* cancel) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("render before set_scene");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    if (count <= 0) return PE_OK;
    PE_CUDA(cudaSetDevice(d->ordinal));
    if ((rc = ensureFilm(d, st->width, st->height))) return rc;
    if ((rc = ensureCapacity(d, kWaveSlots))) return rc;
    if (st->adaptive_sampling) return renderAdaptive(d, cam, st, first, count, cancel, nullptr);
    return renderWaves(d, cam, st, first, count, cancel, d->fSum, d->fCnt, d->fSq, nullptr, d->capacity, true,
                       Tile{0, 0, st->width, st->height});
}

int32_t pe_device_film_clear(pe_device* d) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (!d->fSum) return PE_OK;
    const size_t n = static_cast<size_t>(d->filmW) * static_cast<size_t>(d->filmH);
    PE_CUDA(cudaMemsetAsync(d->fSum, 0, n * 3 * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(d->fCnt, 0, n * sizeof(uint32_t), d->stream));
    PE_CUDA(cudaMemsetAsync(d->fSq, 0, n * sizeof(float), d->stream));
    return PE_OK;
}

int32_t pe_device_film_read(pe_device* d, float* sum, uint32_t* cnt, float* sq) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (!d->fSum) {
        setError("no resident film");
        return PE_ERR_INVALID;
    }
    const size_t n = static_cast<size_t>(d->filmW) * static_cast<size_t>(d->filmH);
    if (sum) PE_CUDA(cudaMemcpyAsync(sum, d->fSum, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
    if (cnt) PE_CUDA(cudaMemcpyAsync(cnt, d->fCnt, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, d->stream));
    if (sq) PE_CUDA(cudaMemcpyAsync(sq, d->fSq, n * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
    PE_CUDA(cudaStreamSynchronize(d->stream));
    return PE_OK;
}

// Adds a device film block (5 floats per pixel: sum 3n, count n, sum of squares n) to a Film's
// host arrays as Film::addBatch does (film.cpp:119-137); a null array is skipped.
static void mergeFilm(const float* fs, size_t n, float* sum, uint32_t* cnt, float* sq) {
    const uint32_t* fc = reinterpret_cast<const uint32_t*>(fs + 3 * n);
    const float* fq = fs + 4 * n;
    if (sum)
        for (size_t i = 0; i < 3 * n; ++i) sum[i] += fs[i];
    if (cnt)
        for (size_t i = 0; i < n; ++i) cnt[i] += fc[i];
    if (sq)
        for (size_t i = 0; i < n; ++i) sq[i] += fq[i];
}

// RenderDevice::render with AOV and / or pass targets: per-slot outputs on both lanes, zeroed
// device films, the beauty render, then every film read back and merged into the caller's.
static int32_t renderTargets(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                             const volatile int32_t* cancel, float* sumRgb, uint32_t* sampleCount, float* sumLumSq,
                             const pe_aov_films* aovs, const pe_pass_films* passes, uint64_t* traced) {
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    if (count <= 0) return PE_OK;
    if (!d->hasScene) {
        setError("render before set_scene");
        return PE_ERR_NO_SCENE;
    }
    if (passes && passes->n_groups != d->lightGroups) {
        setError("pe_device_render_passes: " + std::to_string(passes->n_groups) + " light-group films for a scene with " +
                 std::to_string(d->lightGroups) + " light groups");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    if ((rc = ensureCapacity(d, kWaveSlots))) return rc;
    const size_t n = static_cast<size_t>(st->width) * static_cast<size_t>(st->height);
    if (aovs) {
        for (WaveLane& ln : d->lanes)
            if (!ln.aovA) {
                if ((rc = devAlloc(ln.aovBufs, ln.aovA, d->capacity)) || (rc = devAlloc(ln.aovBufs, ln.aovN, d->capacity))) {
                    freeList(ln.aovBufs);
                    ln.aovA = ln.aovN = nullptr;
                    return rc;
                }
            }
        if (d->aovFilmPixels < n) {
            cudaFree(d->aovFilm);
            d->aovFilm = nullptr;
            d->aovFilmPixels = 0;
            PE_CUDA(cudaMalloc(&d->aovFilm, n * 15 * sizeof(float)));
            d->aovFilmPixels = n;
        }
        PE_CUDA(cudaMemsetAsync(d->aovFilm, 0, n * 15 * sizeof(float), d->stream));
    }
    const int32_t stride = PASS_GROUPS + d->lightGroups;
    const size_t passFloats = static_cast<size_t>(PFILM_GROUPS + d->lightGroups) * 5 * n;
    if (passes) {
        for (WaveLane& ln : d->lanes)
            if (!ln.pass || ln.passStride != stride) {
                freeList(ln.passBufs);
                ln.pass = ln.shPass = nullptr;
                ln.passStride = 0;
                if ((rc = devAlloc(ln.passBufs, ln.pass, d->capacity * static_cast<size_t>(stride))) ||
                    (rc = devAlloc(ln.passBufs, ln.shPass, d->capacity * 3))) {
                    freeList(ln.passBufs);
                    ln.pass = ln.shPass = nullptr;
                    return rc;
                }
                ln.passStride = stride;
            }
        if (d->passFilmFloats < passFloats) {
            cudaFree(d->passFilm);
            d->passFilm = nullptr;
            d->passFilmFloats = 0;
            PE_CUDA(cudaMalloc(&d->passFilm, passFloats * sizeof(float)));
            d->passFilmFloats = passFloats;
        }
        PE_CUDA(cudaMemsetAsync(d->passFilm, 0, passFloats * sizeof(float), d->stream));
    }
    // per-sample Cryptomatte ids: a device buffer for the call, freed on return
    const size_t cryptoFloats = static_cast<size_t>(count) * n;
    float* cryptoBuf = nullptr;
    if (passes && passes->crypto_object && passes->crypto_material) {
        PE_CUDA(cudaMalloc(&cryptoBuf, 2 * cryptoFloats * sizeof(float)));
        PE_CUDA(cudaMemsetAsync(cryptoBuf, 0, 2 * cryptoFloats * sizeof(float), d->stream));
    }
    d->aovTarget = aovs ? d->aovFilm : nullptr;
    d->passTarget = passes ? d->passFilm : nullptr;
    d->passStride = passes ? stride : 0;
    d->cryptoObj = cryptoBuf;
    d->cryptoMat = cryptoBuf ? cryptoBuf + cryptoFloats : nullptr;
    d->cryptoFirst = first;
    struct Reset {
        pe_device* d;
        float* buf;
        ~Reset() {
            d->aovTarget = nullptr;
            d->passTarget = nullptr;
            d->passStride = 0;
            d->cryptoObj = d->cryptoMat = nullptr;
            if (buf) cudaFree(buf);
        }
    } reset{d, cryptoBuf};
    rc = pe_device_render(d, cam, st, first, count, cancel, sumRgb, sampleCount, sumLumSq, traced);
    if (rc != PE_OK && rc != PE_ERR_CANCELLED) return rc;
    if (aovs) {
        std::vector<float> h(n * 15);
        PE_CUDA(cudaMemcpyAsync(h.data(), d->aovFilm, n * 15 * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
        PE_CUDA(cudaStreamSynchronize(d->stream));
        mergeFilm(h.data(), n, aovs->albedo_sum, aovs->albedo_count, aovs->albedo_sum_sq);
        mergeFilm(h.data() + 5 * n, n, aovs->normal_sum, aovs->normal_count, nullptr);
        mergeFilm(h.data() + 10 * n, n, aovs->alpha_sum, aovs->alpha_count, aovs->alpha_sum_sq);
    }
    if (passes) {
        std::vector<float> h(passFloats);
        PE_CUDA(cudaMemcpyAsync(h.data(), d->passFilm, passFloats * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
        PE_CUDA(cudaStreamSynchronize(d->stream));
        const pe_film_arrays* films[PFILM_GROUPS + PE_MAX_LIGHT_GROUPS];
        for (int k = 0; k < PE_LIGHT_PASSES; ++k) films[k] = &passes->light[k];
        films[PFILM_DEPTH] = &passes->depth;
        films[PFILM_POSITION] = &passes->position;
        films[PFILM_OBJECT] = &passes->object_id;
        films[PFILM_MATERIAL] = &passes->material_id;
        for (int g = 0; g < d->lightGroups; ++g) films[PFILM_GROUPS + g] = &passes->groups[g];
        for (int f = 0; f < PFILM_GROUPS + d->lightGroups; ++f)
            mergeFilm(h.data() + static_cast<size_t>(f) * 5 * n, n, films[f]->sum, films[f]->count,
                      f == PFILM_POSITION ? nullptr : films[f]->sum_sq);
        if (cryptoBuf) {
            PE_CUDA(cudaMemcpyAsync(passes->crypto_object, cryptoBuf, cryptoFloats * sizeof(float),
                                    cudaMemcpyDeviceToHost, d->stream));
            PE_CUDA(cudaMemcpyAsync(passes->crypto_material, cryptoBuf + cryptoFloats, cryptoFloats * sizeof(float),
                                    cudaMemcpyDeviceToHost, d->stream));
            PE_CUDA(cudaStreamSynchronize(d->stream));
        }
    }
    return rc;
}

int32_t pe_device_render_aovs(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                              const volatile int32_t* cancel, float* sumRgb, uint32_t* sampleCount, float* sumLumSq,
                              const pe_aov_films* aovs, uint64_t* traced) {
    if (!d || !aovs) {
        setError("pe_device_render_aovs: null argument");
        return PE_ERR_INVALID;
    }
    return renderTargets(d, cam, st, first, count, cancel, sumRgb, sampleCount, sumLumSq, aovs, nullptr, traced);
}

int32_t pe_device_render_passes(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first,
                                int32_t count, const volatile int32_t* cancel, float* sumRgb, uint32_t* sampleCount,
                                float* sumLumSq, const pe_aov_films* aovs, const pe_pass_films* passes,
                                uint64_t* traced) {
    if (!d || !passes) {
        setError("pe_device_render_passes: null argument");
        return PE_ERR_INVALID;
    }
    return renderTargets(d, cam, st, first, count, cancel, sumRgb, sampleCount, sumLumSq, aovs, passes, traced);
}

// One batch into the device film (cleared first), read back through pinned staging and added to
// the caller's host film over the tile's pixels on all host cores, as Film::addBatch does per pixel.
static int32_t renderHostFilm(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                              const volatile int32_t* cancel, float* sumRgb, uint32_t* sampleCount, float* sumLumSq,
                              uint64_t* traced, Tile tile) {
    int32_t rc;
    if ((rc = pe_device_film_clear(d))) return rc;
    if ((rc = ensureCapacity(d, kWaveSlots))) return rc;
    const int32_t rr = renderWaves(d, cam, st, first, count, cancel, d->fSum, d->fCnt, d->fSq, nullptr, d->capacity,
                                   true, tile);
    if (rr != PE_OK && rr != PE_ERR_CANCELLED) return rr;
    const size_t n = static_cast<size_t>(st->width) * static_cast<size_t>(st->height);
    const size_t bytes = n * 5 * sizeof(float);
    if (d->stageBytes < bytes) {
        if (d->stage) cudaFreeHost(d->stage);
        d->stage = nullptr;
        d->stageBytes = 0;
        PE_CUDA(cudaMallocHost(&d->stage, bytes));
        d->stageBytes = bytes;
    }
    float* s = reinterpret_cast<float*>(d->stage);
    uint32_t* c = reinterpret_cast<uint32_t*>(s + 3 * n);
    float* q = s + 4 * n;
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t rows = static_cast<size_t>(tile.h), W = static_cast<size_t>(st->width);
    const size_t chunk = (rows + hw - 1) / hw;
    // the tile's rows come back in hw pieces, one copy each on the device stream; each piece is
    // merged by its own thread as soon as its copy has landed, while the later pieces copy
    std::vector<cudaEvent_t> landed(hw, nullptr);
    struct EventsGuard {
        std::vector<cudaEvent_t>& ev;
        ~EventsGuard() {
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
        }
    } eventsGuard{landed};
    for (unsigned t = 0; t < hw; ++t) {
        const size_t r0 = std::min(rows, t * chunk), r1 = std::min(rows, (t + 1) * chunk);
        const size_t b = (static_cast<size_t>(tile.y0) + r0) * W, e = (static_cast<size_t>(tile.y0) + r1) * W;
        if (e > b) {
            PE_CUDA(cudaMemcpyAsync(s + 3 * b, d->fSum + 3 * b, 3 * (e - b) * sizeof(float), cudaMemcpyDeviceToHost,
                                    d->stream));
            PE_CUDA(cudaMemcpyAsync(c + b, d->fCnt + b, (e - b) * sizeof(uint32_t), cudaMemcpyDeviceToHost, d->stream));
            PE_CUDA(cudaMemcpyAsync(q + b, d->fSq + b, (e - b) * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
        }
        PE_CUDA(cudaEventCreateWithFlags(&landed[t], cudaEventDisableTiming));
        PE_CUDA(cudaEventRecord(landed[t], d->stream));
    }
    std::vector<uint64_t> partial(hw, 0);
    std::vector<int> copyFailed(hw, 0);
    auto merge = [&](unsigned t) {
        uint64_t tr = 0;
        if (cudaEventSynchronize(landed[t]) != cudaSuccess) {
            copyFailed[t] = 1;
            return;
        }
        for (size_t r = t * chunk; r < std::min(rows, (t + 1) * chunk); ++r) {
            const size_t b = (static_cast<size_t>(tile.y0) + r) * W + static_cast<size_t>(tile.x0);
            const size_t e = b + static_cast<size_t>(tile.w);
            for (size_t i = b; i < e; ++i) tr += c[i];
            if (sampleCount)
                for (size_t i = b; i < e; ++i) sampleCount[i] += c[i];
            if (sumRgb)
                for (size_t i = 3 * b; i < 3 * e; ++i) sumRgb[i] += s[i];
            if (sumLumSq)
                for (size_t i = b; i < e; ++i) sumLumSq[i] += q[i];
        }
        partial[t] = tr;
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < hw; ++t) pool.emplace_back(merge, t);
    merge(0);
    for (auto& th : pool) th.join();
    for (int f : copyFailed)
        if (f) {
            setError(std::string("film read-back failed: ") + cudaMsg(cudaGetLastError()));
            return PE_ERR_CUDA;
        }
    uint64_t tr = 0;
    for (uint64_t p : partial) tr += p;
    if (traced) *traced = tr;
    return rr;
}

int32_t pe_device_render(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                         const volatile int32_t* cancel, float* sumRgb, uint32_t* sampleCount, float* sumLumSq,
                         uint64_t* traced) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("render before set_scene");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    if (count <= 0) return PE_OK;
    PE_CUDA(cudaSetDevice(d->ordinal));
    if ((rc = ensureFilm(d, st->width, st->height))) return rc;
    if (st->adaptive_sampling) {
        // the decisions read the accumulated film: the caller's film goes to the device, takes
        // the batch's samples there in sample order, and comes back whole
        if (!sumRgb || !sampleCount || !sumLumSq) {
            setError("adaptive sampling needs the film's sums, counts and squared-luminance sums");
            return PE_ERR_INVALID;
        }
        const size_t n = static_cast<size_t>(st->width) * static_cast<size_t>(st->height);
        if ((rc = ensureCapacity(d, kWaveSlots))) return rc;
        PE_CUDA(cudaMemcpyAsync(d->fSum, sumRgb, n * 3 * sizeof(float), cudaMemcpyHostToDevice, d->stream));
        PE_CUDA(cudaMemcpyAsync(d->fCnt, sampleCount, n * sizeof(uint32_t), cudaMemcpyHostToDevice, d->stream));
        PE_CUDA(cudaMemcpyAsync(d->fSq, sumLumSq, n * sizeof(float), cudaMemcpyHostToDevice, d->stream));
        const int32_t ar = renderAdaptive(d, cam, st, first, count, cancel, traced);
        if (ar != PE_OK && ar != PE_ERR_CANCELLED) return ar;
        if ((rc = pe_device_film_read(d, sumRgb, sampleCount, sumLumSq))) return rc;
        return ar;
    }
    return renderHostFilm(d, cam, st, first, count, cancel, sumRgb, sampleCount, sumLumSq, traced,
                          Tile{0, 0, st->width, st->height});
}

int32_t pe_device_render_region(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t x0, int32_t y0,
                                int32_t w, int32_t h, int32_t first, int32_t count, const volatile int32_t* cancel,
                                float* sumRgb, uint32_t* sampleCount, float* sumLumSq, uint64_t* traced) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("render before set_scene");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    if (x0 < 0 || y0 < 0 || w <= 0 || h <= 0 || x0 + w > st->width || y0 + h > st->height) {
        setError("pe_device_render_region: region outside the film");
        return PE_ERR_INVALID;
    }
    if (st->adaptive_sampling) {
        setError("pe_device_render_region: adaptive sampling renders whole films (pe_device_render)");
        return PE_ERR_INVALID;
    }
    if (count <= 0) return PE_OK;
    PE_CUDA(cudaSetDevice(d->ordinal));
    if ((rc = ensureFilm(d, st->width, st->height))) return rc;
    return renderHostFilm(d, cam, st, first, count, cancel, sumRgb, sampleCount, sumLumSq, traced, Tile{x0, y0, w, h});
}

// A caller's film buffer must be memory of this device that holds `bytes` from `p` on: a host
// pointer, another device's memory or a short buffer would make the film kernel write outside it.
// The allocation's extent comes from the driver's cuMemGetAddressRange, reached through the
// runtime's entry-point query (no link against the driver library).
static int32_t checkFilmPointer(pe_device* d, const char* name, const void* p, size_t bytes) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        setError(std::string("pe_device_render_tile_noalloc: ") + name + " is not CUDA memory: " + cudaMsg(e));
        return PE_ERR_INVALID;
    }
    if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != d->ordinal) {
        setError(std::string("pe_device_render_tile_noalloc: ") + name + " must be device (or managed) memory of device " +
                 std::to_string(d->ordinal));
        return PE_ERR_INVALID;
    }
    using GetRange = int (*)(unsigned long long*, size_t*, unsigned long long);
    static GetRange getRange = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            fn = nullptr;
        }
        return reinterpret_cast<GetRange>(fn);
    }();
    if (getRange) {
        unsigned long long base = 0;
        size_t size = 0;
        const unsigned long long addr = reinterpret_cast<unsigned long long>(p);
        if (getRange(&base, &size, addr) == 0 && addr + bytes > base + size) {
            setError(std::string("pe_device_render_tile_noalloc: ") + name + " holds " +
                     std::to_string(base + size - addr) + " bytes from the given address; the film needs " +
                     std::to_string(bytes));
            return PE_ERR_INVALID;
        }
    }
    return PE_OK;
}

// Tile render that allocates no device memory: path state lives in g_noAllocScratch, the film is
// the caller's.  See include/photon_cuda.h for the contract.
int32_t pe_device_render_tile_noalloc(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t x0, int32_t y0,
                                      int32_t w, int32_t h, int32_t first, int32_t count, float* sumRgb,
                                      uint32_t* sampleCount, float* sumLumSq) {
    if (!d) {
        setError("pe_device_render_tile_noalloc: null device");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("pe_device_render_tile_noalloc: render before set_scene");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    if (!sumRgb || !sampleCount || !sumLumSq) {
        setError("pe_device_render_tile_noalloc: film pointers must be device memory of width*height pixels");
        return PE_ERR_INVALID;
    }
    if (x0 < 0 || y0 < 0 || w <= 0 || h <= 0 || x0 + w > st->width || y0 + h > st->height) {
        setError("pe_device_render_tile_noalloc: tile outside the film");
        return PE_ERR_INVALID;
    }
    if (static_cast<size_t>(w) * static_cast<size_t>(h) > kNoAllocSlots) {
        setError("pe_device_render_tile_noalloc: tile of " + std::to_string(w) + "x" + std::to_string(h) +
                 " pixels exceeds the maximum of " + std::to_string(kNoAllocSlots) + " pixels per call");
        return PE_ERR_LIMIT;
    }
    if (!d->noAllocBase) {
        setError("pe_device_render_tile_noalloc: scratch unavailable: " + d->noAllocError);
        return PE_ERR_CUDA;
    }
    if (st->adaptive_sampling) {
        setError("pe_device_render_tile_noalloc: adaptive sampling needs the device's own film (pe_device_render)");
        return PE_ERR_INVALID;
    }
    // The scratch holds plain path state only: no guiding records, no ray-cone column.
    if (d->guideKind != 0) {
        setError("pe_device_render_tile_noalloc: guided sampling (pe_device_set_guiding) is on; the tile entry "
                 "renders unguided paths only");
        return PE_ERR_INVALID;
    }
    if (d->scene.motions && st->motion_blur) {
        setError("pe_device_render_tile_noalloc: motion blur over moving instances needs a shutter time per path, "
                 "which the fixed scratch does not hold; use pe_device_render");
        return PE_ERR_INVALID;
    }
    if (d->scene.hasMips) {
        setError("pe_device_render_tile_noalloc: the scene has mipmapped image maps, whose level of detail needs a "
                 "per-path ray cone the tile entry does not keep");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    const size_t px = static_cast<size_t>(st->width) * static_cast<size_t>(st->height);
    rc = checkFilmPointer(d, "sum_rgb", sumRgb, px * 3 * sizeof(float));
    if (!rc) rc = checkFilmPointer(d, "sample_count", sampleCount, px * sizeof(uint32_t));
    if (!rc) rc = checkFilmPointer(d, "sum_lum_sq", sumLumSq, px * sizeof(float));
    if (rc) return rc;
    if (count <= 0) return PE_OK;
    Paths P = noAllocPaths(d->noAllocBase);
    // The array keeps the previous call's contents; the queue and shadow counters must start at 0.
    PE_CUDA(cudaMemsetAsync(P.counters, 0, 256, d->stream));
    return renderWaves(d, cam, st, first, count, nullptr, sumRgb, sampleCount, sumLumSq, &P, kNoAllocSlots, false,
                       Tile{x0, y0, w, h});
}

int32_t pe_device_synchronize(pe_device* d) {
    if (!d) return PE_ERR_INVALID;
    PE_CUDA(cudaStreamSynchronize(d->stream));
    return PE_OK;
}

int32_t pe_device_last_stats(pe_device* d, pe_render_stats* out) {
    if (!d || !out) {
        setError("null argument");
        return PE_ERR_INVALID;
    }
    *out = d->stats;
    return PE_OK;
}

// Times a few tail thresholds on probe renders of the caller's view into a scratch film and keeps
// the fastest; the film never depends on the threshold, so tuning is free to pick any of them.
// Coordinate descent over the tuning knobs on probe renders of the caller's frame (samples from
// 2^24 on, into a scratch film): the closest-hit traversal variant, then the shading kernels'
// register budget, then the tail threshold; each candidate is timed twice and its faster render
// counts, after one warm-up render.  The films are the same for every choice.
int32_t pe_device_autotune(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t probeSpp,
                           int64_t* chosen) {
    if (!d) {
        setError("pe_device_autotune: null device");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("pe_device_autotune: set a scene first");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    PE_CUDA(cudaSetDevice(d->ordinal));
    if ((rc = ensureCapacity(d, kWaveSlots))) return rc;
    const size_t n = static_cast<size_t>(st->width) * static_cast<size_t>(st->height);
    std::vector<DevBuf> tmp;
    float* sum = nullptr;
    uint32_t* cnt = nullptr;
    float* sq = nullptr;
    if ((rc = devAlloc(tmp, sum, n * 3)) || (rc = devAlloc(tmp, cnt, n)) || (rc = devAlloc(tmp, sq, n))) {
        freeList(tmp);
        return rc;
    }
    const int spp = std::max(1, probeSpp);
    // probe renders neither train nor sample a guiding field
    const int savedKind = d->guideKind, savedMode = d->guide.mode;
    d->guideKind = 0;
    d->guide.mode = 0;
    const int64_t savedTail = d->tailPaths;
    const int savedClosest = d->closestMode, savedBudget = d->shadeBudget, savedAny = d->anyMode;
    const size_t savedWave = d->waveSlots;
    std::string log;
    auto probe = [&](float& ms) -> int32_t {
        ms = 1e30f;
        for (int k = 0; k < 2; ++k) {
            const int32_t r = renderWaves(d, cam, st, 1 << 24, spp, nullptr, sum, cnt, sq, nullptr, d->capacity, false,
                                          Tile{0, 0, st->width, st->height});
            if (r) return r;
            ms = std::min(ms, d->stats.ms_total);
        }
        return PE_OK;
    };
    float warm = 0.0f;
    rc = probe(warm);
    // one knob at a time, the others at their best so far
    auto tune = [&](const char* name, auto set, const std::vector<int64_t>& values) {
        float best = 1e30f;
        int64_t pick = values.front();
        for (int64_t v : values) {
            if (rc) return;
            set(v);
            float ms = 0.0f;
            rc = probe(ms);
            log += std::string(name) + "=" + std::to_string(v) + " " + std::to_string(ms) + " ms\n";
            if (!rc && ms < best) {
                best = ms;
                pick = v;
            }
        }
        set(pick);
    };
    // paths in flight first: every later probe runs at the chosen wave size (lanes grow as needed)
    tune("wave_slots",
         [&](int64_t v) {
             d->waveSlots = static_cast<size_t>(v);
             if (!rc) rc = ensureCapacity(d, kWaveSlots);
         },
         {static_cast<int64_t>(kWaveSlots), static_cast<int64_t>(kDefaultWaveSlots), static_cast<int64_t>(kMaxWaveSlots)});
    tune("closest_traversal", [&](int64_t v) { d->closestMode = static_cast<int>(v); },
         {TRACE_WIDE, TRACE_BINARY, TRACE_WIDE_SMEM8, TRACE_WIDE_SMEM16, TRACE_WIDE_REG4, TRACE_WIDE_REG8,
          TRACE_WIDE_OCC8, TRACE_WIDE_SMEM8_OCC8, TRACE_WIDE_SMEM16_OCC8});
    tune("any_traversal", [&](int64_t v) { d->anyMode = static_cast<int>(v); }, {0, 1, 2});
    tune("shade_budget", [&](int64_t v) { d->shadeBudget = static_cast<int>(v); }, {0, 1, 2});
    const int64_t grid = static_cast<int64_t>(d->blocksTail) * kTailBlock;
    tune("tail_paths", [&](int64_t v) { d->tailPaths = v; }, {grid / 4, grid / 2, grid, 2 * grid});
    d->guideKind = savedKind;
    d->guide.mode = savedMode;
    freeList(tmp);
    if (rc) {
        d->tailPaths = savedTail;
        d->closestMode = savedClosest;
        d->shadeBudget = savedBudget;
        d->anyMode = savedAny;
        d->waveSlots = savedWave;
    }
    d->tuneLog = log;
    if (chosen) *chosen = d->tailPaths;
    return rc;
}

int32_t pe_device_get_tuning(pe_device* d, pe_tuning* out) {
    if (!d || !out) {
        setError("pe_device_get_tuning: null argument");
        return PE_ERR_INVALID;
    }
    out->tail_paths = d->tailPaths;
    out->closest_traversal = d->closestMode;
    out->shade_budget = d->shadeBudget;
    out->any_traversal = d->anyMode;
    out->wave_slots = static_cast<int64_t>(d->waveSlots);
    return PE_OK;
}

int32_t pe_device_set_tuning(pe_device* d, const pe_tuning* t) {
    if (!d || !t) {
        setError("pe_device_set_tuning: null argument");
        return PE_ERR_INVALID;
    }
    if (t->tail_paths < -1 || t->closest_traversal < 0 || t->closest_traversal >= TRACE_MODES || t->shade_budget < 0 ||
        t->shade_budget > 2 || t->any_traversal < 0 || t->any_traversal > 2 ||
        (t->wave_slots != 0 && (t->wave_slots < static_cast<int64_t>(kMinWaveSlots) ||
                                t->wave_slots > static_cast<int64_t>(kMaxWaveSlots)))) {
        setError("pe_device_set_tuning: value out of range");
        return PE_ERR_INVALID;
    }
    d->tailPaths = t->tail_paths;
    d->closestMode = t->closest_traversal;
    d->shadeBudget = t->shade_budget;
    d->anyMode = t->any_traversal;
    if (t->wave_slots != 0) d->waveSlots = static_cast<size_t>(t->wave_slots);
    return PE_OK;
}

int32_t pe_device_autotune_log(pe_device* d, char* buf, size_t len) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (buf && len > 0) {
        const size_t k = std::min(len - 1, d->tuneLog.size());
        std::memcpy(buf, d->tuneLog.data(), k);
        buf[k] = 0;
    }
    return static_cast<int32_t>(d->tuneLog.size());
}

int32_t pe_device_set_tail_paths(pe_device* d, int64_t paths) {
    if (!d) {
        setError("null device");
        return PE_ERR_INVALID;
    }
    if (paths < -1) {
        setError("tail paths must be -1 (automatic), 0 (off) or a path count");
        return PE_ERR_INVALID;
    }
    d->tailPaths = paths;
    return PE_OK;
}

int64_t pe_device_tail_paths(pe_device* d) {
    if (!d) return -1;
    return d->tailPaths < 0 ? static_cast<int64_t>(d->blocksTail) * kTailBlock : d->tailPaths;
}

int32_t pe_device_set_counting(pe_device* d, int32_t enabled) {
    if (!d) return PE_ERR_INVALID;
    d->counting = enabled != 0;
    return PE_OK;
}

int32_t pe_device_timer_begin(pe_device* d) {
    if (!d) return PE_ERR_INVALID;
    PE_CUDA(cudaEventRecord(d->evT0, d->stream));
    return PE_OK;
}

int32_t pe_device_timer_end(pe_device* d, float* ms) {
    if (!d || !ms) return PE_ERR_INVALID;
    PE_CUDA(cudaEventRecord(d->evT1, d->stream));
    PE_CUDA(cudaEventSynchronize(d->evT1));
    PE_CUDA(cudaEventElapsedTime(ms, d->evT0, d->evT1));
    return PE_OK;
}

static int32_t tracePrimary(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t sampleIndex,
                            int32_t* outShape, int32_t* outPrim, float* outT, bool wide);

int32_t pe_device_trace_primary(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t sampleIndex,
                                int32_t* outShape, int32_t* outPrim, float* outT) {
    return tracePrimary(d, cam, st, sampleIndex, outShape, outPrim, outT, true);
}

int32_t pe_device_trace_primary_ordered(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t sampleIndex,
                                        int32_t* outShape, int32_t* outPrim, float* outT) {
    return tracePrimary(d, cam, st, sampleIndex, outShape, outPrim, outT, false);
}

static int32_t tracePrimary(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t sampleIndex,
                            int32_t* outShape, int32_t* outPrim, float* outT, bool wide) {
    if (!d || !outShape || !outPrim || !outT) {
        setError("null argument");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("trace before set_scene");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = checkSettings(cam, st);
    if (rc) return rc;
    PE_CUDA(cudaSetDevice(d->ordinal));
    WaveSeg A = makeSeg(cam, st);
    A.filterCdf = filterTable(d, st->filter_type, st->filter_width, ++d->filterClock, d->stream);
    if (!A.filterCdf) {
        setError("pixel filter table upload failed");
        return PE_ERR_CUDA;
    }
    A.sampleFirst = sampleIndex;
    const int n = st->width * st->height;
    std::vector<DevBuf> tmp;
    int32_t* dS = nullptr;
    int32_t* dP = nullptr;
    float* dT = nullptr;
    if ((rc = devAlloc(tmp, dS, n)) || (rc = devAlloc(tmp, dP, n)) || (rc = devAlloc(tmp, dT, n))) {
        freeList(tmp);
        return rc;
    }
    if (wide)
        kTracePrimary<true><<<d->prop.multiProcessorCount * 8, 128, 0, d->stream>>>(d->scene, A, n, dS, dP, dT);
    else
        kTracePrimary<false><<<d->prop.multiProcessorCount * 8, 128, 0, d->stream>>>(d->scene, A, n, dS, dP, dT);
    cudaMemcpyAsync(outShape, dS, n * sizeof(int32_t), cudaMemcpyDeviceToHost, d->stream);
    cudaMemcpyAsync(outPrim, dP, n * sizeof(int32_t), cudaMemcpyDeviceToHost, d->stream);
    cudaMemcpyAsync(outT, dT, n * sizeof(float), cudaMemcpyDeviceToHost, d->stream);
    const cudaError_t e = cudaStreamSynchronize(d->stream);
    freeList(tmp);
    if (e != cudaSuccess) {
        setError(std::string("trace_primary: ") + cudaMsg(e));
        return PE_ERR_CUDA;
    }
    return PE_OK;
}

int32_t pe_device_trace_rays(pe_device* d, const float* origins, const float* directions, const float* t_max, int32_t n,
                             int32_t mode, uint32_t mask, float time, int32_t* out_shape, int32_t* out_prim, float* out_t) {
    if (!d || !origins || !directions || !t_max || n < 0 || mode < 0 || mode > 2 || !out_shape || !out_prim || !out_t) {
        setError("pe_device_trace_rays: bad argument");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("pe_device_trace_rays: no scene");
        return PE_ERR_NO_SCENE;
    }
    if (n == 0) return PE_OK;
    PE_CUDA(cudaSetDevice(d->ordinal));
    std::vector<DevBuf> tmp;
    float *dO = nullptr, *dD = nullptr, *dM = nullptr, *dT = nullptr;
    int32_t *dS = nullptr, *dP = nullptr;
    const size_t m = static_cast<size_t>(n);
    int32_t rc;
    if ((rc = devAlloc(tmp, dO, 3 * m)) || (rc = devAlloc(tmp, dD, 3 * m)) || (rc = devAlloc(tmp, dM, m)) ||
        (rc = devAlloc(tmp, dT, m)) || (rc = devAlloc(tmp, dS, m)) || (rc = devAlloc(tmp, dP, m))) {
        freeList(tmp);
        return rc;
    }
    cudaMemcpyAsync(dO, origins, 3 * m * sizeof(float), cudaMemcpyHostToDevice, d->stream);
    cudaMemcpyAsync(dD, directions, 3 * m * sizeof(float), cudaMemcpyHostToDevice, d->stream);
    cudaMemcpyAsync(dM, t_max, m * sizeof(float), cudaMemcpyHostToDevice, d->stream);
    const int grid = d->prop.multiProcessorCount * 8;
    const SceneGPU& S = d->scene;
    if (mode == 0) kTraceRays<0><<<grid, 128, 0, d->stream>>>(S, dO, dD, dM, n, mask, time, dS, dP, dT);
    else if (mode == 1) kTraceRays<1><<<grid, 128, 0, d->stream>>>(S, dO, dD, dM, n, mask, time, dS, dP, dT);
    else kTraceRays<2><<<grid, 128, 0, d->stream>>>(S, dO, dD, dM, n, mask, time, dS, dP, dT);
    cudaMemcpyAsync(out_shape, dS, m * sizeof(int32_t), cudaMemcpyDeviceToHost, d->stream);
    cudaMemcpyAsync(out_prim, dP, m * sizeof(int32_t), cudaMemcpyDeviceToHost, d->stream);
    cudaMemcpyAsync(out_t, dT, m * sizeof(float), cudaMemcpyDeviceToHost, d->stream);
    const cudaError_t e = cudaStreamSynchronize(d->stream);
    freeList(tmp);
    if (e != cudaSuccess) {
        setError(std::string("trace_rays: ") + cudaMsg(e));
        return PE_ERR_CUDA;
    }
    return PE_OK;
}

int32_t pe_device_sobol(pe_device* d, uint64_t seed, const int32_t* px, const int32_t* py, const int32_t* index, size_t n,
                        int32_t nd, float* out) {
    if (!d || !px || !py || !index || !out || nd <= 0) {
        setError("pe_device_sobol: bad argument");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    std::vector<DevBuf> tmp;
    int32_t *dx = nullptr, *dy = nullptr, *di = nullptr;
    float* dout = nullptr;
    int32_t rc;
    if ((rc = devAlloc(tmp, dx, n)) || (rc = devAlloc(tmp, dy, n)) || (rc = devAlloc(tmp, di, n)) ||
        (rc = devAlloc(tmp, dout, n * static_cast<size_t>(nd) * 2))) {
        freeList(tmp);
        return rc;
    }
    cudaMemcpyAsync(dx, px, n * 4, cudaMemcpyHostToDevice, d->stream);
    cudaMemcpyAsync(dy, py, n * 4, cudaMemcpyHostToDevice, d->stream);
    cudaMemcpyAsync(di, index, n * 4, cudaMemcpyHostToDevice, d->stream);
    kSobol<<<d->prop.multiProcessorCount * 4, 128, 0, d->stream>>>(d->dTables, seed, dx, dy, di, static_cast<int>(n), nd, dout);
    cudaMemcpyAsync(out, dout, n * static_cast<size_t>(nd) * 2 * sizeof(float), cudaMemcpyDeviceToHost, d->stream);
    const cudaError_t e = cudaStreamSynchronize(d->stream);
    freeList(tmp);
    if (e != cudaSuccess) {
        setError(std::string("sobol: ") + cudaMsg(e));
        return PE_ERR_CUDA;
    }
    return PE_OK;
}

int32_t pe_device_bsdf_probe(pe_device* d, int32_t material, const pe_bsdf_query* q, size_t n, pe_bsdf_result* out) {
    if (!d || !q || !out) {
        setError("pe_device_bsdf_probe: null argument");
        return PE_ERR_INVALID;
    }
    if (!d->hasScene) {
        setError("probe before set_scene");
        return PE_ERR_NO_SCENE;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    std::vector<DevBuf> tmp;
    pe_bsdf_query* dq = nullptr;
    pe_bsdf_result* dr = nullptr;
    int32_t rc;
    if ((rc = devAlloc(tmp, dq, n)) || (rc = devAlloc(tmp, dr, n))) {
        freeList(tmp);
        return rc;
    }
    cudaMemcpyAsync(dq, q, n * sizeof(pe_bsdf_query), cudaMemcpyHostToDevice, d->stream);
    kBsdfProbe<<<d->prop.multiProcessorCount * 2, 128, 0, d->stream>>>(d->scene, material, dq, static_cast<int>(n), dr);
    cudaMemcpyAsync(out, dr, n * sizeof(pe_bsdf_result), cudaMemcpyDeviceToHost, d->stream);
    const cudaError_t e = cudaStreamSynchronize(d->stream);
    freeList(tmp);
    if (e != cudaSuccess) {
        setError(std::string("bsdf_probe: ") + cudaMsg(e));
        return PE_ERR_CUDA;
    }
    return PE_OK;
}

} // extern "C"
