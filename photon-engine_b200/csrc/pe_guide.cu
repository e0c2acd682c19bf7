// pe_guide.cu — kernels and host control of the learned directional proposal (pe_guide.cuh):
//   kGuideInferTC    tensor-core MLP inference, 128 queries per tile, TMEM accumulators
//   kGuideInferSimt  the same network in FP32 on the SIMT cores (reference for the tensor path)
//   kGuideTrain      one warp per training sample: forward, mixture NLL gradient, backward into
//                    the MLP (shared-memory accumulation) and the hash grid (global atomics)
//   kGuideAdam       Adam step over MLP and grid, then the FP16 weight copy
//   kGuideQuery      per-bounce query rows (hit point, shading normal, view direction) of the
//                    rays whose next vertex samples with the proposal
//   kGuideCollect    per-path training samples from the first guided vertex once the path ended
#include "pe_device_impl.h"
#include "pe_guide.cuh"
#include "pe_tc.cuh"
#include "pe_trace.cuh"

#include <cmath>
#include <cstring>
#include <random>

using namespace pe;
using namespace pe_dev;

namespace {

// ---- tensor-core inference ---------------------------------------------------------------------
constexpr int kTcRows = 128;
constexpr uint32_t kSmW0 = 0;                 // 64 × 48 halves
constexpr uint32_t kSmW1 = 6144;              // 64 × 64
constexpr uint32_t kSmW2 = 14336;
constexpr uint32_t kSmW3 = 22528;
constexpr uint32_t kSmA = 30720;              // 128 × 64 halves (activations)
constexpr uint32_t kSmBias = 47104;           // 4 × 64 floats
constexpr uint32_t kSmBar = 48128;            // mbarrier
constexpr uint32_t kSmTmem = 48136;           // TMEM base address
constexpr uint32_t kSmBytes = 48256;
constexpr uint32_t kTmemCols = 128;           // two 64-column accumulators, alternating by layer
constexpr uint32_t kWaitPolls = 1u << 24;

__device__ __forceinline__ void storeRow8(unsigned char* tile, int row, int k0, const float* v) {
    __align__(16) __half h[8];
    for (int i = 0; i < 8; ++i) h[i] = __float2half_rn(v[i]);
    *reinterpret_cast<uint4*>(tile + coreOffset(row, k0, kTcRows)) = *reinterpret_cast<const uint4*>(h);
}

// Queries: 3 float4 per row (position | shading normal | direction to the viewer).  Row r's 40
// mixture outputs go to out[slot(r) · 10 ...] as 10 float4; mark[slot] = 1 tells the shading
// kernel that this bounce's proposal is there.
__global__ void __launch_bounds__(kTcRows) kGuideInferTC(GuideNet g, const float4* q, const int32_t* slots,
                                                         const uint32_t* count, int nFixed, float4* out, uint32_t* mark,
                                                         uint32_t* err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int n = count ? static_cast<int>(*count) : nFixed;
    const int tid = threadIdx.x, warp = tid >> 5;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(sm + kSmTmem);
    float* bias = reinterpret_cast<float*>(sm + kSmBias);
    // weights → core-matrix tiles (N = 64 rows each)
    const uint32_t wOff[4] = {kSmW0, kSmW1, kSmW2, kSmW3};
    const int wSrc[4] = {kOffW1, kOffW2, kOffW3, kOffW4};
    const int bSrc[4] = {kOffB1, kOffB2, kOffB3, kOffB4};
    for (int L = 0; L < 4; ++L) {
        const int K = L == 0 ? kNetIn : kNetHidden;
        for (int i = tid; i < 64 * K; i += kTcRows) {
            const int row = i / K, k = i - row * K;
            *reinterpret_cast<__half*>(sm + wOff[L] + coreOffset(row, k, 64)) = g.mlp16[wSrc[L] + i];
        }
        for (int j = tid; j < 64; j += kTcRows) bias[L * 64 + j] = g.mlp[bSrc[L] + j];
    }
    if (tid == 0) mbarInit(bar, 1);
    if (warp == 0) {
        tmemAlloc(tmemSlot, kTmemCols);
        tmemRelinquish();
    }
    fenceProxyAsync();
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = *tmemSlot;
    const uint32_t laneBase = static_cast<uint32_t>(warp * 32) << 16;
    unsigned char* A = sm + kSmA;
    uint32_t phase = 0;
    bool failed = false;
    for (int tile = blockIdx.x; tile * kTcRows < n && !failed; tile += gridDim.x) {
        const int row = tile * kTcRows + tid;
        const bool valid = row < n;
        float x[kNetIn];
        if (valid) {
            const float4 a = q[3 * row], b = q[3 * row + 1], c = q[3 * row + 2];
            guideInput(g, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), mk(c.x, c.y, c.z), x);
        } else {
            for (int i = 0; i < kNetIn; ++i) x[i] = 0.0f;
        }
        for (int k0 = 0; k0 < kNetIn; k0 += 8) storeRow8(A, tid, k0, x + k0);
        fenceProxyAsync();
        tcFenceBefore();
        __syncthreads();
        tcFenceAfter();
        for (int L = 0; L < 4; ++L) {
            const int K = L == 0 ? kNetIn : kNetHidden;
            const uint32_t dcol = static_cast<uint32_t>(L & 1) * 64;
            if (tid == 0) {
                for (int ks = 0; ks < K / 16; ++ks) {
                    const uint64_t ad = smemDesc(smemAddr(A) + ks * 2 * 2048, 2048, 128);
                    const uint64_t bd = smemDesc(smemAddr(sm + wOff[L]) + ks * 2 * 1024, 1024, 128);
                    tcMma(tmem + dcol, ad, bd, instrDescF16(kTcRows, 64), ks > 0);
                }
                tcCommit(bar);
            }
            const bool ok = mbarWait(bar, phase, kWaitPolls);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            tcFenceAfter();
            float v[64];
            for (int c = 0; c < 4; ++c) tmemLoad16(tmem + laneBase + dcol + 16 * c, v + 16 * c);
            if (L < 3) {
                for (int j = 0; j < 64; ++j) v[j] = fmaxf(v[j] + bias[L * 64 + j], 0.0f);
                for (int k0 = 0; k0 < 64; k0 += 8) storeRow8(A, tid, k0, v + k0);
                fenceProxyAsync();
                tcFenceBefore();
                __syncthreads();
                tcFenceAfter();
            } else if (valid) {
                const int dst = slots ? slots[row] : row;
                for (int j = 0; j < kNetUsedOut; j += 4)
                    out[static_cast<size_t>(dst) * 10 + j / 4] =
                        make_float4(v[j] + bias[192 + j], v[j + 1] + bias[193 + j], v[j + 2] + bias[194 + j],
                                    v[j + 3] + bias[195 + j]);
                if (mark) mark[dst] = 1u;
            }
        }
        __syncthreads();
    }
    if (failed) {
        // a commit never arrived: record it, give the MMAs in flight a bounded time to land,
        // then release TMEM
        if (tid == 0) atomicOr(err, 1u);
        mbarWait(bar, phase, kWaitPolls);
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0) tmemDealloc(tmem, kTmemCols);
}

__global__ void kGuideInferSimt(GuideNet g, const float4* q, int n, float4* out) {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const float4 a = q[3 * row], b = q[3 * row + 1], c = q[3 * row + 2];
        float x[kNetIn], h1[kNetHidden], h2[kNetHidden], h3[kNetHidden], o[kNetOut];
        guideInput(g, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), mk(c.x, c.y, c.z), x);
        mlpForward(g.mlp, x, h1, h2, h3, o);
        for (int j = 0; j < kNetUsedOut; j += 4)
            out[static_cast<size_t>(row) * 10 + j / 4] = make_float4(o[j], o[j + 1], o[j + 2], o[j + 3]);
    }
}

// ---- training ----------------------------------------------------------------------------------
// Samples: 4 float4 per row — position | shading normal | view direction | (sampled direction,
// weight c).  Loss Σ c · (−log q(ω | x)); gradients are accumulated into gradMlp / gradGrid.
constexpr int kTrainWarps = 8;

__device__ __forceinline__ void layerForward(const float* W, const float* b, const float* in, int nIn, float* outv,
                                             int lane, bool relu) {
    for (int j = lane; j < 64; j += 32) {
        float a = b[j];
        for (int i = 0; i < nIn; ++i) a += W[j * nIn + i] * in[i];
        outv[j] = relu ? fmaxf(a, 0.0f) : a;
    }
    __syncwarp();
}

// dIn[i] = Σ_j W[j][i] · dOut[j] (masked by the input's ReLU when `mask` is given); dW, db
// accumulate into shared memory.
__device__ __forceinline__ void layerBackward(const float* W, float* gW, float* gb, const float* in, int nIn,
                                              const float* dOut, float* dIn, const float* mask, int lane) {
    for (int j = lane; j < 64; j += 32) {
        const float d = dOut[j];
        if (d != 0.0f) {
            atomicAdd(&gb[j], d);
            for (int i = 0; i < nIn; ++i)
                if (in[i] != 0.0f) atomicAdd(&gW[j * nIn + i], d * in[i]);
        }
    }
    if (dIn) {
        for (int i = lane; i < nIn; i += 32) {
            float a = 0.0f;
            for (int j = 0; j < 64; ++j) a += W[j * nIn + i] * dOut[j];
            dIn[i] = (mask && !(mask[i] > 0.0f)) ? 0.0f : a;
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kTrainWarps * 32) kGuideTrain(GuideNet g, const float4* samples, const uint32_t* count,
                                                                int nFixed, float* gradMlp, float* gradGrid, float* loss) {
    extern __shared__ float smf[];
    float* P = smf;                                  // kNetParams
    float* G = smf + kNetParams;                     // kNetParams
    float* act = smf + 2 * kNetParams;               // per warp: x 48, h1 64, h2 64, h3 64, o 64, d0 64, d1 64
    const int n = count ? static_cast<int>(*count) : nFixed;
    for (int i = threadIdx.x; i < kNetParams; i += blockDim.x) {
        P[i] = g.mlp[i];
        G[i] = 0.0f;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* x = act + warp * 432;
    float* h1 = x + 48;
    float* h2 = h1 + 64;
    float* h3 = h2 + 64;
    float* o = h3 + 64;
    float* d0 = o + 64;
    float* d1 = d0 + 64;
    float lossSum = 0.0f;
    for (int s = blockIdx.x * kTrainWarps + warp; s < n; s += gridDim.x * kTrainWarps) {
        const float4 a = samples[4 * s], b = samples[4 * s + 1], c = samples[4 * s + 2], w4 = samples[4 * s + 3];
        const float weight = w4.w;
        if (lane == 0) guideInput(g, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), mk(c.x, c.y, c.z), x);
        __syncwarp();
        layerForward(P + kOffW1, P + kOffB1, x, kNetIn, h1, lane, true);
        layerForward(P + kOffW2, P + kOffB2, h1, kNetHidden, h2, lane, true);
        layerForward(P + kOffW3, P + kOffB3, h2, kNetHidden, h3, lane, true);
        layerForward(P + kOffW4, P + kOffB4, h3, kNetHidden, o, lane, false);
        if (lane == 0) {
            const float l = nllGrad(o, mk(w4.x, w4.y, w4.z), d0);
            for (int j = 0; j < kNetOut; ++j) d0[j] *= weight;
            lossSum += weight * l;
        }
        __syncwarp();
        layerBackward(P + kOffW4, G + kOffW4, G + kOffB4, h3, kNetHidden, d0, d1, h3, lane);
        layerBackward(P + kOffW3, G + kOffW3, G + kOffB3, h2, kNetHidden, d1, d0, h2, lane);
        layerBackward(P + kOffW2, G + kOffW2, G + kOffB2, h1, kNetHidden, d0, d1, h1, lane);
        layerBackward(P + kOffW1, G + kOffW1, G + kOffB1, x, kNetIn, d1, d0, nullptr, lane);
        // hash grid: lane i < 32 carries feature i = 2·level + f
        const V3 u = guideUnit(g, mk(a.x, a.y, a.z));
        {
            const int level = lane >> 1, f = lane & 1;
            const float dg = d0[lane];
            if (dg != 0.0f) {
                GridCorners cc;
                gridCorners(level, u, cc);
                for (int k = 0; k < 8; ++k) atomicAdd(&gradGrid[2 * cc.idx[k] + f], cc.w[k] * dg);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kNetParams; i += blockDim.x)
        if (G[i] != 0.0f) atomicAdd(&gradMlp[i], G[i]);
    if (lane == 0 && lossSum != 0.0f) atomicAdd(loss, lossSum);
}

__global__ void kGuideAdam(float* p, float* grad, float* m, float* v, int n, float lr, float scale, float c1, float c2) {
    // ε as small as instant-ngp's: hash-grid gradients are tiny and sparse
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-15f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = grad[i] * scale;
        grad[i] = 0.0f;
        if (gi == 0.0f && m[i] == 0.0f) continue;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void kGuideHalf(const float* p, __half* h, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) h[i] = __float2half_rn(p[i]);
}

// ---- rendering: per-bounce queries and per-wave training samples -------------------------------
// Query rows for the queued rays whose hit the next shading step may sample with the proposal:
// surface hits (not random-walk steps) below the depth limit on guidable materials.
__global__ void kGuideQuery(SceneGPU S, Paths P, Wave W, const int32_t* queue, const uint32_t* count) {
    const int n = static_cast<int>(*count);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = queue[i];
        const float4 hr = P.hit[slot];
        const int prim = __float_as_int(hr.w);
        bool want = false;
        V3 pnt, nrm, wo;
        if (!isMiss(prim)) {
            const float4 ro = P.rayO[slot];
            const int depth = static_cast<int>(__float_as_uint(P.pickN[slot].w) & 0xFFu);
            const WaveSeg& A = W.segs[segOfSlot(W, slot)];
            if (!(__float_as_uint(ro.w) & RAY_WALK) && depth < A.maxDepth) {
                const float4 rd = P.rayD[slot];
                Hit h;
                h.t = hr.x;
                h.u = hr.y;
                h.v = hr.z;
                h.prim = prim;
                Isect is;
                fillHit(S, h, mk(ro.x, ro.y, ro.z), mk(rd.x, rd.y, rd.z), is, pathTime(S, P, slot));
                const MatGPU& m = S.materials[is.material];
                want = (m.flags & (MF_DELTA | MF_VOLUME_BOUNDARY | MF_TRANSMITS_SHADOWS)) == 0;
                pnt = is.point;
                nrm = is.normal;
                wo = mk(-rd.x, -rd.y, -rd.z);
            }
        }
        if (want) {
            const uint32_t r = atomicAdd(&P.counters[CNT_GUIDE_Q], 1u);
            P.guideQ[3 * r + 0] = make_float4(pnt.x, pnt.y, pnt.z, 0.0f);
            P.guideQ[3 * r + 1] = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
            P.guideQ[3 * r + 2] = make_float4(wo.x, wo.y, wo.z, 0.0f);
            P.guideSlot[r] = slot;
        }
    }
}

// Training samples of the wave's recorded paths.  A record holds the first guidable vertex
// (point, normal, view direction, sampled direction ω, throughput before the bounce) and the
// radiance the path had gathered before anything arrived along ω; what the path added since,
// over that throughput, is f·cos·L(ω)/pdf for this one sample — the weight c of −c·log q(ω).
__global__ void kGuideCollect(Paths P, int nSlots) {
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) * P.guideStride; s < nSlots;
         s += gridDim.x * blockDim.x * P.guideStride) {
        float4* rec = P.guideRec + static_cast<size_t>(s) * 6;
        const float4 r4 = rec[4];
        if (r4.w == 0.0f) continue;
        rec[4] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float4 L = P.L[s];
        const V3 snap = r4.w == 2.0f ? mk(r4.x, r4.y, r4.z) : mk(L.x, L.y, L.z);
        const float4 tb = rec[5];
        const float tl = luminance(mk(tb.x, tb.y, tb.z));
        const float gained = luminance(mk(L.x - snap.x, L.y - snap.y, L.z - snap.z));
        if (!(tl > 0.0f) || !(gained > 0.0f)) continue;
        const float c = fminf(gained / tl, 64.0f);
        if (!pe::finitef(c)) continue;
        const uint32_t r = atomicAdd(&P.counters[CNT_TRAIN], 1u);
        const float4 wi = rec[3];
        P.trainBuf[4 * r + 0] = rec[0];
        P.trainBuf[4 * r + 1] = rec[1];
        P.trainBuf[4 * r + 2] = rec[2];
        P.trainBuf[4 * r + 3] = make_float4(wi.x, wi.y, wi.z, c);
    }
}

} // namespace

// ---- host ----------------------------------------------------------------------------------------
namespace pe_dev {

GuideNet guideNet(const pe_device* d) {
    GuideNet g{};
    g.mlp = d->guide.mlp;
    g.mlp16 = d->guide.mlp16;
    g.grid = d->guide.grid;
    for (int i = 0; i < 3; ++i) {
        g.boxMin[i] = d->guide.boxMin[i];
        const float ext = d->guide.boxMax[i] - d->guide.boxMin[i];
        g.boxInv[i] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
    return g;
}

int32_t guideAlloc(pe_device* d) {
    GuideState& G = d->guide;
    if (G.mlp) return PE_OK;
    int32_t rc = 0;
    if ((rc = devAlloc(G.bufs, G.mlp, kNetParams)) || (rc = devAlloc(G.bufs, G.mlp16, kNetParams)) ||
        (rc = devAlloc(G.bufs, G.grid, kGridParams)) || (rc = devAlloc(G.bufs, G.gradMlp, kNetParams)) ||
        (rc = devAlloc(G.bufs, G.gradGrid, kGridParams)) || (rc = devAlloc(G.bufs, G.mMlp, kNetParams)) ||
        (rc = devAlloc(G.bufs, G.vMlp, kNetParams)) || (rc = devAlloc(G.bufs, G.mGrid, kGridParams)) ||
        (rc = devAlloc(G.bufs, G.vGrid, kGridParams)) || (rc = devAlloc(G.bufs, G.loss, 1)) ||
        (rc = devAlloc(G.bufs, G.err, 1))) {
        freeList(G.bufs);
        G = GuideState{};
        return rc;
    }
    cudaFuncSetAttribute(kGuideTrain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>((2 * kNetParams + kTrainWarps * 432) * sizeof(float)));
    return PE_OK;
}

// Seeded initial network: Xavier-uniform hidden layers, a small output layer whose lobes start
// broad (log κ bias 0) around eight spread directions, grid features ~ U(−1e-4, 1e-4).
int32_t guideReset(pe_device* d, uint64_t seed) {
    int32_t rc = guideAlloc(d);
    if (rc) return rc;
    GuideState& G = d->guide;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> U(-1.0f, 1.0f);
    std::vector<float> P(kNetParams, 0.0f);
    auto xavier = [&](int off, int nOut, int nIn, float gain) {
        const float a = gain * std::sqrt(6.0f / static_cast<float>(nIn + nOut));
        for (int i = 0; i < nOut * nIn; ++i) P[off + i] = a * U(rng);
    };
    xavier(kOffW1, kNetHidden, kNetIn, 1.0f);
    xavier(kOffW2, kNetHidden, kNetHidden, 1.0f);
    xavier(kOffW3, kNetHidden, kNetHidden, 1.0f);
    xavier(kOffW4, kNetOut, kNetHidden, 0.1f);
    for (int k = 0; k < kLobes; ++k) {
        // Fibonacci-sphere directions
        const float z = 1.0f - (2.0f * k + 1.0f) / kLobes;
        const float r = std::sqrt(std::max(0.0f, 1.0f - z * z));
        const float phi = 2.39996323f * k;
        P[kOffB4 + 5 * k + 0] = r * std::cos(phi);
        P[kOffB4 + 5 * k + 1] = r * std::sin(phi);
        P[kOffB4 + 5 * k + 2] = z;
    }
    std::vector<float> grid(kGridParams);
    for (float& v : grid) v = 1e-4f * U(rng);
    PE_CUDA(cudaMemcpyAsync(G.mlp, P.data(), P.size() * sizeof(float), cudaMemcpyHostToDevice, d->stream));
    PE_CUDA(cudaMemcpyAsync(G.grid, grid.data(), grid.size() * sizeof(float), cudaMemcpyHostToDevice, d->stream));
    PE_CUDA(cudaMemsetAsync(G.gradMlp, 0, kNetParams * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(G.gradGrid, 0, static_cast<size_t>(kGridParams) * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(G.mMlp, 0, kNetParams * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(G.vMlp, 0, kNetParams * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(G.mGrid, 0, static_cast<size_t>(kGridParams) * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(G.vGrid, 0, static_cast<size_t>(kGridParams) * sizeof(float), d->stream));
    PE_CUDA(cudaMemsetAsync(G.err, 0, sizeof(uint32_t), d->stream));
    kGuideHalf<<<64, 256, 0, d->stream>>>(G.mlp, G.mlp16, kNetParams);
    PE_CUDA(cudaStreamSynchronize(d->stream));
    G.step = 0;
    G.samples = 0;
    return PE_OK;
}

int32_t guideInfer(pe_device* d, cudaStream_t s, const float4* q, const int32_t* slots, const uint32_t* count, int nFixed,
                   int maxRows, float4* out, uint32_t* mark) {
    const int sm = d->prop.multiProcessorCount;
    const int tiles = (maxRows + kTcRows - 1) / kTcRows;
    const int grid = std::max(1, std::min(tiles, 2 * sm));
    kGuideInferTC<<<grid, kTcRows, kSmBytes, s>>>(guideNet(d), q, slots, count, nFixed, out, mark, d->guide.err);
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

// Accumulates the gradient of a batch (device samples) and, with lr > 0, takes one Adam step.
int32_t guideTrain(pe_device* d, cudaStream_t s, const float4* samples, const uint32_t* count, int nFixed, int maxRows,
                   float lr) {
    GuideState& G = d->guide;
    const int sm = d->prop.multiProcessorCount;
    const int blocks = std::max(1, std::min(sm, (maxRows + kTrainWarps - 1) / kTrainWarps));
    const size_t smem = (2 * kNetParams + kTrainWarps * 432) * sizeof(float);
    kGuideTrain<<<blocks, kTrainWarps * 32, smem, s>>>(guideNet(d), samples, count, nFixed, G.gradMlp, G.gradGrid, G.loss);
    PE_CUDA(cudaGetLastError());
    if (lr > 0.0f) {
        ++G.step;
        const float c1 = 1.0f - std::pow(0.9f, static_cast<float>(G.step));
        const float c2 = 1.0f - std::pow(0.99f, static_cast<float>(G.step));
        const float scale = 1.0f / static_cast<float>(std::max(1, maxRows));
        kGuideAdam<<<sm * 4, 256, 0, s>>>(G.mlp, G.gradMlp, G.mMlp, G.vMlp, kNetParams, lr, scale, c1, c2);
        kGuideAdam<<<sm * 8, 256, 0, s>>>(G.grid, G.gradGrid, G.mGrid, G.vGrid, kGridParams, lr, scale, c1, c2);
        kGuideHalf<<<64, 256, 0, s>>>(G.mlp, G.mlp16, kNetParams);
        PE_CUDA(cudaGetLastError());
    }
    return PE_OK;
}

int32_t guideQueries(pe_device* d, cudaStream_t s, Paths& P, const Wave& W, const int32_t* queue, const uint32_t* count) {
    PE_CUDA(cudaMemsetAsync(&P.counters[CNT_GUIDE_Q], 0, sizeof(uint32_t), s));
    kGuideQuery<<<d->blocksIntersect, 128, 0, s>>>(d->scene, P, W, queue, count);
    PE_CUDA(cudaGetLastError());
    return guideInfer(d, s, P.guideQ, P.guideSlot, &P.counters[CNT_GUIDE_Q], 0, static_cast<int>(P.capacity), P.guideOut,
                      P.guideMark);
}

int32_t guideLearn(pe_device* d, cudaStream_t s, Paths& P, int nSlots) {
    GuideState& G = d->guide;
    const int maxRows = (nSlots + P.guideStride - 1) / P.guideStride;
    kGuideCollect<<<std::max(1, (maxRows + 255) / 256), 256, 0, s>>>(P, nSlots);
    PE_CUDA(cudaGetLastError());
    const int32_t rc = guideTrain(d, s, P.trainBuf, &P.counters[CNT_TRAIN], 0, maxRows, G.lr);
    if (rc) return rc;
    PE_CUDA(cudaMemsetAsync(&P.counters[CNT_TRAIN], 0, sizeof(uint32_t), s));
    return PE_OK;
}

// Per-slot proposal buffers of lane 0 (guided renders run on one lane, so that training between
// waves never races an inference still reading the weights).
int32_t guideBuffers(pe_device* d) {
    GuideState& G = d->guide;
    Paths& P = d->lanes[0].paths;
    if (G.bufCapacity == d->capacity && P.guideQ) return PE_OK;
    freeList(G.laneBufs);
    const size_t cap = d->capacity;
    int32_t rc = 0;
    if ((rc = devAlloc(G.laneBufs, P.guideQ, cap * 3)) || (rc = devAlloc(G.laneBufs, P.guideSlot, cap)) ||
        (rc = devAlloc(G.laneBufs, P.guideOut, cap * 10)) || (rc = devAlloc(G.laneBufs, P.guideMark, cap)) ||
        (rc = devAlloc(G.laneBufs, P.guideRec, cap * 6)) ||
        (rc = devAlloc(G.laneBufs, P.trainBuf, static_cast<size_t>(kGuideTrainRows + 1) * 4))) {
        freeList(G.laneBufs);
        P.guideQ = nullptr;
        return rc;
    }
    PE_CUDA(cudaMemsetAsync(P.guideMark, 0, cap * sizeof(uint32_t), d->stream));
    PE_CUDA(cudaMemsetAsync(P.guideRec, 0, cap * 6 * sizeof(float4), d->stream));
    G.bufCapacity = cap;
    return PE_OK;
}

} // namespace pe_dev

extern "C" {

// The hash grid's box: the scene's bounds, padded by 0.1 % of its extent.
static void sceneGuideBox(const pe_device* d, float lo[3], float hi[3]) {
    for (int i = 0; i < 3; ++i) {
        const float pad = 1e-3f * (d->scene.rootMax[i] - d->scene.rootMin[i]) + 1e-6f;
        lo[i] = d->scene.rootMin[i] - pad;
        hi[i] = d->scene.rootMax[i] + pad;
    }
}

int32_t pe_device_set_guiding(pe_device* d, int32_t mode, int32_t warmupSteps, float lr) {
    if (!d || mode < 0 || mode > 2 || warmupSteps < 0 || !(lr >= 0.0f)) {
        setError("pe_device_set_guiding: bad argument");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    GuideState& G = d->guide;
    d->guideKind = mode;
    if (mode != 2) d->sd.initialised = false; // the SD-tree field is dropped with its setting
    G.mode = mode == 1 ? 1 : 0;
    G.warmup = warmupSteps;
    G.lr = lr;
    if (mode == 0) return PE_OK;
    if (mode == 2) {
        // SD-tree guiding: the field is built by the first render (RenderSettings::pathGuiding)
        if (!d->hasScene) {
            setError("pe_device_set_guiding: set a scene first (its bounds span the spatial tree)");
            return PE_ERR_NO_SCENE;
        }
        int32_t rc = ensureCapacity(d, kWaveSlots);
        return rc ? rc : sdBuffers(d);
    }
    if (!d->hasScene) {
        setError("pe_device_set_guiding: set a scene first (its box bounds the hash grid)");
        return PE_ERR_NO_SCENE;
    }
    int32_t rc = PE_OK;
    // a network is kept across calls while it was built over this scene's box
    float lo[3], hi[3];
    sceneGuideBox(d, lo, hi);
    bool same = G.mlp != nullptr;
    for (int i = 0; i < 3; ++i) same = same && lo[i] == G.boxMin[i] && hi[i] == G.boxMax[i];
    if (!same) {
        for (int i = 0; i < 3; ++i) {
            G.boxMin[i] = lo[i];
            G.boxMax[i] = hi[i];
        }
        if ((rc = guideReset(d, 0x9E3779B97F4A7C15ull))) return rc;
    }
    if ((rc = ensureCapacity(d, kWaveSlots))) return rc;
    return guideBuffers(d);
}

int32_t pe_device_guide_info(pe_device* d, pe_guide_info* out) {
    if (!d || !out) {
        setError("pe_device_guide_info: null argument");
        return PE_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    const GuideState& G = d->guide;
    out->mode = d->guideKind;
    out->steps = G.step;
    out->ready = G.mlp && G.step >= G.warmup ? 1 : 0;
    if (G.mlp) {
        PE_CUDA(cudaStreamSynchronize(d->stream));
        PE_CUDA(cudaMemcpy(&out->last_loss, G.loss, sizeof(float), cudaMemcpyDeviceToHost));
    }
    return PE_OK;
}

int32_t pe_device_guide_reset(pe_device* d, uint64_t seed, const float boxMin[3], const float boxMax[3]) {
    if (!d || (!boxMin) != (!boxMax)) {
        setError("pe_device_guide_reset: null argument");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    if (!boxMin) {
        // the scene's box, padded as pe_device_set_guiding pads it
        if (!d->hasScene) {
            setError("pe_device_guide_reset: no box given and no scene set");
            return PE_ERR_NO_SCENE;
        }
        sceneGuideBox(d, d->guide.boxMin, d->guide.boxMax);
    } else {
        for (int i = 0; i < 3; ++i) {
            d->guide.boxMin[i] = boxMin[i];
            d->guide.boxMax[i] = boxMax[i];
        }
    }
    return guideReset(d, seed);
}

int32_t pe_device_guide_get(pe_device* d, float* mlp, float* grid) {
    if (!d || !d->guide.mlp) {
        setError("pe_device_guide_get: no guide (call pe_device_guide_reset)");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaStreamSynchronize(d->stream));
    if (mlp) PE_CUDA(cudaMemcpy(mlp, d->guide.mlp, kNetParams * sizeof(float), cudaMemcpyDeviceToHost));
    if (grid) PE_CUDA(cudaMemcpy(grid, d->guide.grid, static_cast<size_t>(kGridParams) * sizeof(float), cudaMemcpyDeviceToHost));
    return PE_OK;
}

int32_t pe_device_guide_set(pe_device* d, const float* mlp, const float* grid) {
    if (!d || !d->guide.mlp) {
        setError("pe_device_guide_set: no guide (call pe_device_guide_reset)");
        return PE_ERR_INVALID;
    }
    PE_CUDA(cudaStreamSynchronize(d->stream));
    if (mlp) PE_CUDA(cudaMemcpy(d->guide.mlp, mlp, kNetParams * sizeof(float), cudaMemcpyHostToDevice));
    if (grid) PE_CUDA(cudaMemcpy(d->guide.grid, grid, static_cast<size_t>(kGridParams) * sizeof(float), cudaMemcpyHostToDevice));
    kGuideHalf<<<64, 256, 0, d->stream>>>(d->guide.mlp, d->guide.mlp16, kNetParams);
    PE_CUDA(cudaStreamSynchronize(d->stream));
    return PE_OK;
}

int32_t pe_device_guide_eval(pe_device* d, const float* queries, int64_t n, int32_t tensorCores, float* out) {
    if (!d || !d->guide.mlp || (n > 0 && (!queries || !out))) {
        setError("pe_device_guide_eval: bad argument or no guide");
        return PE_ERR_INVALID;
    }
    if (n <= 0) return PE_OK;
    if (n > (int64_t(1) << 24)) {
        setError("pe_device_guide_eval: at most 16M queries per call");
        return PE_ERR_LIMIT;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    std::vector<DevBuf> tmp;
    float4* dq = nullptr;
    float4* dout = nullptr;
    int32_t rc = 0;
    if ((rc = devAlloc(tmp, dq, static_cast<size_t>(n) * 3)) || (rc = devAlloc(tmp, dout, static_cast<size_t>(n) * 10))) {
        freeList(tmp);
        return rc;
    }
    std::vector<float4> hq(static_cast<size_t>(n) * 3);
    for (int64_t r = 0; r < n; ++r)
        for (int j = 0; j < 3; ++j)
            hq[static_cast<size_t>(3 * r + j)] = make_float4(queries[9 * r + 3 * j], queries[9 * r + 3 * j + 1], queries[9 * r + 3 * j + 2], 0.0f);
    cudaMemcpyAsync(dq, hq.data(), hq.size() * sizeof(float4), cudaMemcpyHostToDevice, d->stream);
    cudaMemsetAsync(d->guide.err, 0, sizeof(uint32_t), d->stream);
    if (tensorCores) {
        rc = guideInfer(d, d->stream, dq, nullptr, nullptr, static_cast<int>(n), static_cast<int>(n), dout, nullptr);
    } else {
        kGuideInferSimt<<<d->prop.multiProcessorCount * 4, 128, 0, d->stream>>>(guideNet(d), dq, static_cast<int>(n), dout);
        rc = cudaGetLastError() == cudaSuccess ? PE_OK : PE_ERR_CUDA;
    }
    uint32_t err = 0;
    if (rc == PE_OK) {
        std::vector<float4> ho(static_cast<size_t>(n) * 10);
        cudaMemcpyAsync(ho.data(), dout, ho.size() * sizeof(float4), cudaMemcpyDeviceToHost, d->stream);
        cudaMemcpyAsync(&err, d->guide.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, d->stream);
        const cudaError_t e = cudaStreamSynchronize(d->stream);
        if (e != cudaSuccess) {
            setError(std::string("pe_device_guide_eval: ") + cudaMsg(e));
            rc = PE_ERR_CUDA;
        } else {
            std::memcpy(out, ho.data(), static_cast<size_t>(n) * kNetUsedOut * sizeof(float));
        }
    }
    freeList(tmp);
    if (rc == PE_OK && err) {
        setError("pe_device_guide_eval: a tensor-core wait ran out");
        rc = PE_ERR_DEVICE;
    }
    return rc;
}

int32_t pe_device_guide_grad(pe_device* d, const float* samples, int64_t n, float lr, float* mlpGrad, float* gridGrad,
                             float* loss) {
    if (!d || !d->guide.mlp || (n > 0 && !samples)) {
        setError("pe_device_guide_grad: bad argument or no guide");
        return PE_ERR_INVALID;
    }
    if (n > (int64_t(1) << 22)) {
        setError("pe_device_guide_grad: at most 4M samples per call");
        return PE_ERR_LIMIT;
    }
    PE_CUDA(cudaSetDevice(d->ordinal));
    GuideState& G = d->guide;
    std::vector<DevBuf> tmp;
    float4* ds = nullptr;
    int32_t rc = devAlloc(tmp, ds, static_cast<size_t>(std::max<int64_t>(n, 1)) * 4);
    if (rc) return rc;
    std::vector<float4> hs(static_cast<size_t>(n) * 4);
    for (int64_t r = 0; r < n; ++r) {
        const float* s = samples + 13 * r;
        hs[4 * r + 0] = make_float4(s[0], s[1], s[2], 0.0f);
        hs[4 * r + 1] = make_float4(s[3], s[4], s[5], 0.0f);
        hs[4 * r + 2] = make_float4(s[6], s[7], s[8], 0.0f);
        hs[4 * r + 3] = make_float4(s[9], s[10], s[11], s[12]);
    }
    cudaMemcpyAsync(ds, hs.data(), hs.size() * sizeof(float4), cudaMemcpyHostToDevice, d->stream);
    cudaMemsetAsync(G.loss, 0, sizeof(float), d->stream);
    // gradients are read before the step zeroes them
    rc = guideTrain(d, d->stream, ds, nullptr, static_cast<int>(n), static_cast<int>(n), 0.0f);
    if (rc == PE_OK) {
        if (mlpGrad) cudaMemcpyAsync(mlpGrad, G.gradMlp, kNetParams * sizeof(float), cudaMemcpyDeviceToHost, d->stream);
        if (gridGrad)
            cudaMemcpyAsync(gridGrad, G.gradGrid, static_cast<size_t>(kGridParams) * sizeof(float), cudaMemcpyDeviceToHost,
                            d->stream);
        if (loss) cudaMemcpyAsync(loss, G.loss, sizeof(float), cudaMemcpyDeviceToHost, d->stream);
        if (lr > 0.0f) {
            ++G.step;
            const int sm = d->prop.multiProcessorCount;
            const float c1 = 1.0f - std::pow(0.9f, static_cast<float>(G.step));
            const float c2 = 1.0f - std::pow(0.99f, static_cast<float>(G.step));
            const float scale = 1.0f / static_cast<float>(std::max<int64_t>(1, n));
            kGuideAdam<<<sm * 4, 256, 0, d->stream>>>(G.mlp, G.gradMlp, G.mMlp, G.vMlp, kNetParams, lr, scale, c1, c2);
            kGuideAdam<<<sm * 8, 256, 0, d->stream>>>(G.grid, G.gradGrid, G.mGrid, G.vGrid, kGridParams, lr, scale, c1, c2);
            kGuideHalf<<<64, 256, 0, d->stream>>>(G.mlp, G.mlp16, kNetParams);
        } else {
            cudaMemsetAsync(G.gradMlp, 0, kNetParams * sizeof(float), d->stream);
            cudaMemsetAsync(G.gradGrid, 0, static_cast<size_t>(kGridParams) * sizeof(float), d->stream);
        }
        const cudaError_t e = cudaStreamSynchronize(d->stream);
        if (e != cudaSuccess) {
            setError(std::string("pe_device_guide_grad: ") + cudaMsg(e));
            rc = PE_ERR_CUDA;
        }
    }
    freeList(tmp);
    return rc;
}

} // extern "C"
