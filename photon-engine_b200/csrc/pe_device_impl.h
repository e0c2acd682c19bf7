// pe_device_impl.h — the device object behind the pe_device_* C ABI and the wave machinery the
// single-request render path and the request server share (definitions in pe_device.cu).
#pragma once

#include "photon_cuda.h"
#include "pe_host.h"
#include "pe_wave.h"

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <utility>
#include <vector>

namespace pe_dev {

using namespace pe;

inline const char* cudaMsg(cudaError_t e) { return cudaGetErrorString(e); }

#define PE_CUDA(call)                                                                              \
    do {                                                                                           \
        const cudaError_t err__ = (call);                                                          \
        if (err__ != cudaSuccess) {                                                                \
            ::pe::setError(std::string(#call) + ": " + ::pe_dev::cudaMsg(err__));                  \
            return err__ == cudaErrorMemoryAllocation ? PE_ERR_OOM : PE_ERR_CUDA;                  \
        }                                                                                          \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

constexpr int kFilterSlots = 16;
constexpr int kMaxSegs = 64;                    // requests sharing one wave
constexpr size_t kWaveSlots = size_t(1) << 21;  // paths in flight per wave (guided, AOV and pass waves; servers)
// Paths in flight per regenerating wave (pe_tuning::wave_slots): the default, and the range
constexpr size_t kDefaultWaveSlots = size_t(1) << 23;
constexpr size_t kMinWaveSlots = size_t(1) << 20;
constexpr size_t kMaxWaveSlots = size_t(1) << 23;
// Live paths at or below which a guided wave hands its last paths to the tail kernel.
constexpr int64_t kGuideTailPaths = 2048;
// Bound on the bounce-by-bounce iterations of one wave (closest-hit queries of its longest path).
constexpr int kMaxWavefrontIterations = kMaxPathQueries;

struct FilterSlot {
    int type = -1;
    float width = -1.0f;
    uint64_t used = 0;
};

struct Tile {
    int x0, y0, w, h;
};

// One of a device's two wave pipelines: a stream, a path-state buffer, a segment table and a
// counter readback.  Consecutive waves of a render alternate lanes, so one wave's tail runs
// while the next wave traces its bounces; the film kernels stay in wave order.
struct WaveLane {
    cudaStream_t stream = nullptr;    // lane 0 runs on the device stream
    std::vector<DevBuf> bufs;
    Paths paths{};
    WaveSeg* hSegs = nullptr;         // pinned
    WaveSeg* dSegs = nullptr;
    cudaEvent_t evSegs = nullptr;     // the segment upload of the lane's last wave
    bool segsInFlight = false;
    uint32_t* hCounters = nullptr;    // pinned
    float4* aovA = nullptr;           // AOVs per slot (allocated on first use, in aovBufs)
    float4* aovN = nullptr;
    std::vector<DevBuf> aovBufs;
    float4* pass = nullptr;           // render passes per slot and per shadow record (passBufs)
    float4* shPass = nullptr;
    int32_t passStride = 0;
    std::vector<DevBuf> passBufs;
    int32_t* pathOf = nullptr;        // path regeneration buffers (in bufs)
    int32_t* freeQ = nullptr;
    float4* Lout = nullptr;
    cudaEvent_t evDone = nullptr;     // after the lane's last film kernel (timed)
    bool pending = false;             // evDone recorded since the render call began
};

// Event bookkeeping of one render call: per-kernel device times when timing.
struct RenderTimer {
    bool timing = false;
    size_t evUsed = 0;
    std::vector<std::pair<size_t, size_t>> isect, shade, shadow, tail;
};

// The learned directional proposal's parameters, optimiser state and control.
struct GuideState {
    std::vector<DevBuf> bufs;
    float* mlp = nullptr;       // FP32 master weights
    __half* mlp16 = nullptr;    // FP16 copy for the tensor cores
    float* grid = nullptr;      // hash-grid features
    float* gradMlp = nullptr;
    float* gradGrid = nullptr;
    float* mMlp = nullptr;
    float* vMlp = nullptr;
    float* mGrid = nullptr;
    float* vGrid = nullptr;
    float* loss = nullptr;
    uint32_t* err = nullptr;    // tensor-core wait ran out
    float boxMin[3] = {0, 0, 0}, boxMax[3] = {1, 1, 1};
    int64_t step = 0;
    int64_t samples = 0;
    // rendering with the proposal
    int mode = 0;               // 0 off, 1 learned proposal (train every wave, sample once ready)
    int warmup = 8;             // training steps before the renderer samples with the proposal
    float lr = 5e-3f;
    std::vector<DevBuf> laneBufs; // per-slot buffers of lane 0
    size_t bufCapacity = 0;
};

// SD-tree guiding field: host trees, their device copies, training schedule (pe_sdtree.cu).
struct SdHost {
    struct Node {
        int axis = -1;
        int child[2] = {-1, -1};
        int leaf = -1;
    };
    struct Leaf {
        std::vector<SdQuad> samp = std::vector<SdQuad>(1);
        float sampSum = 0.0f;
        std::vector<SdQuad> build = std::vector<SdQuad>(1);
        int buildOffset = 0;
    };
    float boxMin[3] = {0, 0, 0}, boxMax[3] = {1, 1, 1};
    std::vector<Node> nodes;
    std::vector<Leaf> leaves;
    bool ready = false;
    int iteration = 0;
    int samplesSeen = 0;      // samples traced since the last reset
    int nextRefine = 2;       // refine at 2, 4, 8, 16, 32 samples, then frozen
    size_t buildNodes = 0;
    SdField field{};
    std::vector<DevBuf> bufs;     // device copies of the trees
    std::vector<DevBuf> laneBufs; // per-slot records of lane 0
    size_t bufCapacity = 0;
    uint64_t sceneSerial = 0;     // the scene the field was trained on
    bool initialised = false;
    int waveMode = 0;             // SdModeBits of the waves being launched

    void reset(const float bmin[3], const float bmax[3]);
    void split(int idx, int depth);
    void refine(const std::vector<SdQuad>& buildSums, const std::vector<float>& buildSum,
                const std::vector<uint32_t>& counts);
    int32_t upload(cudaStream_t s);
    int32_t refineOnDevice(cudaStream_t s);
};

std::vector<SdQuad> refineTopology(const std::vector<SdQuad>& samp, float sum, float frac, int maxDepth);

} // namespace pe_dev

// One CUDA device: stream, resident scene, wave buffers, films and counters.
struct pe_device {
    using DevBuf = pe_dev::DevBuf;
    using FilterSlot = pe_dev::FilterSlot;
    using SceneGPU = pe::SceneGPU;
    using TablesGPU = pe::TablesGPU;
    using WaveSeg = pe::WaveSeg;
    using Paths = pe::Paths;
    int ordinal = 0;
    cudaStream_t stream = nullptr;
    cudaDeviceProp prop{};
    // scene
    std::vector<DevBuf> sceneBufs;
    SceneGPU scene{};
    bool hasScene = false;
    // adaptive sampling: the pixels still sampled (two lists), the clean-pixel mask, list sizes
    int32_t* adaptList[2] = {nullptr, nullptr};
    uint8_t* adaptClean = nullptr;
    uint32_t* adaptCount = nullptr;
    size_t adaptPixels = 0;
    int32_t lightGroups = 0;
    const pe_scene* sceneSrc = nullptr; // the scene last set, and its build version
    uint64_t sceneVersion = 0;
    size_t sceneMaterials = 0;
    size_t sceneLightNodes = 0;        // light groups of the scene set (its pass films need one each)
    TablesGPU* dTables = nullptr;
    TablesGPU hTables{};
    // pixel-filter inverse CDFs, one slot per (type, width) in use, least recently used replaced
    float* dFilters = nullptr;
    FilterSlot filterSlots[pe_dev::kFilterSlots];
    uint64_t filterClock = 0;
    // wavefront state: two lanes of `capacity` path slots each
    size_t capacity = 0;
    pe_dev::WaveLane lanes[2];
    int nextLane = 0;
    cudaEvent_t evFilm = nullptr;     // after the last film kernel of the render call
    int filmLane = -1;                // lane that recorded evFilm (-1: none yet)
    // [0] nodes, [1] tris (closest), [2] nodes, [3] tris (any), [4] rejected, [5] closest rays,
    // [6] shadow rays (both of the tail kernel), [7] paths ended at the per-path query bound
    unsigned long long* dStats = nullptr;
    // resident film
    int filmW = 0, filmH = 0;
    float* fSum = nullptr;
    uint32_t* fCnt = nullptr;
    float* fSq = nullptr;
    // timing
    cudaEvent_t evStart = nullptr, evStop = nullptr;
    cudaEvent_t evT0 = nullptr, evT1 = nullptr;
    std::vector<cudaEvent_t> evPool;
    bool counting = false;
    pe_render_stats stats{};
    int blocksIntersect = 0, blocksShade = 0, blocksShadow = 0, blocksGen = 0, blocksTail = 0;
    int blocksShadeKey[3][5] = {}; // lean shading kernels: [budget][key]
    int blocksShadowAny = 0;
    int blocksTailLockstep[2] = {}; // kTailLockstep<LEAN>: [0] full, [1] lean shading; 128-thread blocks
    int blocksIntersectMode[10] = {}; // per TraceMode
    size_t waveSlots = pe_dev::kDefaultWaveSlots; // pe_tuning::wave_slots: paths in flight per regenerating wave
    size_t laneSlots = 0;                 // slots of path state allocated per lane (>= capacity, waveSlots)
    int blocksShadowAnyOcc8 = 0;   // kShadow capped at 64 registers
    int blocksShadowAnyWindow = 0; // kShadow with the any-hit stack's top entries in registers
    int anyMode = 2;               // pe_tuning::any_traversal (default: the 64-register cap)
    // tuning (pe_tuning): closest-hit traversal variant, register budget of the lean shading kernels
    int closestMode = 6;  // TraceMode (default: TRACE_WIDE_OCC8, the autotuner's pick on the knot frame)
    int shadeBudget = 1;  // 0 the compiler's register count, 1 (default) at most 128 registers (4 blocks per SM)
    std::string tuneLog;  // the last autotune's probe times
    int64_t tailPaths = -1; // -1: one resident grid of the tail kernel; 0: no tail kernel
    unsigned char* noAllocBase = nullptr; // device address of g_noAllocScratch on this device
    void* stage = nullptr;                 // pinned staging of the batch film (host-film render)
    size_t stageBytes = 0;
    std::string noAllocError;
    pe_dev::GuideState guide;
    float* aovTarget = nullptr;     // AOV films of the render in progress (pe_device_render_aovs)
    float* aovFilm = nullptr;       // device AOV films (15 floats per pixel)
    size_t aovFilmPixels = 0;
    float* passTarget = nullptr;    // render-pass films of the render in progress (pe_device_render_passes)
    float* cryptoObj = nullptr;     // per-sample Cryptomatte ids of that render (or null)
    float* cryptoMat = nullptr;
    int32_t cryptoFirst = 0;
    int32_t passStride = 0;         // its per-path block (PASS_GROUPS + light groups)
    float* passFilm = nullptr;      // device pass films (5 floats per pixel per film)
    size_t passFilmFloats = 0;
    int guideKind = 0;      // 0 none, 1 learned proposal, 2 SD-tree
    pe_dev::SdHost sd;
    uint64_t sceneSerial = 0; // counts pe_device_set_scene calls
};


namespace pe_dev {

template <typename T>
int32_t devAlloc(std::vector<DevBuf>& list, T*& out, size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        setError(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaMsg(e));
        return e == cudaErrorMemoryAllocation ? PE_ERR_OOM : PE_ERR_CUDA;
    }
    list.push_back({p, bytes});
    out = static_cast<T*>(p);
    return PE_OK;
}

template <typename T>
int32_t upload(pe_device* d, std::vector<DevBuf>& list, const T*& dst, const std::vector<T>& src) {
    T* p = nullptr;
    const int32_t st = devAlloc(list, p, src.size());
    if (st) return st;
    if (!src.empty()) PE_CUDA(cudaMemcpyAsync(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, d->stream));
    dst = p;
    return PE_OK;
}

inline void freeList(std::vector<DevBuf>& list) {
    for (DevBuf& b : list) cudaFree(b.p);
    list.clear();
}

int32_t ensureCapacity(pe_device* d, size_t slots);
int32_t checkSettings(const pe_camera* cam, const pe_settings* st);
WaveSeg makeSeg(const pe_camera* cam, const pe_settings* st);
const float* filterTable(pe_device* d, int type, float width, uint64_t wave, cudaStream_t stream);
int32_t segsWritable(pe_device* d, int lane);
int32_t beginRender(pe_device* d);
int32_t endRender(pe_device* d, const RenderTimer& tm);
// One wave on `lane` over the nSegs segments in lanes[lane].hSegs, with path state `P` (the
// lane's own buffer, or the no-allocation scratch).
int32_t runWave(pe_device* d, int lane, Paths& P, int nSegs, int nSlots, int nPix, RenderTimer& tm);
// Uploads a built scene into device buffers owned by `bufs`; `out` gets their device view.
int32_t uploadScene(pe_device* d, const pe_scene* s, SceneGPU& out, std::vector<DevBuf>& bufs);
// Learned proposal in the wave loop (pe_guide.cu): the bounce's queries and their tensor-core
// inference, and after the film kernel the wave's training samples and one Adam step.
int32_t guideQueries(pe_device* d, cudaStream_t s, Paths& P, const Wave& W, const int32_t* queue, const uint32_t* count);
int32_t guideLearn(pe_device* d, cudaStream_t s, Paths& P, int nSlots);
// A continuous wave on one lane (the request server): paths are injected into the slots that
// ended paths free, bounce after bounce, until the server drains the lane with the tail kernel.
struct LaneLoop {
    WaveLane* ln = nullptr;  // the lane's path state, stream and readback buffers
    SceneGPU scene{};   // the wave's scene (each lane may trace its own)
    int32_t* qIn = nullptr;
    int32_t* qOut = nullptr;
    uint32_t* cIn = nullptr;
    uint32_t* cOut = nullptr;
    uint32_t live = 0;  // paths in the next closest-hit queue
    bool lean = false;  // the lean per-key shading kernels (a lean-shading scene, no segment with AO)
    int freeTop = 0;    // free slots on the stack
    int nextPath = 0;   // wave path index of the next injected path
    int pathCap = 0;    // paths the wave can hold (Lout)
    int iter = 0;
    // sweeps: paths alive for sweepAge bounces finish in tail-kernel launches on `side`
    static constexpr int kSweepBufs = 8;
    int sweepAge = 0;                    // 0: off
    int64_t sweepLive = 0;               // sweep only when the wave holds at most this many live paths (0: always)
    cudaStream_t side = nullptr;
    int32_t* born = nullptr;             // device, one per slot
    int32_t* sweepBuf[kSweepBufs] = {};  // device, one slot list per sweep in flight
    uint32_t* sweepCnt = nullptr;        // device [kSweepBufs]
    uint32_t* sweepCursor = nullptr;     // device [kSweepBufs]
    cudaEvent_t evReady[kSweepBufs] = {}, evDone[kSweepBufs] = {};
    int sweepN[kSweepBufs] = {};         // slots out in each sweep (0: buffer free)
    int sweeping = 0;                    // slots out in all sweeps
};
// Path state of `slots` slots (with regeneration buffers) for one lane.
int32_t allocLane(WaveLane& ln, size_t slots);
int32_t loopBegin(pe_device* d, LaneLoop& L, uint32_t* segLeft);
int32_t loopInject(pe_device* d, LaneLoop& L, const Wave& W, int fresh);
// One bounce; syncs the lane, then reads back the live count, the freed slots and the remaining
// path counts of segments [segFirst, segFirst + segCount).
int32_t loopBounce(pe_device* d, LaneLoop& L, const Wave& W, uint32_t* hSegLeft, const uint32_t* dSegLeft, int segFirst,
                   int segCount);
int32_t loopTail(pe_device* d, LaneLoop& L, const Wave& W);
// Returns the slots of finished sweeps to the free stack; with `wait`, waits for every sweep.
int32_t loopReturn(pe_device* d, LaneLoop& L, bool wait);
int32_t loopFilm(pe_device* d, LaneLoop& L, const WaveSeg* dSeg, int nPix);

// SD-tree guiding (pe_sdtree.cu): splats of a wave's recorded vertices; per-slot record buffers.
int32_t sdRecord(pe_device* d, cudaStream_t s, Paths& P, int nSlots);
int32_t sdBuffers(pe_device* d);
// The render's training schedule: a new field for a new scene or a render from sample 0; the end
// of the chunk of samples [cur, end) that runs under one field (waveMode set for its waves); the
// refinement once a chunk's samples bring the count to the next refinement point.
int32_t sdBeginRender(pe_device* d, int first);
int sdChunkEnd(pe_device* d, int cur, int end);
int32_t sdEndChunk(pe_device* d, int samples);

} // namespace pe_dev
