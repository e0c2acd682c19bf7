// pe_wave.h — the wavefront's data layout: per-path state columns in HBM, queue counters, and
// the segment table that lets several render requests share one wave.  Plain structs, so the
// host-side scheduler (compiled without device code) can build waves.
#pragma once

#include "pe_math.h"
#include "pe_sdtree.h"

#include <cstdint>
#include <vector_types.h>

namespace pe {

// Pinhole camera as PerspectiveCamera stores it (perspective_camera.cpp:36-40).
struct CamDev {
    V3 position, lowerLeft, horizontal, vertical;
    V3 u, v, forward;       // lens plane axes and view direction
    float lensRadius;       // > 0: thin lens
    int blades;             // thin lens: polygon aperture sides (0 = disk)
    float bladeRotation;    // radians
    int orthographic;
    // Camera::setShutterEnd: the description at shutter close (hasEnd = 0: none)
    int hasEnd;
    V3 position1, lowerLeft1, horizontal1, vertical1, u1, v1, forward1;
    float lensRadius1;
};

enum VisMask : uint32_t { VIS_CAMERA = 1u, VIS_DIFFUSE = 2u, VIS_GLOSSY = 4u, VIS_TRANSMISSION = 8u, VIS_SHADOW = 16u,
                          VIS_ALL = 0x1Fu };
// Marks a random-walk ray in the ray's mask word.  Triangle masks never carry it, so it does
// not change what the ray can hit; the closest-hit kernel bins such rays under their own key.
constexpr uint32_t RAY_WALK = 1u << 31;
constexpr int kMaxMediumEvents = 1024; // path_tracer.cpp:51
constexpr int kMaxWalkSteps = 256;     // path_tracer.cpp:52
// Closest-hit queries one path can make: at most 255 bounces, each preceded by up to 64 skipped
// camera-invisible hits and 65 pass-throughs and followed by up to 256 walk steps, plus 1025
// medium events, stays below this; a path that reaches it is counted as an error and ended.
constexpr int kMaxPathQueries = 1 << 17;

// path flags (bits of state word)
enum PathFlags : uint32_t {
    PF_SPECULAR_BOUNCE = 1u << 0,
    PF_CAMERA_RAY = 1u << 1,
    PF_PICKER_VALID = 1u << 2,
    PF_FIRST_SEGMENT = 1u << 3,
    PF_WALK = 1u << 4,   // inside a random walk: lastP = σt, lastN = albedo, pickP.x = g
    PF_GUIDE_SNAP = 1u << 5, // the path's guide training record waits for its radiance snapshot
};
// Bits 24..31 of the flags word: the light-link node of the path's last surface vertex.
constexpr uint32_t kPrevNodeShift = 24;
constexpr uint32_t kPrevNodeMask = 0xFFu << kPrevNodeShift;

// Per-slot state columns (capacity P slots).
struct Paths {
    float4* rayO;    // origin xyz, visibility mask (bits)
    float4* rayD;    // direction xyz, lastBsdfPdf
    float4* thr;     // throughput xyz, wavelength
    float4* L;       // radiance xyz, unused
    float4* lastN;   // last shading normal xyz, flags (bits)
    float4* lastP;   // last point xyz, Sobol dimension (bits)
    float4* pickP;   // light-picker point xyz, pixel hash (bits)
    float4* pickN;   // light-picker normal xyz, counters (bits: depth | diffuseBounces<<8 | passThroughs<<16 | skips<<24)
    float4* hit;     // t, u, v, leaf prim (bits)
    float* time;     // shutter time of the path's rays (read where the scene has moving instances)
    float4* med;     // media stack slots 0,1 | slots 2,3 (bits), mediumEvents | walkStep<<16, stack depth
    int32_t* queueA;
    int32_t* queueB;
    int32_t* shadowQ;
    float4* shO;     // shadow origin xyz, tMax
    float4* shD;     // shadow direction xyz, scalar (cos*w/(pdf*n))
    float4* shC;     // f*Li xyz, flags (bit0: indirect)
    float4* shT;     // throughput at NEE xyz
    int32_t* sortQ;  // kShadeKeys segments of `capacity` slots: rays binned by shading key
    // learned proposal (null / 0 when off)
    float4* guideQ;      // 3 per query row, compacted per bounce: hit point | shading normal | view direction
    int32_t* guideSlot;  // slot of each query row
    float4* guideOut;    // 10 per slot: the 40 network outputs of this bounce's proposal
    uint32_t* guideMark; // 1 = guideOut holds this bounce's proposal for the slot
    float4* guideRec;    // 6 per slot: training record of the first guidable vertex (see kGuideCollect)
    float4* trainBuf;    // 4 per training sample, compacted per wave
    int32_t guiding;     // 0 off, 1 record training samples, 2 record and sample with the proposal
    int32_t guideStride; // one slot in guideStride records a training sample (about 64K per wave)
    // SD-tree guiding (null / 0 when off)
    SdField sd;          // sampling trees (read), building trees (splats)
    int32_t sdMode;      // bit 0: record training vertices, bit 1: sample with the SD-tree
    float4* sdRec;       // kSdRecords × 4 per slot: (point, pdf) | (ω, 0) | (throughput after, 0) | (radiance snapshot, state)
    uint32_t* sdCount;   // recorded vertices per slot
    // path regeneration (null in a wave whose paths are its slots): a wave of more paths than
    // slots refills each slot freed by an ended path with the wave's next path
    int32_t* pathOf;     // wave path index held by each slot
    int32_t* freeQ;      // slots freed by the shading kernel this bounce
    float4* Lout;        // radiance of each ended path, by wave path index (read by the film kernel)
    uint32_t* segLeft;   // per segment: paths not yet ended (null unless the server tracks segments)
    // AOVs of each path (null unless requested): albedo + alpha, primary normal
    float4* aovA;
    float4* aovN;
    // render passes of each path (null unless requested): passStride float4 per path, laid out
    // as PassSlots says; shPass: 3 per shadow record, the lobe shares of a first-vertex NEE term
    float4* pass;
    float4* shPass;
    int32_t passStride;
    // ray cone of each slot's current ray: width, spread (null without; read only in scenes
    // with mipmapped textures)
    float2* cone;
    // sweeps (continuous waves): a path alive for sweepAge bounces leaves the wavefront for a
    // tail-kernel launch on a side stream (sweepAge 0: off)
    int32_t* born;       // bounce at which each slot's path was injected
    int32_t* sweepQ;     // this bounce's swept slots (counted in counters[CNT_SWEEP])
    int32_t sweepAge;
    int32_t iter;        // current bounce of the continuous wave
    uint32_t capacity;
    // [0] queue A count, [1] queue B count, [2] shadow count, [3] closest-hit work cursor,
    // [4] any-hit work cursor, [5] shade work cursor, [6..11] rays per shading key, [12] errors,
    // [13] tail work cursor, [14] guide query rows, [15] training samples
    uint32_t* counters;
};

// A path's render-pass block (float4 slots): the eight light passes (LightPass order), the
// lobe shares of the first bounce (firstLobe, path_tracer.cpp:375), the camera ray's origin and
// then the first hit (xyz, w = distance), the object and material id colours (w of the object
// slot: 1 on a hit), the Cryptomatte object and material ids of the hit, then one slot per
// light group.
enum PassSlots { PASS_DIFFUSE_DIRECT = 0, PASS_EMISSION = 6, PASS_BACKGROUND = 7, PASS_LOBES = 8, PASS_HIT = 11,
                 PASS_OBJECT = 12, PASS_MATERIAL = 13, PASS_CRYPTO = 14, PASS_GROUPS = 15 };
// Films of the pass target, 5 floats per pixel each (sum 3n, count n, sum of squares n).
enum PassFilms { PFILM_DEPTH = 8, PFILM_POSITION = 9, PFILM_OBJECT = 10, PFILM_MATERIAL = 11, PFILM_GROUPS = 12 };

// Shading keys: 0 = miss, 1 + material type (Lambert, Disney, Dielectric, Mirror), 5 = random-walk step.
constexpr int kShadeKeys = 6;
enum CounterSlots { CNT_QA = 0, CNT_QB = 1, CNT_SHADOW = 2, CNT_WORK_ISECT = 3, CNT_WORK_SHADOW = 4,
                    CNT_WORK_SHADE = 5, CNT_KEYS = 6, CNT_ERRORS = 12, CNT_WORK_TAIL = 13, CNT_GUIDE_Q = 14,
                    CNT_TRAIN = 15, CNT_FREE = 16, CNT_SWEEP = 17, CNT_WORK_KEYS = 18,
                    CNT_TOTAL = CNT_WORK_KEYS + kShadeKeys };
// Paths per wave with regeneration, as a multiple of the slots.
constexpr int kStreamFactor = 16;
// Vertices an SD-tree training path records (the reference records up to 32; its paths in these
// workloads rarely pass 8 guidable vertices).
constexpr int kSdRecords = 8;
enum SdModeBits { SD_RECORD = 1, SD_SAMPLE = 2 };
// Training samples of the learned proposal per wave (the record stride is chosen to give about this many).
constexpr int kGuideTrainRows = 1 << 16;

// One request's share of a wave: a rectangle of its film, a range of its sample indices and its
// render settings.  Wave slots [slotFirst, slotFirst + nPix·nSamples) are its paths, sample-major
// (slot = slotFirst + s·nPix + p), and its pixels are wave pixels [pixFirst, pixFirst + nPix).
struct WaveSeg {
    CamDev cam;
    int width, height;      // film
    int tileX, tileY, tileW; // rendered rectangle of the film (whole frame: 0, 0, width)
    const int32_t* pixList;  // film pixel (y·width + x) of each tile-linear pixel, or null: the rectangle
    int pixelFirst, nPix;   // range of tile-linear pixel indices in this wave
    int sampleFirst, nSamples;
    uint64_t seed;
    float filterWidth;
    int maxDepth, rrDepth, shadowSamples;
    float clampIndirect;
    const float* filterCdf; // inverse-CDF table of the request's pixel filter
    float* sum;             // the request's film on the device
    uint32_t* cnt;
    float* sq;
    float* aov;             // AOV films (albedo, normal, alpha: each sum 3n, count n, sum of squares n), or null
    float* pass;            // render-pass films (PassFilms order, 5n floats each), or null
    float* cryptoObj;       // Cryptomatte ids per (sample − cryptoFirst, film pixel), or null
    float* cryptoMat;
    int cryptoFirst;
    int slotFirst;
    int pixFirst;
    int flags;              // SegFlags
    float aoStrength;       // RenderSettings::aoStrength (contact AO at camera hits)
    float coneWidth, coneSpread; // camera rays' cone (Camera::pixelConeWidth / pixelConeSpread)
};
// SEG_SWEEP: paths of the segment may leave a continuous wave for a sweep; SEG_MOTION:
// RenderSettings::motionBlur (each camera sample draws a shutter time)
enum SegFlags { SEG_SWEEP = 1, SEG_MOTION = 2 };

// The segments of one wave, ordered by slotFirst (and so by pixFirst).
struct Wave {
    const WaveSeg* segs;
    int nSegs;
    int nSlots;
    int nPix;
};

#ifdef __CUDACC__
// Wave path index held by a slot.
__device__ __forceinline__ int pathOfSlot(const Paths& P, int slot) { return P.pathOf ? P.pathOf[slot] : slot; }
// Segment owning a wave path / a wave pixel (binary search; one segment for a lone request).
__device__ __forceinline__ int segOfSlot(const Wave& W, int slot) {
    int lo = 0, hi = W.nSegs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (W.segs[mid].slotFirst <= slot) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int segOfPixel(const Wave& W, int p) {
    int lo = 0, hi = W.nSegs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (W.segs[mid].pixFirst <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

#endif

} // namespace pe
