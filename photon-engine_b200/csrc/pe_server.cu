// pe_server.cu — the request server behind the pe_server_* C ABI: resident scenes, device films
// admitted against an HBM budget, and continuous waves that take in new requests' paths as the
// paths in flight end (continuous batching at path granularity).
//
// Four lanes, each driven by its own host thread and running one scene's continuous wave at a
// time: the device's two lanes take the bulk requests, and two express lanes of their own path
// state on high-priority streams take the interactive ones (at most 8M paths, or a priority above
// 0; two, so that interactive requests of two scenes need not wait for each other); while an
// express lane runs, the bulk lanes pause between bounces, so the GPU goes to the interactive
// requests (stream priority alone does not preempt the bulk lanes' persistent kernels).  After every bounce the slots of ended paths hand their radiance to
// the wave's per-path buffer and return to a free stack; the lane then injects the next paths of
// the admitted requests of its scene, ordered by (priority desc, remaining paths asc, id asc).
// A request's paths are planned as segments — whole-frame sample rows [s, s+k), or a pixel range
// of one row — in increasing sample order, and each segment is added to the request's film once
// all its paths have ended, in segment order, so every pixel adds its samples in the order a
// lone render does and the film is bit-identical to pe_device_render's.
//
// A lane drains its wave (stops injecting, finishes the last paths with the tail kernel) when
// its scene has no more work, when its path buffer is used up, or (bulk lanes) when a request of
// a scene no lane is tracing outranks its own best pending request; the lane then starts a wave
// of the best-ranked waiting scene.  A request is bound to one lane while it has segments in
// flight.  Interactive paths that stay in a wave for 4 (express lanes) or 8 bounces finish in tail-kernel sweeps on a
// side stream, so an interactive request does not wait one wavefront step per bounce of its
// longest paths.

#include "pe_device_impl.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

using namespace pe;
using namespace pe_dev;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    int32_t scene = 0;
    pe_camera cam{};
    pe_settings st{};
    int32_t spp = 0;
    int32_t priority = 0;
    int32_t state = PE_REQ_QUEUED;
    int32_t error = PE_OK;
    std::string message; // of a failed request
    float* sum = nullptr;
    uint32_t* cnt = nullptr;
    float* sq = nullptr;
    size_t filmBytes = 0;
    int32_t sampleCursor = 0; // next sample row to hand out
    int32_t pixelCursor = 0;  // > 0 while a row is split over several waves
    int32_t samplesDone = 0;
    uint64_t paths = 0;
    const float* filterCdf = nullptr; // the server's device table of its pixel filter
    int32_t lane = -1;        // the lane holding its segments in flight (-1: none)
    int32_t openSegs = 0;     // segments planned and not yet added to the film
    double submitMs = 0.0, startMs = 0.0, doneMs = 0.0;
    double firstPathMs = -1.0, lastPathMs = -1.0, filmMs = -1.0; // trace: injections, last film kernel

    int64_t pixels() const { return static_cast<int64_t>(st.width) * st.height; }
    int64_t remaining() const { return (static_cast<int64_t>(spp) - sampleCursor) * pixels() - pixelCursor; }
};

struct ResidentScene {
    SceneGPU gpu{};
    std::vector<DevBuf> bufs;
    size_t bytes = 0;
};

// One planned segment of a continuous wave.
struct SegInfo {
    int64_t id;         // request
    int32_t samples;    // whole rows it completes (a split row's last pixel range completes 1)
    int32_t nPix;
    bool filmed;
};

constexpr int kServerSegs = 16384;      // segments per continuous wave
constexpr int kMinChunk = 4096;         // smallest segment unless it finishes a request
constexpr int kSweepAge = 8;            // bounces after which an interactive path leaves a bulk wave for a sweep
constexpr int kExpressSweepAge = 4;     // the same on the express lanes
constexpr size_t kExpressSlots = (size_t(1) << 22) + (size_t(1) << 20); // a 512² × 16-spp preview in one go
constexpr int64_t kUrgentPaths = 8 << 20; // requests of at most this many paths are interactive (512² × 16 spp: 4.2M)

size_t filmBytesOf(const pe_settings& st) {
    return static_cast<size_t>(st.width) * static_cast<size_t>(st.height) * (3 * sizeof(float) + sizeof(uint32_t) + sizeof(float));
}

} // namespace

struct pe_server {
    pe_device* d = nullptr;
    uint64_t budget = 0;
    uint64_t sceneBytes = 0, filmBytes = 0, filmPeak = 0;
    std::vector<ResidentScene> scenes;
    std::map<int64_t, Request> requests;
    std::deque<int64_t> queued;
    std::vector<int64_t> active;
    int64_t nextId = 0;
    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    std::thread worker;
    bool stop = false;
    std::thread watcher;             // marks requests done as soon as their film kernels have run
    Clock::time_point t0;
    SceneGPU savedScene{};
    bool savedHasScene = false;
    cudaStream_t copyStream = nullptr;
    cudaStream_t admitStream = nullptr; // film allocation and clearing
    cudaEvent_t evAdmit = nullptr;   // after the film allocations of the last admission
    FILE* trace = nullptr;           // PE_SERVER_TRACE: one line per finished request and per wave
    // pixel-filter tables, one per (type, width) in use; kept until the server is destroyed, as
    // paths of a continuous wave may read them at any later bounce
    std::map<std::pair<int, float>, float*> filters;
    pe_server_stats stats{};
    // one continuous wave per lane, each driven by its own thread
    struct LaneRun {
        std::thread th;
        WaveSeg* hSegs = nullptr;     // pinned segment table
        WaveSeg* dSegs = nullptr;
        uint32_t* hLeft = nullptr;    // pinned: paths left per segment (read back)
        uint32_t* hInit = nullptr;    // pinned: initial counts (uploaded)
        uint32_t* dLeft = nullptr;
        std::vector<SegInfo> segs;
        int scene = -1;
        bool running = false;
        bool draining = false;        // taking in no paths: the wave ends once its live paths fit the tail kernel
        bool yielding = false;        // draining so that another scene gets this lane
        int firstOpen = 0;            // first segment not yet filmed
        int aoChecked = 0;            // segments looked at for contact AO
        bool anyAo = false;           // some segment of the wave has contact AO (full shading kernel)
        int uploaded = 0;             // segments on the device
        LaneLoop loop;
        WaveLane own;                 // the express lane's own path state (bulk lanes use the device's)
        cudaStream_t stream = nullptr;
        std::vector<int64_t> doneAfterSync; // requests whose last film kernel is queued (no event free)
        std::vector<std::pair<int64_t, cudaEvent_t>> doneEvents; // ... with an event after it
        std::vector<cudaEvent_t> eventPool;
        cudaEvent_t evStart = nullptr, evEnd = nullptr;
    } lanes[4];

    double now() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

// The server's table of a pixel filter, uploaded at its first use (lock held).
const float* serverFilter(pe_server* S, int type, float width) {
    const auto key = std::make_pair(type, width);
    auto it = S->filters.find(key);
    if (it != S->filters.end()) return it->second;
    float cdf[kFilterBins + 1];
    fillFilterCdf(type, width, cdf);
    float* dev = nullptr;
    if (cudaMalloc(&dev, sizeof(cdf)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(dev, cdf, sizeof(cdf), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(dev);
        return nullptr;
    }
    S->filters[key] = dev;
    return dev;
}

// Gives films to queued requests, in priority order, while the budget has room.  Called with
// the lock held, on the worker thread.
bool admit(pe_server* S) {
    bool any = false;
    std::stable_sort(S->queued.begin(), S->queued.end(), [&](int64_t a, int64_t b) {
        const Request& ra = S->requests[a];
        const Request& rb = S->requests[b];
        if (ra.priority != rb.priority) return ra.priority > rb.priority;
        return ra.remaining() < rb.remaining();
    });
    for (auto it = S->queued.begin(); it != S->queued.end();) {
        Request& r = S->requests[*it];
        if (S->sceneBytes + S->filmBytes + r.filmBytes > S->budget) {
            ++it;
            continue;
        }
        const size_t n = static_cast<size_t>(r.pixels());
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, r.filmBytes, S->admitStream);
        if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, r.filmBytes, S->admitStream);
        if (e != cudaSuccess) {
            r.state = PE_REQ_FAILED;
            r.error = e == cudaErrorMemoryAllocation ? PE_ERR_OOM : PE_ERR_CUDA;
            r.doneMs = S->now();
            ++S->stats.failed;
            it = S->queued.erase(it);
            S->cvDone.notify_all();
            continue;
        }
        r.filterCdf = serverFilter(S, r.st.filter_type, r.st.filter_width);
        if (!r.filterCdf) {
            cudaFreeAsync(p, S->admitStream);
            r.state = PE_REQ_FAILED;
            r.error = PE_ERR_CUDA;
            r.message = "pixel filter table upload failed";
            r.doneMs = S->now();
            ++S->stats.failed;
            it = S->queued.erase(it);
            S->cvDone.notify_all();
            continue;
        }
        r.sum = static_cast<float*>(p);
        r.cnt = reinterpret_cast<uint32_t*>(r.sum + 3 * n);
        r.sq = reinterpret_cast<float*>(r.cnt + n);
        r.state = PE_REQ_ACTIVE;
        r.startMs = S->now();
        S->filmBytes += r.filmBytes;
        S->filmPeak = std::max(S->filmPeak, S->filmBytes);
        S->active.push_back(r.id);
        it = S->queued.erase(it);
        any = true;
    }
    return any;
}

bool ranksBefore(const Request& a, const Request& b) {
    if (a.priority != b.priority) return a.priority > b.priority;
    if (a.remaining() != b.remaining()) return a.remaining() < b.remaining();
    return a.id < b.id;
}

bool hasWork(const Request& r) { return r.state == PE_REQ_ACTIVE && r.sampleCursor < r.spp; }

bool urgent(const Request& r) { return r.priority > 0 || static_cast<int64_t>(r.spp) * r.pixels() <= kUrgentPaths; }

constexpr int kLanes = 4;
// lanes 0 and 1 trace bulk requests on the device's lanes, 2 and 3 are the express lanes
bool express(int li) { return li >= 2; }

// Whether an express lane is running (lock held): the bulk lanes then take in nothing.
bool expressBusy(pe_server* S) {
    for (int li = 2; li < kLanes; ++li)
        if (S->lanes[li].running) return true;
    return false;
}

// Whether lane `li` may take request `r` (lock held): the express lane takes the interactive
// requests; a bulk lane takes the others, and an interactive one of its own scene while the
// express lane is busy with another scene.
bool eligible(pe_server* S, int li, const Request& r) {
    if (r.lane >= 0 && r.lane != li) return false;
    if (express(li)) return urgent(r);
    if (!urgent(r)) return true;
    // an interactive request of this bulk lane's scene while both express lanes trace others
    for (int x = 2; x < kLanes; ++x)
        if (!S->lanes[x].running || S->lanes[x].scene == r.scene) return false;
    return S->lanes[li].running && S->lanes[li].scene == r.scene;
}

// The best-ranked admitted request with rows left that lane `li` may take (lock held).
const Request* bestFor(pe_server* S, int li, int scene) {
    const Request* best = nullptr;
    for (int64_t id : S->active) {
        const Request& r = S->requests[id];
        if (!hasWork(r) || !eligible(S, li, r) || (scene >= 0 && r.scene != scene)) continue;
        if (!best || ranksBefore(r, *best)) best = &r;
    }
    return best;
}

// Whether bulk lane `li` should stop taking paths so that a waiting scene gets a lane (lock
// held): a bulk request of a scene that no running bulk lane traces outranks this lane's best
// pending one, and the other bulk lane is not already making room.
bool yieldLane(pe_server* S, int li) {
    if (express(li)) return false;
    const auto& me = S->lanes[li];
    const auto& other = S->lanes[li ^ 1];
    if (other.running && other.draining) return false;
    if (!other.running) return false; // the idle bulk lane will take it
    const Request* mine = bestFor(S, li, me.scene);
    const Request* waiting = nullptr;
    for (int64_t id : S->active) {
        const Request& r = S->requests[id];
        if (!hasWork(r) || r.lane >= 0 || urgent(r)) continue;
        if (r.scene == me.scene || r.scene == other.scene) continue;
        if (!waiting || ranksBefore(r, *waiting)) waiting = &r;
    }
    return waiting && (!mine || ranksBefore(*waiting, *mine));
}

// Plans up to `budget` paths of lane `li`'s scene as new segments (lock held); returns the paths.
int planPaths(pe_server* S, int li, int budget) {
    auto& R = S->lanes[li];
    std::vector<int64_t> order;
    for (int64_t id : S->active) {
        const Request& r = S->requests[id];
        if (hasWork(r) && r.scene == R.scene && eligible(S, li, r)) order.push_back(id);
    }
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return ranksBefore(S->requests[a], S->requests[b]); });
    int planned = 0;
    for (int64_t id : order) {
        Request& r = S->requests[id];
        while (r.sampleCursor < r.spp) {
            const int room = budget - planned;
            const int64_t npix = r.pixels();
            const int64_t left = r.remaining();
            if (room < std::min<int64_t>(kMinChunk, left)) return planned;
            if (static_cast<int>(R.segs.size()) >= kServerSegs) return planned;
            WaveSeg seg = makeSeg(&r.cam, &r.st);
            seg.filterCdf = r.filterCdf;
            seg.tileX = 0;
            seg.tileY = 0;
            seg.tileW = r.st.width;
            seg.sum = r.sum;
            seg.cnt = r.cnt;
            seg.sq = r.sq;
            seg.slotFirst = R.loop.nextPath + planned;
            seg.pixFirst = 0;
            seg.flags = (seg.flags & SEG_MOTION) | (urgent(r) ? SEG_SWEEP : 0);
            SegInfo info{id, 0, 0, false};
            if (r.pixelCursor == 0 && npix <= room) {
                const int64_t rows = std::min<int64_t>(r.spp - r.sampleCursor, room / npix);
                seg.pixelFirst = 0;
                seg.nPix = static_cast<int>(npix);
                seg.sampleFirst = r.sampleCursor;
                seg.nSamples = static_cast<int>(rows);
                r.sampleCursor += static_cast<int32_t>(rows);
                info.samples = static_cast<int32_t>(rows);
            } else {
                const int64_t take = std::min<int64_t>(npix - r.pixelCursor, room);
                seg.pixelFirst = r.pixelCursor;
                seg.nPix = static_cast<int>(take);
                seg.sampleFirst = r.sampleCursor;
                seg.nSamples = 1;
                r.pixelCursor += static_cast<int32_t>(take);
                if (r.pixelCursor == npix) {
                    r.pixelCursor = 0;
                    r.sampleCursor += 1;
                    info.samples = 1;
                }
            }
            info.nPix = seg.nPix;
            const int paths = seg.nPix * seg.nSamples;
            const int k = static_cast<int>(R.segs.size());
            R.hSegs[k] = seg;
            R.hInit[k] = static_cast<uint32_t>(paths);
            R.segs.push_back(info);
            r.lane = li;
            ++r.openSegs;
            if (r.firstPathMs < 0.0) r.firstPathMs = S->now();
            r.lastPathMs = S->now();
            r.paths += static_cast<uint64_t>(paths);
            planned += paths;
            ++S->stats.segments;
        }
    }
    return planned;
}

// Adds every completed segment to its request's film, in order (lock held, after a lane sync:
// hLeft holds the counts read back).  `all`: the wave has ended, every segment is complete.
int32_t filmSegments(pe_server* S, int li, bool all) {
    auto& R = S->lanes[li];
    const cudaStream_t cs = R.stream;
    bool waited = false;
    std::map<int64_t, bool> blocked; // a request with an earlier segment not yet complete
    for (int k = R.firstOpen; k < static_cast<int>(R.segs.size()); ++k) {
        SegInfo& g = R.segs[k];
        if (g.filmed) continue;
        if (blocked.count(g.id)) continue;
        if (!all && R.hLeft[k] != 0u) {
            blocked[g.id] = true;
            continue;
        }
        if (!waited) {
            // films are allocated and cleared on the admission stream: film kernels come after
            if (cudaStreamWaitEvent(cs, S->evAdmit, 0) != cudaSuccess) return PE_ERR_CUDA;
            waited = true;
        }
        int32_t rc = loopFilm(S->d, R.loop, R.dSegs + k, g.nPix);
        if (rc) return rc;
        g.filmed = true;
        Request& r = S->requests[g.id];
        r.samplesDone += g.samples;
        --r.openSegs;
        if (r.samplesDone >= r.spp) {
            r.filmMs = S->now();
            // done once the film kernel has run: an event after it, polled by the lane
            if (!R.eventPool.empty() && cudaEventRecord(R.eventPool.back(), cs) == cudaSuccess) {
                R.doneEvents.emplace_back(g.id, R.eventPool.back());
                R.eventPool.pop_back();
            } else {
                R.doneAfterSync.push_back(g.id);
            }
        }
    }
    while (R.firstOpen < static_cast<int>(R.segs.size()) && R.segs[R.firstOpen].filmed) ++R.firstOpen;
    return PE_OK;
}

// Requests whose film kernels have run (lock held, after a lane sync).
void settleDone(pe_server* S, int li) {
    auto& R = S->lanes[li];
    const double t = S->now();
    for (size_t k = 0; k < R.doneEvents.size();) {
        if (cudaEventQuery(R.doneEvents[k].second) != cudaSuccess) {
            ++k;
            continue;
        }
        R.doneAfterSync.push_back(R.doneEvents[k].first);
        R.eventPool.push_back(R.doneEvents[k].second);
        R.doneEvents.erase(R.doneEvents.begin() + static_cast<long>(k));
    }
    for (int64_t id : R.doneAfterSync) {
        Request& r = S->requests[id];
        if (r.state != PE_REQ_ACTIVE) continue;
        r.state = PE_REQ_DONE;
        r.doneMs = t;
        ++S->stats.completed;
        if (S->trace)
            std::fprintf(S->trace, "request %lld scene %d paths %llu lane %d submit %.2f admit %.2f first %.2f last %.2f film %.2f done %.2f\n",
                         static_cast<long long>(r.id), r.scene, static_cast<unsigned long long>(r.paths), li, r.submitMs,
                         r.startMs, r.firstPathMs, r.lastPathMs, r.filmMs, r.doneMs);
        r.lane = -1;
    }
    if (!R.doneAfterSync.empty()) {
        R.doneAfterSync.clear();
        S->active.erase(std::remove_if(S->active.begin(), S->active.end(),
                                       [&](int64_t id) { return S->requests[id].state != PE_REQ_ACTIVE; }),
                        S->active.end());
        S->cvDone.notify_all();
        S->cvWork.notify_all();
    }
}

// A lane's wave failed: its requests fail with it (lock held).
void failLane(pe_server* S, int li, int32_t rc, const std::string& msg) {
    auto& R = S->lanes[li];
    const double t = S->now();
    for (int64_t id : S->active) {
        Request& r = S->requests[id];
        if (r.lane != li || r.state != PE_REQ_ACTIVE) continue;
        r.state = PE_REQ_FAILED;
        r.error = rc;
        r.message = msg;
        r.doneMs = t;
        ++S->stats.failed;
    }
    S->active.erase(std::remove_if(S->active.begin(), S->active.end(),
                                   [&](int64_t id) { return S->requests[id].state != PE_REQ_ACTIVE; }),
                    S->active.end());
    R.running = false;
    R.draining = false;
    R.yielding = false;
    R.segs.clear();
    R.firstOpen = 0;
    R.uploaded = 0;
    R.doneAfterSync.clear();
    S->cvDone.notify_all();
    S->cvWork.notify_all();
}

// Ends lane `li`'s wave (lock not held): the last live paths run to their end in the tail
// kernel, every segment goes to its film, and the lane is free for another scene.
int32_t endWave(pe_server* S, int li, const Wave& W) {
    auto& R = S->lanes[li];
    pe_device* d = S->d;
    int32_t rc = loopReturn(d, R.loop, true);
    if (rc == PE_OK) rc = loopTail(d, R.loop, W);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        rc = filmSegments(S, li, true);
    }
    if (rc) return rc;
    const cudaStream_t cs = R.stream;
    if (cudaEventRecord(R.evEnd, cs) != cudaSuccess || cudaStreamSynchronize(cs) != cudaSuccess) return PE_ERR_CUDA;
    std::lock_guard<std::mutex> lk(S->mu);
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, R.evStart, R.evEnd) == cudaSuccess) S->stats.busy_ms += ms;
    if (S->trace)
        std::fprintf(S->trace, "wave lane %d scene %d paths %d segments %zu bounces %d device_ms %.2f end %.2f yield %d\n", li,
                     R.scene, R.loop.nextPath, R.segs.size(), R.loop.iter, ms, S->now(), R.yielding ? 1 : 0);
    settleDone(S, li);
    for (int64_t id : S->active) {
        Request& r = S->requests[id];
        if (r.lane == li && r.openSegs == 0) r.lane = -1; // free to continue on either lane
    }
    R.running = false;
    R.draining = false;
    R.yielding = false;
    R.segs.clear();
    R.firstOpen = 0;
    R.uploaded = 0;
    S->cvWork.notify_all();
    return PE_OK;
}

void laneThread(pe_server* S, int li) {
    pe_device* d = S->d;
    cudaSetDevice(d->ordinal);
    auto& R = S->lanes[li];
    const cudaStream_t cs = R.stream;
    // the express lane hands its last paths to the tail kernel earlier: latency over efficiency
    const int64_t tailPaths = pe_device_tail_paths(d) * (express(li) ? 4 : 1);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        if (S->stop) break;
        settleDone(S, li);
        if (admit(S)) cudaEventRecord(S->evAdmit, S->admitStream);
        if (!R.running) {
            const Request* best = bestFor(S, li, -1);
            if (!best) {
                S->cvWork.wait_for(lk, std::chrono::milliseconds(5));
                continue;
            }
            R.scene = best->scene;
            R.running = true;
            R.draining = false;
            R.yielding = false;
            R.segs.clear();
            R.firstOpen = 0;
            R.aoChecked = 0;
            R.anyAo = false;
            R.uploaded = 0;
            R.loop.scene = S->scenes[static_cast<size_t>(R.scene)].gpu;
            ++S->stats.waves;
            lk.unlock();
            int32_t rc = loopBegin(d, R.loop, R.dLeft);
            if (rc == PE_OK && cudaEventRecord(R.evStart, cs) != cudaSuccess) rc = PE_ERR_CUDA;
            lk.lock();
            if (rc) {
                failLane(S, li, rc, pe_last_error());
                continue;
            }
        }
        LaneLoop& L = R.loop;
        int fresh = 0;
        if (!express(li) && expressBusy(S)) {
            // an express lane runs: this bulk lane launches nothing, so that the interactive
            // requests' kernels get every SM (running blocks are not preempted by priority);
            // the express lanes notify when their waves end
            S->cvWork.wait_for(lk, std::chrono::milliseconds(20), [&] { return S->stop || !expressBusy(S); });
            continue;
        }
        {
            // slots of finished sweeps are free again
            const int32_t rr = loopReturn(d, L, false);
            if (rr) {
                failLane(S, li, rr, pe_last_error());
                continue;
            }
        }
        // making room for a waiting scene is final; running out of work is not (requests of
        // this scene that arrive meanwhile are taken in while the wave has room)
        if (!R.yielding && yieldLane(S, li)) R.yielding = true;
        const bool room = L.pathCap - L.nextPath >= kMinChunk && static_cast<int>(R.segs.size()) < kServerSegs;
        if (!R.yielding && room) {
            fresh = planPaths(S, li, std::min(L.freeTop, L.pathCap - L.nextPath));
            S->stats.paths += static_cast<uint64_t>(fresh);
        }
        R.draining = R.yielding || !room || !bestFor(S, li, R.scene);
        const int nSegs = static_cast<int>(R.segs.size());
        for (; R.aoChecked < nSegs; ++R.aoChecked)
            if (R.hSegs[R.aoChecked].aoStrength > 0.0f) R.anyAo = true;
        L.lean = L.scene.leanShading && !R.anyAo;
        const int upFirst = R.uploaded;
        R.uploaded = nSegs;
        const bool draining = R.draining;
        const int open = R.firstOpen;
        lk.unlock();
        int32_t rc = PE_OK;
        const Wave W{R.dSegs, std::max(1, nSegs), L.nextPath + fresh, 0};
        if (nSegs > upFirst) {
            const size_t n = static_cast<size_t>(nSegs - upFirst);
            if (cudaMemcpyAsync(R.dSegs + upFirst, R.hSegs + upFirst, n * sizeof(WaveSeg), cudaMemcpyHostToDevice, cs) !=
                    cudaSuccess ||
                cudaMemcpyAsync(R.dLeft + upFirst, R.hInit + upFirst, n * sizeof(uint32_t), cudaMemcpyHostToDevice, cs) !=
                    cudaSuccess)
                rc = PE_ERR_CUDA;
        }
        if (rc == PE_OK) rc = loopInject(d, L, W, fresh);
        bool ended = false;
        if (rc == PE_OK && (L.live == 0 || (draining && static_cast<int64_t>(L.live) <= tailPaths))) {
            if (L.live == 0 && !draining) {
                // nothing in flight and nothing to inject yet: wait for work
                lk.lock();
                S->cvWork.wait_for(lk, std::chrono::milliseconds(1));
                continue;
            }
            rc = endWave(S, li, W);
            ended = true;
        } else if (rc == PE_OK) {
            rc = loopBounce(d, L, W, R.hLeft, R.dLeft, open, nSegs - open);
        }
        const std::string msg = rc == PE_OK ? std::string() : std::string(pe_last_error());
        lk.lock();
        if (rc) {
            failLane(S, li, rc, msg);
            continue;
        }
        if (ended) continue;
        settleDone(S, li);
        rc = filmSegments(S, li, false);
        if (rc) failLane(S, li, rc, "film kernel launch failed");
    }
    lk.unlock();
    cudaStreamSynchronize(cs);
}

// Polls the lanes' completion events every 0.2 ms, so that a request is done (and its waiters
// wake) when its last film kernel has run, not when its lane next returns from a bounce.
void watchThread(pe_server* S) {
    cudaSetDevice(S->d->ordinal);
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->stop) return;
            for (int li = 0; li < kLanes; ++li)
                if (!S->lanes[li].doneEvents.empty()) settleDone(S, li);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
}

// Frees the server's streams, events and segment tables, then the server.
void releaseServer(pe_server* S) {
    if (S->trace) std::fclose(S->trace);
    if (S->copyStream) cudaStreamDestroy(S->copyStream);
    if (S->admitStream) cudaStreamDestroy(S->admitStream);
    if (S->evAdmit) cudaEventDestroy(S->evAdmit);
    for (auto& kv : S->filters) cudaFree(kv.second);
    for (auto& R : S->lanes) {
        if (R.evStart) cudaEventDestroy(R.evStart);
        if (R.evEnd) cudaEventDestroy(R.evEnd);
        if (R.hSegs) cudaFreeHost(R.hSegs);
        if (R.hLeft) cudaFreeHost(R.hLeft);
        if (R.hInit) cudaFreeHost(R.hInit);
        if (R.dSegs) cudaFree(R.dSegs);
        if (R.dLeft) cudaFree(R.dLeft);
        for (cudaEvent_t ev : R.eventPool) cudaEventDestroy(ev);
        for (auto& pe : R.doneEvents) cudaEventDestroy(pe.second);
        if (R.own.stream) {
            cudaStreamSynchronize(R.own.stream);
            freeList(R.own.bufs);
            cudaStreamDestroy(R.own.stream);
        }
        if (R.own.hCounters) cudaFreeHost(R.own.hCounters);
        LaneLoop& L = R.loop;
        if (L.side) {
            cudaStreamSynchronize(L.side);
            cudaStreamDestroy(L.side);
        }
        if (L.born) cudaFree(L.born);
        if (L.sweepCnt) cudaFree(L.sweepCnt);
        if (L.sweepCursor) cudaFree(L.sweepCursor);
        for (int b = 0; b < LaneLoop::kSweepBufs; ++b) {
            if (L.sweepBuf[b]) cudaFree(L.sweepBuf[b]);
            if (L.evReady[b]) cudaEventDestroy(L.evReady[b]);
            if (L.evDone[b]) cudaEventDestroy(L.evDone[b]);
        }
    }
    delete S;
}

pe_server* failCreate(char* err, size_t n, const std::string& msg) {
    setError(msg);
    if (err && n) {
        std::strncpy(err, msg.c_str(), n - 1);
        err[n - 1] = '\0';
    }
    return nullptr;
}

} // namespace

extern "C" {

pe_server* pe_server_create(pe_device* d, uint64_t budget, char* err, size_t errLen) {
    if (!d) return failCreate(err, errLen, "pe_server_create: null device");
    if (cudaSetDevice(d->ordinal) != cudaSuccess) return failCreate(err, errLen, "pe_server_create: cudaSetDevice failed");
    if (ensureCapacity(d, kWaveSlots) != PE_OK) return failCreate(err, errLen, std::string("pe_server_create: ") + pe_last_error());
    cudaStreamSynchronize(d->stream);
    pe_server* S = new pe_server();
    S->d = d;
    S->budget = budget;
    S->t0 = Clock::now();
    S->savedScene = d->scene;
    S->savedHasScene = d->hasScene;
    S->stats.budget_bytes = budget;
    bool ok = cudaStreamCreateWithFlags(&S->copyStream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&S->admitStream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&S->evAdmit, cudaEventDisableTiming) == cudaSuccess;
    int loPrio = 0, hiPrio = 0;
    cudaDeviceGetStreamPriorityRange(&loPrio, &hiPrio);
    for (int li = 0; li < kLanes && ok; ++li) {
        auto& R = S->lanes[li];
        if (express(li)) {
            // the express lane: its own path state, on the highest-priority streams
            ok = cudaStreamCreateWithPriority(&R.own.stream, cudaStreamNonBlocking, hiPrio) == cudaSuccess &&
                 cudaMallocHost(&R.own.hCounters, 32 * sizeof(uint32_t)) == cudaSuccess &&
                 allocLane(R.own, kExpressSlots) == PE_OK;
            R.loop.ln = &R.own;
        } else {
            R.loop.ln = &d->lanes[li];
        }
        R.stream = R.loop.ln->stream;
        for (int e = 0; e < 64 && ok; ++e) {
            cudaEvent_t ev = nullptr;
            ok = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
            if (ok) R.eventPool.push_back(ev);
        }
        ok = ok && cudaEventCreate(&R.evStart) == cudaSuccess && cudaEventCreate(&R.evEnd) == cudaSuccess &&
             cudaMallocHost(&R.hSegs, kServerSegs * sizeof(WaveSeg)) == cudaSuccess &&
             cudaMallocHost(&R.hLeft, kServerSegs * sizeof(uint32_t)) == cudaSuccess &&
             cudaMallocHost(&R.hInit, kServerSegs * sizeof(uint32_t)) == cudaSuccess &&
             cudaMalloc(&R.dSegs, kServerSegs * sizeof(WaveSeg)) == cudaSuccess &&
             cudaMalloc(&R.dLeft, kServerSegs * sizeof(uint32_t)) == cudaSuccess;
        LaneLoop& L = R.loop;
        const size_t cap = ok ? R.loop.ln->paths.capacity : 0;
        L.sweepAge = express(li) ? kExpressSweepAge : kSweepAge;
        // an express wave holds only interactive paths: sweeping millions of them into the tail
        // kernel (one thread per path) would be slower than their wavefront bounces, so it sweeps
        // only the stragglers of a wave that has shrunk to a few tail grids
        L.sweepLive = express(li) ? 4 * pe_device_tail_paths(d) : 0;
        ok = ok && cudaStreamCreateWithPriority(&L.side, cudaStreamNonBlocking, express(li) ? hiPrio : loPrio) == cudaSuccess &&
             cudaMalloc(&L.born, cap * sizeof(int32_t)) == cudaSuccess &&
             cudaMalloc(&L.sweepCnt, LaneLoop::kSweepBufs * sizeof(uint32_t)) == cudaSuccess &&
             cudaMalloc(&L.sweepCursor, LaneLoop::kSweepBufs * sizeof(uint32_t)) == cudaSuccess;
        for (int b = 0; b < LaneLoop::kSweepBufs; ++b)
            ok = ok && cudaMalloc(&L.sweepBuf[b], cap * sizeof(int32_t)) == cudaSuccess &&
                 cudaEventCreateWithFlags(&L.evReady[b], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&L.evDone[b], cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        releaseServer(S);
        return failCreate(err, errLen, "pe_server_create: stream, event or segment table allocation failed");
    }
    d->filmLane = -1;
    if (const char* tp = std::getenv("PE_SERVER_TRACE")) S->trace = std::fopen(tp, "w");
    for (int li = 0; li < kLanes; ++li) S->lanes[li].th = std::thread(laneThread, S, li);
    S->watcher = std::thread(watchThread, S);
    return S;
}

void pe_server_destroy(pe_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cvWork.notify_all();
    for (auto& R : S->lanes)
        if (R.th.joinable()) R.th.join();
    if (S->watcher.joinable()) S->watcher.join();
    pe_device* d = S->d;
    cudaSetDevice(d->ordinal);
    cudaStreamSynchronize(d->stream);
    cudaStreamSynchronize(d->lanes[1].stream);
    for (int li = 2; li < kLanes; ++li)
        if (S->lanes[li].stream) cudaStreamSynchronize(S->lanes[li].stream);
    cudaStreamSynchronize(S->copyStream);
    cudaStreamSynchronize(S->admitStream);
    for (auto& kv : S->requests)
        if (kv.second.sum) cudaFreeAsync(kv.second.sum, d->stream);
    cudaStreamSynchronize(d->stream);
    for (ResidentScene& rs : S->scenes) freeList(rs.bufs);
    d->scene = S->savedScene;
    d->hasScene = S->savedHasScene;
    releaseServer(S);
}

int32_t pe_server_add_scene(pe_server* S, const pe_scene* scene) {
    if (!S || !scene) {
        setError("pe_server_add_scene: null argument");
        return -PE_ERR_INVALID;
    }
    if (!scene->built) {
        setError("pe_server_add_scene: scene not built (call pe_scene_build)");
        return -PE_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    cudaSetDevice(S->d->ordinal);
    ResidentScene rs;
    const int32_t rc = uploadScene(S->d, scene, rs.gpu, rs.bufs);
    if (rc) {
        freeList(rs.bufs);
        return -rc;
    }
    for (const DevBuf& b : rs.bufs) rs.bytes += b.bytes;
    if (S->sceneBytes + S->filmBytes + rs.bytes > S->budget) {
        freeList(rs.bufs);
        setError("pe_server_add_scene: scene of " + std::to_string(rs.bytes) + " bytes exceeds the budget");
        return -PE_ERR_LIMIT;
    }
    S->sceneBytes += rs.bytes;
    S->stats.scene_bytes = S->sceneBytes;
    S->scenes.push_back(std::move(rs));
    return static_cast<int32_t>(S->scenes.size() - 1);
}

int64_t pe_server_submit(pe_server* S, const pe_request_desc* q) {
    if (!S || !q) {
        setError("pe_server_submit: null argument");
        return -PE_ERR_INVALID;
    }
    int32_t rc = checkSettings(&q->camera, &q->settings);
    if (rc == PE_OK && q->settings.shadow_quality > 1) {
        setError("pe_server_submit: shadow_quality > 1 (several shadow rays a vertex): render the request with "
                 "pe_device_render");
        rc = PE_ERR_LIMIT;
    }
    if (rc) return -rc;
    if (q->spp <= 0) {
        setError("pe_server_submit: spp must be positive");
        return -PE_ERR_INVALID;
    }
    Request r;
    r.cam = q->camera;
    r.st = q->settings;
    r.spp = q->spp;
    r.priority = q->priority;
    r.filmBytes = filmBytesOf(q->settings);
    std::lock_guard<std::mutex> lk(S->mu);
    if (q->scene < 0 || q->scene >= static_cast<int32_t>(S->scenes.size())) {
        setError("pe_server_submit: unknown scene id");
        return -PE_ERR_INVALID;
    }
    if (S->sceneBytes + r.filmBytes > S->budget) {
        setError("pe_server_submit: film of " + std::to_string(r.filmBytes) + " bytes cannot fit the budget");
        return -PE_ERR_LIMIT;
    }
    r.scene = q->scene;
    r.id = S->nextId++;
    r.submitMs = S->now();
    S->requests[r.id] = r;
    S->queued.push_back(r.id);
    ++S->stats.submitted;
    S->cvWork.notify_all();
    return r.id;
}

int32_t pe_server_status(pe_server* S, int64_t id, pe_request_status* out) {
    if (!S || !out) {
        setError("pe_server_status: null argument");
        return PE_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->requests.find(id);
    if (it == S->requests.end()) {
        setError("pe_server_status: unknown request id");
        return PE_ERR_INVALID;
    }
    const Request& r = it->second;
    std::memset(out, 0, sizeof(*out));
    out->state = r.state;
    out->samples_done = r.samplesDone;
    out->submit_ms = r.submitMs;
    out->start_ms = r.startMs;
    out->done_ms = r.doneMs;
    out->paths = r.paths;
    out->error = r.error;
    return PE_OK;
}

int32_t pe_server_wait(pe_server* S, int64_t id, int32_t timeoutMs) {
    if (!S) {
        setError("pe_server_wait: null server");
        return PE_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->requests.find(id);
    if (it == S->requests.end()) {
        setError("pe_server_wait: unknown request id");
        return PE_ERR_INVALID;
    }
    auto finished = [&] {
        const int32_t st = S->requests[id].state;
        return st == PE_REQ_DONE || st == PE_REQ_FAILED || st == PE_REQ_RELEASED;
    };
    if (timeoutMs < 0) {
        S->cvDone.wait(lk, finished);
    } else if (!S->cvDone.wait_for(lk, std::chrono::milliseconds(timeoutMs), finished)) {
        setError("pe_server_wait: timed out");
        return PE_ERR_CANCELLED;
    }
    const Request& r = S->requests[id];
    if (r.state == PE_REQ_FAILED) {
        setError("pe_server_wait: request failed: " + r.message);
        return r.error;
    }
    return PE_OK;
}

int32_t pe_server_take(pe_server* S, int64_t id, float* sum, uint32_t* cnt, float* sq) {
    if (!S) {
        setError("pe_server_take: null server");
        return PE_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->requests.find(id);
    if (it == S->requests.end() || it->second.state != PE_REQ_DONE) {
        setError("pe_server_take: request is not done (or already taken)");
        return PE_ERR_INVALID;
    }
    Request& r = it->second;
    float* dSum = r.sum;
    uint32_t* dCnt = r.cnt;
    float* dSq = r.sq;
    const size_t n = static_cast<size_t>(r.pixels());
    const size_t bytes = r.filmBytes;
    r.state = PE_REQ_RELEASED;
    r.sum = nullptr;
    r.cnt = nullptr;
    r.sq = nullptr;
    lk.unlock();
    cudaSetDevice(S->d->ordinal);
    // the film's last wave ran on the device stream before the request was marked done
    cudaError_t e = cudaSuccess;
    if (sum && e == cudaSuccess) e = cudaMemcpyAsync(sum, dSum, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, S->copyStream);
    if (cnt && e == cudaSuccess) e = cudaMemcpyAsync(cnt, dCnt, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, S->copyStream);
    if (sq && e == cudaSuccess) e = cudaMemcpyAsync(sq, dSq, n * sizeof(float), cudaMemcpyDeviceToHost, S->copyStream);
    const cudaError_t f = cudaFreeAsync(dSum, S->copyStream);
    const cudaError_t g = cudaStreamSynchronize(S->copyStream);
    lk.lock();
    S->filmBytes -= bytes;
    S->cvWork.notify_all();
    if (e != cudaSuccess || f != cudaSuccess || g != cudaSuccess) {
        setError(std::string("pe_server_take: ") + cudaMsg(e != cudaSuccess ? e : (f != cudaSuccess ? f : g)));
        return PE_ERR_CUDA;
    }
    return PE_OK;
}

int32_t pe_server_get_stats(pe_server* S, pe_server_stats* out) {
    if (!S || !out) {
        setError("pe_server_get_stats: null argument");
        return PE_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->queued = S->queued.size();
    out->active = S->active.size();
    out->film_bytes = S->filmBytes;
    out->film_bytes_peak = S->filmPeak;
    out->budget_bytes = S->budget;
    out->scene_bytes = S->sceneBytes;
    return PE_OK;
}

} // extern "C"
