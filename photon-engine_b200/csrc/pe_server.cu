// pe_server.cu — the request server behind the pe_server_* C ABI: resident scenes, device films
// admitted against an HBM budget, and a worker thread that packs the pending sample ranges of
// many requests into shared waves (continuous batching).
//
// Waves alternate the device's two lanes: wave k+1 is planned and its bounces traced while wave
// k's tail still runs; a request is done once the lane of its last wave has finished.
//
// Scheduling.  Admitted requests are ordered by (priority desc, remaining paths asc, id asc).
// The first request picks the wave's scene; the wave is then filled, in that order, with one
// chunk per admitted request of the same scene until its 2M path slots are used.  A chunk is
// either whole-frame sample rows [s, s+k) or, when a frame does not fit, a pixel range of one
// sample row.  A request's rows run in increasing sample order, so every pixel adds its samples
// in the order a lone render does and the film is bit-identical to pe_device_render's.
#include "pe_device_impl.h"

#include <chrono>
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
    double submitMs = 0.0, startMs = 0.0, doneMs = 0.0;

    int64_t pixels() const { return static_cast<int64_t>(st.width) * st.height; }
    int64_t remaining() const { return (static_cast<int64_t>(spp) - sampleCursor) * pixels() - pixelCursor; }
};

struct ResidentScene {
    SceneGPU gpu{};
    std::vector<DevBuf> bufs;
    size_t bytes = 0;
};

// A wave's chunk of one request, kept for the progress update after the wave.
struct Chunk {
    int64_t id;
    int32_t samples;    // whole rows handed out (0 for a partial row)
    bool closesRow;     // a split row's last pixel range
};

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
    Clock::time_point t0;
    SceneGPU savedScene{};
    bool savedHasScene = false;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evAdmit = nullptr;   // after the film allocations of the last admission
    pe_server_stats stats{};
    // the wave in flight on each lane, booked once the lane's done-event fires
    struct InFlight {
        bool valid = false;
        std::vector<Chunk> chunks;
        int32_t rc = PE_OK;
        std::string message;
        cudaEvent_t evStart = nullptr;
    } inflight[2];
    int lane = 0;

    double now() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

// Gives films to queued requests, in priority order, while the budget has room.  Called with
// the lock held, on the worker thread.
void admit(pe_server* S) {
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
        cudaError_t e = cudaMallocAsync(&p, r.filmBytes, S->d->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, r.filmBytes, S->d->stream);
        if (e != cudaSuccess) {
            r.state = PE_REQ_FAILED;
            r.error = e == cudaErrorMemoryAllocation ? PE_ERR_OOM : PE_ERR_CUDA;
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
    }
}

// Packs the next wave into the lane's segment table; returns its segment count (0 = nothing to do).
int planWave(pe_server* S, int lane, int& sceneOut, int& nSlots, int& nPix, std::vector<Chunk>& chunks) {
    pe_device* d = S->d;
    std::vector<int64_t> order = S->active;
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        const Request& ra = S->requests[a];
        const Request& rb = S->requests[b];
        if (ra.priority != rb.priority) return ra.priority > rb.priority;
        if (ra.remaining() != rb.remaining()) return ra.remaining() < rb.remaining();
        return a < b;
    });
    chunks.clear();
    nSlots = 0;
    nPix = 0;
    int nSegs = 0;
    int scene = -1;
    const int64_t cap = static_cast<int64_t>(d->capacity);
    const uint64_t clock = ++d->filterClock;
    for (int64_t id : order) {
        Request& r = S->requests[id];
        if (r.sampleCursor >= r.spp) continue; // all rows handed out; waiting for its last wave
        if (scene < 0) scene = r.scene;
        if (r.scene != scene) continue;
        const int64_t room = cap - nSlots;
        if (room <= 0 || nSegs >= kMaxSegs) break;
        if (nSegs > 0 && room < 4096) break; // not worth a segment
        const float* filter = filterTable(d, r.st.filter_type, r.st.filter_width, clock, d->lanes[lane].stream);
        if (!filter) break; // every filter slot is taken by this wave
        WaveSeg seg = makeSeg(&r.cam, &r.st);
        seg.filterCdf = filter;
        seg.tileX = 0;
        seg.tileY = 0;
        seg.tileW = r.st.width;
        seg.sum = r.sum;
        seg.cnt = r.cnt;
        seg.sq = r.sq;
        seg.slotFirst = nSlots;
        seg.pixFirst = nPix;
        const int64_t npix = r.pixels();
        Chunk c{id, 0, false};
        if (r.pixelCursor == 0 && npix <= room) {
            const int64_t rows = std::min<int64_t>(r.spp - r.sampleCursor, room / npix);
            seg.pixelFirst = 0;
            seg.nPix = static_cast<int>(npix);
            seg.sampleFirst = r.sampleCursor;
            seg.nSamples = static_cast<int>(rows);
            r.sampleCursor += static_cast<int32_t>(rows);
            c.samples = static_cast<int32_t>(rows);
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
                c.closesRow = true;
            }
        }
        d->lanes[lane].hSegs[nSegs++] = seg;
        nSlots += seg.nPix * seg.nSamples;
        nPix += seg.nPix;
        r.paths += static_cast<uint64_t>(seg.nPix) * static_cast<uint64_t>(seg.nSamples);
        chunks.push_back(c);
    }
    sceneOut = scene;
    return nSegs;
}

// Books a lane's finished wave (lock held): progress of its requests, completions, device time.
// Returns false while the wave is still running.
bool settleLane(pe_server* S, int l) {
    auto& f = S->inflight[l];
    if (!f.valid) return true;
    WaveLane& ln = S->d->lanes[l];
    if (f.rc == PE_OK) {
        const cudaError_t e = cudaEventQuery(ln.evDone);
        if (e == cudaErrorNotReady) return false;
        if (e != cudaSuccess) {
            f.rc = PE_ERR_CUDA;
            f.message = std::string("wave: ") + cudaMsg(e);
        } else {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, f.evStart, ln.evDone) == cudaSuccess) S->stats.busy_ms += ms;
        }
    }
    const double t = S->now();
    for (const Chunk& c : f.chunks) {
        Request& r = S->requests[c.id];
        if (f.rc != PE_OK) {
            if (r.state == PE_REQ_ACTIVE) {
                r.state = PE_REQ_FAILED;
                r.error = f.rc;
                r.message = f.message;
                r.doneMs = t;
                ++S->stats.failed;
            }
            continue;
        }
        r.samplesDone += c.samples + (c.closesRow ? 1 : 0);
        if (r.samplesDone >= r.spp && r.state == PE_REQ_ACTIVE) {
            r.state = PE_REQ_DONE;
            r.doneMs = t;
            ++S->stats.completed;
        }
    }
    S->active.erase(std::remove_if(S->active.begin(), S->active.end(),
                                   [&](int64_t id) { return S->requests[id].state != PE_REQ_ACTIVE; }),
                    S->active.end());
    f.valid = false;
    S->cvDone.notify_all();
    return true;
}

// The worker: alternates the device's two lanes, so the next wave's bounces run while the
// previous wave finishes its tail.  The host waits on a lane only when it needs that lane again.
void workerLoop(pe_server* S) {
    pe_device* d = S->d;
    cudaSetDevice(d->ordinal);
    std::vector<Chunk> chunks;
    for (;;) {
        std::unique_lock<std::mutex> lk(S->mu);
        settleLane(S, 0);
        settleLane(S, 1);
        const bool inflight = S->inflight[0].valid || S->inflight[1].valid;
        if (!inflight)
            S->cvWork.wait(lk, [&] { return S->stop || !S->queued.empty() || !S->active.empty(); });
        if (S->stop) break;
        admit(S);
        cudaEventRecord(S->evAdmit, d->stream);
        const int L = S->lane;
        if (S->inflight[L].valid) {
            // the lane is still busy with the wave before last: wait for it outside the lock
            lk.unlock();
            cudaEventSynchronize(d->lanes[L].evDone);
            continue;
        }
        int scene = -1, nSlots = 0, nPix = 0;
        if (segsWritable(d, L) != PE_OK) break;
        const int nSegs = planWave(S, L, scene, nSlots, nPix, chunks);
        if (nSegs == 0) {
            if (inflight) {
                // nothing new to trace: wait for the other lane's wave to finish
                lk.unlock();
                cudaEventSynchronize(d->lanes[L ^ 1].evDone);
            } else {
                // everything queued waits for budget held by films not yet taken
                S->cvWork.wait_for(lk, std::chrono::milliseconds(2));
            }
            continue;
        }
        auto& f = S->inflight[L];
        f.chunks = chunks;
        f.valid = true;
        ++S->stats.waves;
        S->stats.segments += static_cast<uint64_t>(nSegs);
        S->stats.paths += static_cast<uint64_t>(nSlots);
        lk.unlock();
        d->scene = S->scenes[static_cast<size_t>(scene)].gpu;
        d->hasScene = true;
        const cudaStream_t cs = d->lanes[L].stream;
        RenderTimer tm;
        int32_t rc = PE_OK;
        if (cudaStreamWaitEvent(cs, S->evAdmit, 0) != cudaSuccess || cudaEventRecord(f.evStart, cs) != cudaSuccess)
            rc = PE_ERR_CUDA;
        if (rc == PE_OK) rc = runWave(d, L, d->lanes[L].paths, nSegs, nSlots, nPix, tm);
        const std::string msg = rc == PE_OK ? std::string() : std::string(pe_last_error());
        lk.lock();
        f.rc = rc;
        f.message = msg;
        S->lane = L ^ 1;
    }
    cudaStreamSynchronize(d->lanes[0].stream);
    cudaStreamSynchronize(d->lanes[1].stream);
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
    if (cudaStreamCreateWithFlags(&S->copyStream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->evAdmit, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&S->inflight[0].evStart) != cudaSuccess || cudaEventCreate(&S->inflight[1].evStart) != cudaSuccess) {
        delete S;
        return failCreate(err, errLen, "pe_server_create: stream or event creation failed");
    }
    d->filmLane = -1;
    S->worker = std::thread(workerLoop, S);
    return S;
}

void pe_server_destroy(pe_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cvWork.notify_all();
    if (S->worker.joinable()) S->worker.join();
    pe_device* d = S->d;
    cudaSetDevice(d->ordinal);
    cudaStreamSynchronize(d->stream);
    cudaStreamSynchronize(d->lanes[1].stream);
    cudaStreamSynchronize(S->copyStream);
    for (auto& kv : S->requests)
        if (kv.second.sum) cudaFreeAsync(kv.second.sum, d->stream);
    cudaStreamSynchronize(d->stream);
    for (ResidentScene& rs : S->scenes) freeList(rs.bufs);
    cudaStreamDestroy(S->copyStream);
    cudaEventDestroy(S->evAdmit);
    cudaEventDestroy(S->inflight[0].evStart);
    cudaEventDestroy(S->inflight[1].evStart);
    d->scene = S->savedScene;
    d->hasScene = S->savedHasScene;
    delete S;
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
    const int32_t rc = checkSettings(&q->camera, &q->settings);
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
