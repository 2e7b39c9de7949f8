// server.cu -- slot-serving loop: continuous batching of per-cell slot
// requests into fused equalization launches.
//
// Cells are registered once; their channel estimates (H) and noise level stay
// resident in device memory owned by the server and are refreshed in place by
// SRS filter-multiply updates.  Slot requests reference the slot's received
// samples and LLR output in device memory (fronthaul data lands in GPU memory)
// and are admitted against a device-memory budget that covers the resident
// channels plus the buffers of every admitted request; a request that does not
// fit waits, in arrival order, until completions free memory.  A dispatcher
// thread takes whatever is admitted and pending as soon as one of the server's
// streams is free and launches it as ONE fused kernel, so batches overlap on
// the device; completion is observed by polling CUDA events.  Per-subcarrier
// results do not depend on batch composition (the fused kernel's guarantee),
// so a slot's LLRs are the same alone and in any mix.
//
// The reference has no serving layer: its multi-cell study
// (src/multicell_contention.cu:167-235) launches one kernel per cell on its
// own stream and measures the contention; this loop replaces that pattern.
#include "common.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace aeq {

static int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct SrvCell {
    aerial_cell_desc shape{};   // H points at the resident channel; Y_rx/llr unused
    aerial_cf32* H = nullptr;
    size_t hBytes = 0;
    int inflight = 0;           // requests of this cell inside launched batches
    bool srsBusy = false;       // an SRS update of the resident channel is running
    int64_t reqBytes = 0;       // Y_rx + LLR bytes of one slot
    long res = 0;               // REs per slot (subcarriers x symbols)
};

struct SrvReq {
    uint64_t id = 0;
    int kind = 0;               // 0 slot, 1 SRS update
    int cell = 0;
    const aerial_cf32* Y = nullptr;
    float* llr = nullptr;
    // SRS update operands
    const aerial_ch2 *srs = nullptr, *W = nullptr, *focc = nullptr;
    int K = 0, P = 0, F = 0, nSrs = 1;
    int64_t arrival = 0, submitted = 0, launched = 0, done = 0;
    int status = AERIAL_OK;
    bool admitted = false, finished = false;
};

struct SrvBatch {
    cudaEvent_t ev = nullptr;
    std::vector<SrvReq*> reqs;
    bool busy = false;
};

}  // namespace aeq

using namespace aeq;

struct aerial_server {
    aerial_server_config cfg{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv;        // wakes the dispatcher
    std::condition_variable doneCv;    // wakes waiters
    std::vector<SrvCell> cells;
    std::deque<SrvReq*> pending;
    std::unordered_map<uint64_t, SrvReq*> byId;
    std::deque<SrvReq*> completed;     // not yet returned by poll
    std::vector<cudaStream_t> streams;
    std::vector<SrvBatch> batches;     // one per stream
    std::vector<void*> plainWs;        // per-stream workspace of the plain-chain mode
    std::vector<char> blocked;         // per-cell scratch of form_batch
    size_t plainWsBytes = 0;
    int64_t used = 0;                  // budget in use (resident H + admitted requests)
    uint64_t nextId = 1;
    bool stop = false, paused = false;
    std::thread th;
    // statistics
    std::vector<int64_t> lat;          // completion - arrival (ns) of finished slots
    std::vector<int64_t> qlat, slat;   // arrival -> launch, launch -> completion
    std::vector<int64_t> sublag;       // arrival stamp -> submit call (client side)
    int64_t gapMax = 0;                // longest dispatcher iteration while work was pending or in flight
    int64_t launchCallMax = 0;         // longest host call that enqueued a batch
    long missesLateSubmit = 0;         // misses whose submission alone came half a deadline late
    int64_t firstArrival = 0, lastDone = 0;
    long resDone = 0, batchesLaunched = 0, slotsLaunched = 0, srsDone = 0, misses = 0;
    int launchError = 0;
    int inflightBatches = 0;           // batches launched and not finished (under mu)
    int failAllocIn = 0;               // fault injection: the n-th next device allocation fails (0 = off)
};

// A device allocation of the server, as a status (rt_status clears a failed
// cudaMalloc's error from the thread's last-error state).  With fault
// injection armed the n-th allocation fails with cudaErrorMemoryAllocation
// without calling the runtime (host side only).  Lock held.
static int srv_malloc(aerial_server* s, void** p, size_t bytes) {
    *p = nullptr;
    if (s->failAllocIn > 0 && --s->failAllocIn == 0) return (int)cudaErrorMemoryAllocation;
    const int status = rt_status(cudaMalloc(p, bytes));
    if (status) *p = nullptr;
    return status;
}

static void finish_batch(aerial_server* s, SrvBatch& b, int status) {
    const int64_t t = now_ns();
    for (SrvReq* r : b.reqs) {
        r->done = t;
        r->finished = true;
        if (status) r->status = status;
        SrvCell& c = s->cells[r->cell];
        c.inflight--;
        if (r->kind == 0) {
            s->used -= c.reqBytes;
            const int64_t l = r->done - r->arrival;
            const int64_t deadline = (int64_t)(s->cfg.deadline_us * 1000.0);
            s->lat.push_back(l);
            s->qlat.push_back(r->launched - r->arrival);
            s->slat.push_back(r->done - r->launched);
            s->sublag.push_back(r->submitted - r->arrival);
            if (l > deadline) {
                s->misses++;
                if (2 * (r->submitted - r->arrival) > deadline) s->missesLateSubmit++;
            }
            s->resDone += c.res;
            s->lastDone = std::max(s->lastDone, t);
        } else {
            s->srsDone++;
            c.srsBusy = false;
        }
        s->completed.push_back(r);
    }
    b.reqs.clear();
    b.busy = false;
}

// A batch formed under the lock and launched outside it.
struct Formed {
    int n = 0;                          // slot requests (0: none)
    aerial_cell_desc descs[AERIAL_MAX_CELLS];
    bool srs = false;                   // an SRS update instead
    aerial_cf32* H = nullptr;
    const aerial_ch2 *S = nullptr, *W = nullptr, *F = nullptr;
    int nAnt = 0, nBlocks = 0, K = 0, P = 0, foccLen = 0, nSrs = 1;
    void* ws = nullptr;                 // the plain chain's workspace of this stream
    size_t wsBytes = 0;
};

// Form one batch for stream i from the pending queue; lock held.
//
// Order is kept per cell, not globally: a cell's slots never overtake its
// queued SRS update (which waits until none of that cell's slots is in
// flight, then runs alone), but other cells' slots pass it.  Admission is in
// arrival order: the first slot that does not fit the budget stops the scan.
static void form_batch(aerial_server* s, int i, Formed& f) {
    SrvBatch& b = s->batches[i];
    const int cap = std::min(std::max(1, s->cfg.max_batch), (int)AERIAL_MAX_CELLS);
    std::vector<char>& blocked = s->blocked;
    blocked.assign(s->cells.size(), 0);
    int scanned = 0;
    for (size_t k = 0; k < s->pending.size() && f.n < cap && scanned < 1024; scanned++) {
        SrvReq* r = s->pending[k];
        SrvCell& c = s->cells[r->cell];
        if (r->kind == 1) {
            if (!blocked[r->cell] && !c.inflight && !c.srsBusy && f.n == 0) {
                s->pending.erase(s->pending.begin() + k);
                r->launched = now_ns();
                c.inflight++;
                c.srsBusy = true;
                b.reqs.push_back(r);
                f.srs = true;
                f.H = c.H;
                f.S = r->srs;
                f.W = r->W;
                f.F = r->focc;
                f.nAnt = c.shape.nAnt;
                f.nBlocks = c.shape.nPRB * 12 / r->K;
                f.K = r->K;
                f.P = r->P;
                f.foccLen = r->F;
                f.nSrs = r->nSrs;
                return;
            }
            blocked[r->cell] = 1;       // the cell's later slots wait behind its update
            k++;
            continue;
        }
        if (blocked[r->cell] || c.srsBusy) {
            blocked[r->cell] = 1;
            k++;
            continue;
        }
        if (!r->admitted) {
            if (s->used + c.reqBytes > s->cfg.memory_budget_bytes) break;   // waits, in arrival order
            s->used += c.reqBytes;
            r->admitted = true;
        }
        s->pending.erase(s->pending.begin() + k);
        aerial_cell_desc d = c.shape;
        d.Y_rx = r->Y;
        d.llr = r->llr;
        d.Y_eq = nullptr;
        f.descs[f.n++] = d;
        c.inflight++;
        r->launched = now_ns();
        b.reqs.push_back(r);
    }
}

// Batching window: launch fewer than min_batch pending slots only once the
// oldest has waited batch_window_us; lock held.
static bool batch_ready(aerial_server* s) {
    if (s->cfg.min_batch <= 1 || s->cfg.batch_window_us <= 0.f) return true;
    if ((int)s->pending.size() >= s->cfg.min_batch) return true;
    return now_ns() - s->pending.front()->arrival >= (int64_t)(s->cfg.batch_window_us * 1000.0);
}

// Launch a formed batch on stream i; no lock held.  Returns the status.
static int launch_formed(aerial_server* s, int i, const Formed& f) {
    cudaStream_t st = s->streams[i];
    int status = AERIAL_OK;
    if (f.srs) {
        status = aerial_srs_to_channel_avg(f.H, f.S, f.nSrs, f.W, f.F, f.nAnt, f.nBlocks, f.K, f.P, f.foccLen, st);
    } else if (s->cfg.mode == AERIAL_SERVER_PLAIN) {
        // the plain FP32 chain, request by request (comparison mode)
        for (int k = 0; k < f.n && !status; k++)
            status = aerial_pusch_eq_plain(&f.descs[k], 1, f.ws, f.wsBytes, st);
    } else {
        aerial_tuning t{s->cfg.precision, 0, 0, 0};
        status = aerial_pusch_eq_fused(f.descs, f.n, &t, st);
    }
    if (!status) {
        cudaError_t e = cudaEventRecord(s->batches[i].ev, st);
        if (e != cudaSuccess) status = rt_status(e);
    }
    return status;
}

// The dispatcher: CUDA calls (launches, event queries) happen outside the
// lock, so submissions are never held up by a launch in progress.
static void dispatcher(aerial_server* s) {
    cudaSetDevice(s->device);
    Formed f;
    std::unique_lock<std::mutex> lk(s->mu, std::defer_lock);
    int64_t lastIter = 0;                 // start of the previous iteration that had work (0: idle)
    while (true) {
        const int64_t iterStart = now_ns();
        bool progress = false;
        // completions (the busy flags and events are the dispatcher's own)
        for (SrvBatch& b : s->batches) {
            if (!b.busy) continue;
            const cudaError_t e = cudaEventQuery(b.ev);
            if (e == cudaErrorNotReady) continue;
            lk.lock();
            finish_batch(s, b, rt_status(e));
            s->inflightBatches--;
            lk.unlock();
            s->doneCv.notify_all();
            progress = true;
        }
        // launches
        for (size_t i = 0; i < s->batches.size(); i++) {
            SrvBatch& b = s->batches[i];
            if (b.busy) continue;
            lk.lock();
            if (s->stop) {
                lk.unlock();
                return;
            }
            f.n = 0;
            f.srs = false;
            if (!s->paused && !s->pending.empty() && batch_ready(s)) form_batch(s, (int)i, f);
            if (s->cfg.mode == AERIAL_SERVER_PLAIN) {
                f.ws = s->plainWs.empty() ? nullptr : s->plainWs[i];
                f.wsBytes = s->plainWsBytes;
            }
            const bool formed = f.n > 0 || f.srs;
            if (formed) {
                b.busy = true;
                s->inflightBatches++;
                if (!f.srs) {
                    s->batchesLaunched++;
                    s->slotsLaunched += f.n;
                }
            }
            lk.unlock();
            if (!formed) continue;
            progress = true;
            const int64_t c0 = now_ns();
            const int status = launch_formed(s, (int)i, f);
            const int64_t callNs = now_ns() - c0;
            if (status || callNs > s->launchCallMax) {
                lk.lock();
                s->launchCallMax = std::max(s->launchCallMax, callNs);
                if (status) {
                    s->launchError = status;
                    finish_batch(s, b, status);
                    s->inflightBatches--;
                }
                lk.unlock();
                if (status) s->doneCv.notify_all();
            }
        }
        bool anyBusy = false;
        for (SrvBatch& b : s->batches) anyBusy |= b.busy;
        lk.lock();
        if (s->stop) {
            lk.unlock();
            return;
        }
        const bool waiting = !s->pending.empty() && !s->paused;   // e.g. inside a batching window
        // the host's view of the loop: the longest step between two
        // iterations that had work (a descheduled dispatcher shows here)
        if (lastIter && (anyBusy || waiting)) s->gapMax = std::max(s->gapMax, iterStart - lastIter);
        lastIter = (anyBusy || waiting || progress) ? iterStart : 0;
        if (!anyBusy && !progress && !waiting) {
            // idle: sleep until a submission (or stop) notifies; the timeout
            // only bounds a missed wake-up
            s->cv.wait_for(lk, std::chrono::milliseconds(2));
            lk.unlock();
            continue;
        }
        lk.unlock();
        // work in flight or pending: poll again at once (a yield keeps the
        // core available to the submitting threads on a busy host)
        std::this_thread::yield();
    }
}

// Room for kStatsReserve latency samples and for as many unpolled requests
// before any container under the lock has to grow (8 bytes a sample per
// statistic, a few MB in all); beyond that they still grow.
constexpr size_t kStatsReserve = 1 << 18;
static void reserve_tables(aerial_server* s) {
    s->byId.reserve(kStatsReserve);
    for (std::vector<int64_t>* v : {&s->lat, &s->qlat, &s->slat, &s->sublag}) v->reserve(kStatsReserve);
}

extern "C" int aerial_server_create(const aerial_server_config* cfg, aerial_server** out) {
    if (!cfg || !out || cfg->memory_budget_bytes <= 0 || cfg->streams < 1 || cfg->streams > 16 ||
        cfg->max_batch < 1 || cfg->deadline_us <= 0.f)
        return AERIAL_ERR_INVALID_ARG;
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return AERIAL_ERR_NO_DEVICE;
    const int prep = aerial_prepare();
    if (prep != AERIAL_OK) return prep;
    aerial_server* s = new aerial_server();
    s->cfg = *cfg;
    s->device = dev;
    s->paused = cfg->start_paused != 0;
    s->streams.resize(cfg->streams);
    s->batches.resize(cfg->streams);
    for (int i = 0; i < cfg->streams; i++) {
        e = cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->batches[i].ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            for (int k = 0; k <= i; k++) {
                if (s->streams[k]) cudaStreamDestroy(s->streams[k]);
                if (s->batches[k].ev) cudaEventDestroy(s->batches[k].ev);
            }
            delete s;
            return rt_status(e);
        }
    }
    // Containers that grow with the requests in flight or not yet polled are
    // sized up front: growing one (a hash-table rehash, a vector copy) under
    // the server's lock stalled submissions and the dispatcher together for
    // about a millisecond at a time.
    reserve_tables(s);
    s->th = std::thread(dispatcher, s);
    *out = s;
    return AERIAL_OK;
}

extern "C" int aerial_server_destroy(aerial_server* s) {
    if (!s) return AERIAL_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    s->th.join();
    for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
    for (size_t i = 0; i < s->streams.size(); i++) {
        cudaEventDestroy(s->batches[i].ev);
        cudaStreamDestroy(s->streams[i]);
    }
    for (SrvCell& c : s->cells) cudaFree(c.H);
    for (void* w : s->plainWs) cudaFree(w);
    for (auto& kv : s->byId) delete kv.second;
    delete s;
    return AERIAL_OK;
}

extern "C" int aerial_server_add_cell(aerial_server* s, int nPRB, int nAnt, int nLayers, int nSym, int nPamBits,
                                      float sigma2, int* cellId) {
    if (!s || !cellId || nPRB < 1 || nPRB > AERIAL_MAX_PRB || nAnt < 1 || nAnt > AERIAL_MAX_ANTS || nLayers < 1 ||
        nLayers > AERIAL_MAX_LAYERS || nSym < 1 || nSym > AERIAL_MAX_SYMS || nPamBits < 1 || nPamBits > 4 ||
        !(sigma2 >= 0.f))
        return AERIAL_ERR_INVALID_ARG;
    SrvCell c;
    const long nSC = 12L * nPRB;
    c.hBytes = sizeof(aerial_cf32) * nSC * nAnt * nLayers;
    c.reqBytes = (int64_t)(sizeof(aerial_cf32) * nSC * nSym * nAnt + sizeof(float) * nSC * nLayers * nSym * 2 * nPamBits);
    c.res = nSC * nSym;
    c.shape.sigma2 = sigma2;
    c.shape.nPRB = nPRB;
    c.shape.nAnt = nAnt;
    c.shape.nLayers = nLayers;
    c.shape.nSym = nSym;
    c.shape.nPamBits = nPamBits;
    std::unique_lock<std::mutex> lk(s->mu);
    // plain mode: the per-stream workspaces grow to the largest cell
    size_t need = 0;
    int64_t extra = 0;
    if (s->cfg.mode == AERIAL_SERVER_PLAIN) {
        need = aerial_pusch_eq_plain_workspace(&c.shape, 1);
        if (need > s->plainWsBytes) extra = (int64_t)(need - s->plainWsBytes) * (int64_t)s->streams.size();
        else need = 0;
    }
    if (s->used + (int64_t)c.hBytes + extra + c.reqBytes > s->cfg.memory_budget_bytes) return AERIAL_ERR_BUDGET;
    // Everything is allocated before anything is committed: a failed
    // allocation leaves the server as it was.
    void* h = nullptr;
    int status = srv_malloc(s, &h, c.hBytes);
    if (status) return status;
    std::vector<void*> fresh(need ? s->streams.size() : 0, nullptr);
    for (void*& w : fresh)
        if (!status) status = srv_malloc(s, &w, need);
    if (!status && need) {
        // the old workspaces may be in use: wait (bounded) until no batch is in
        // flight; none can form while the lock is held afterwards
        const auto limit = std::chrono::steady_clock::now() + std::chrono::seconds(10);
        while (s->inflightBatches > 0 && !status)
            if (s->doneCv.wait_until(lk, limit) == std::cv_status::timeout && s->inflightBatches > 0)
                status = AERIAL_ERR_TIMEOUT;
    }
    if (status) {
        for (void* w : fresh) cudaFree(w);
        cudaFree(h);
        return status;
    }
    c.H = static_cast<aerial_cf32*>(h);
    cudaMemset(c.H, 0, c.hBytes);
    c.shape.H = c.H;
    s->used += (int64_t)c.hBytes;
    if (need) {
        for (void* w : s->plainWs) cudaFree(w);
        s->plainWs = std::move(fresh);
        s->plainWsBytes = need;
        s->used += extra;
    }
    s->cells.push_back(c);
    *cellId = (int)s->cells.size() - 1;
    return AERIAL_OK;
}

extern "C" int aerial_server_inject_alloc_failure(aerial_server* s, int nth) {
    if (!s || nth < 0) return AERIAL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->failAllocIn = nth;
    return AERIAL_OK;
}

extern "C" int aerial_server_set_channel(aerial_server* s, int cellId, const aerial_cf32* H, float sigma2) {
    if (!s || !H || !(sigma2 >= 0.f)) return AERIAL_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (cellId < 0 || cellId >= (int)s->cells.size()) return AERIAL_ERR_NOT_FOUND;
    SrvCell& c = s->cells[cellId];
    // wait (bounded) until no launched batch reads the resident channel
    const auto limit = std::chrono::steady_clock::now() + std::chrono::seconds(5);
    while (c.inflight) {
        if (s->doneCv.wait_until(lk, limit) == std::cv_status::timeout && c.inflight) return AERIAL_ERR_TIMEOUT;
    }
    cudaError_t e = cudaMemcpy(c.H, H, c.hBytes, cudaMemcpyDefault);
    c.shape.sigma2 = sigma2;
    return rt_status(e);
}

extern "C" int aerial_server_submit(aerial_server* s, int cellId, const aerial_cf32* Y_rx, float* llr,
                                    int64_t arrival_ns, uint64_t* requestId) {
    if (!s || !Y_rx || !llr) return AERIAL_ERR_INVALID_ARG;
    SrvReq* r = new SrvReq();
    r->Y = Y_rx;
    r->llr = llr;
    r->submitted = now_ns();
    r->arrival = arrival_ns > 0 ? arrival_ns : r->submitted;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (cellId < 0 || cellId >= (int)s->cells.size()) { delete r; return AERIAL_ERR_NOT_FOUND; }
        if (s->cells[cellId].reqBytes + (int64_t)s->cells[cellId].hBytes > s->cfg.memory_budget_bytes) {
            delete r;
            return AERIAL_ERR_BUDGET;
        }
        if ((int)s->pending.size() >= (s->cfg.queue_capacity > 0 ? s->cfg.queue_capacity : 1 << 20)) {
            delete r;
            return AERIAL_ERR_QUEUE_FULL;
        }
        r->cell = cellId;
        r->id = s->nextId++;
        if (!s->firstArrival || r->arrival < s->firstArrival) s->firstArrival = r->arrival;
        s->byId[r->id] = r;
        s->pending.push_back(r);
        if (requestId) *requestId = r->id;
    }
    s->cv.notify_one();
    return AERIAL_OK;
}

extern "C" int aerial_server_srs_update(aerial_server* s, int cellId, const aerial_ch2* SRS, const aerial_ch2* W,
                                        const aerial_ch2* FOCC, int K, int foccLen, uint64_t* requestId) {
    return aerial_server_srs_update_n(s, cellId, SRS, 1, W, FOCC, K, foccLen, requestId);
}

extern "C" int aerial_server_srs_update_n(aerial_server* s, int cellId, const aerial_ch2* SRS, int nSrsSym,
                                          const aerial_ch2* W, const aerial_ch2* FOCC, int K, int foccLen,
                                          uint64_t* requestId) {
    if (!s || !SRS || !W || !FOCC || K < 1 || foccLen < 1 || (nSrsSym != 1 && nSrsSym != 2 && nSrsSym != 4))
        return AERIAL_ERR_INVALID_ARG;
    SrvReq* r = new SrvReq();
    r->kind = 1;
    r->nSrs = nSrsSym;
    r->srs = SRS;
    r->W = W;
    r->focc = FOCC;
    r->K = K;
    r->F = foccLen;
    r->arrival = r->submitted = now_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (cellId < 0 || cellId >= (int)s->cells.size()) { delete r; return AERIAL_ERR_NOT_FOUND; }
        const SrvCell& c = s->cells[cellId];
        if ((c.shape.nPRB * 12) % K) { delete r; return AERIAL_ERR_INVALID_ARG; }
        r->P = c.shape.nLayers;           // one SRS port per layer
        r->cell = cellId;
        r->id = s->nextId++;
        s->byId[r->id] = r;
        s->pending.push_back(r);
        if (requestId) *requestId = r->id;
    }
    s->cv.notify_one();
    return AERIAL_OK;
}

extern "C" int aerial_server_poll(aerial_server* s, aerial_server_completion* out, int maxOut, int* nOut) {
    if (!s || !nOut || (maxOut > 0 && !out)) return AERIAL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    int n = 0;
    while (n < maxOut && !s->completed.empty()) {
        SrvReq* r = s->completed.front();
        s->completed.pop_front();
        out[n].request_id = r->id;
        out[n].cell_id = r->cell;
        out[n].status = r->status;
        out[n].latency_us = (float)((r->done - r->arrival) * 1e-3);
        n++;
        s->byId.erase(r->id);
        delete r;
    }
    *nOut = n;
    return AERIAL_OK;
}

extern "C" int aerial_server_wait(aerial_server* s, uint64_t requestId, int timeout_ms) {
    if (!s) return AERIAL_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->byId.find(requestId);
    if (it == s->byId.end()) return AERIAL_ERR_NOT_FOUND;
    SrvReq* r = it->second;
    const auto limit = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    while (!r->finished) {
        if (s->doneCv.wait_until(lk, limit) == std::cv_status::timeout && !r->finished) return AERIAL_ERR_TIMEOUT;
    }
    return r->status;
}

extern "C" int aerial_server_drain(aerial_server* s, int timeout_ms) {
    if (!s) return AERIAL_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const auto limit = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    auto busy = [&] { return !s->pending.empty() || s->inflightBatches > 0; };
    while (busy()) {
        if (s->doneCv.wait_until(lk, limit) == std::cv_status::timeout && busy()) return AERIAL_ERR_TIMEOUT;
    }
    return s->launchError;
}

extern "C" int aerial_server_pause(aerial_server* s, int paused) {
    if (!s) return AERIAL_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->paused = paused != 0;
    }
    s->cv.notify_one();
    return AERIAL_OK;
}

extern "C" int aerial_server_stats(aerial_server* s, aerial_server_statistics* out) {
    if (!s || !out) return AERIAL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    aerial_server_statistics st{};
    std::vector<int64_t> l = s->lat;
    st.slots_done = (long)l.size();
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            size_t i = (size_t)std::ceil(p / 100.0 * l.size());
            if (i < 1) i = 1;
            return l[std::min(l.size(), i) - 1] * 1e-3;
        };
        st.p50_us = (float)pct(50);
        st.p99_us = (float)pct(99);
        st.max_us = (float)(l.back() * 1e-3);
        double sum = 0;
        for (int64_t v : l) sum += v;
        st.mean_us = (float)(sum / l.size() * 1e-3);
        auto p99 = [](std::vector<int64_t> v) {
            std::sort(v.begin(), v.end());
            size_t i = (size_t)std::ceil(0.99 * v.size());
            if (i < 1) i = 1;
            return (float)(v[std::min(v.size(), i) - 1] * 1e-3);
        };
        st.queue_p99_us = p99(s->qlat);
        st.service_p99_us = p99(s->slat);
        st.submit_lag_p99_us = p99(s->sublag);
        st.submit_lag_max_us = (float)(*std::max_element(s->sublag.begin(), s->sublag.end()) * 1e-3);
    }
    st.dispatch_gap_max_us = (float)(s->gapMax * 1e-3);
    st.launch_call_max_us = (float)(s->launchCallMax * 1e-3);
    st.misses_late_submit = s->missesLateSubmit;
    st.deadline_misses = s->misses;
    st.res_done = s->resDone;
    st.span_s = (s->lastDone > s->firstArrival) ? (double)(s->lastDone - s->firstArrival) * 1e-9 : 0.0;
    st.res_per_s = st.span_s > 0 ? st.res_done / st.span_s : 0.0;
    st.batches = s->batchesLaunched;
    st.mean_batch = s->batchesLaunched ? (float)s->slotsLaunched / s->batchesLaunched : 0.f;
    st.srs_updates = s->srsDone;
    st.budget_used_bytes = s->used;
    st.pending = (long)s->pending.size();
    *out = st;
    return AERIAL_OK;
}

extern "C" int aerial_server_reset_stats(aerial_server* s) {
    if (!s) return AERIAL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat.clear();
    s->qlat.clear();
    s->slat.clear();
    s->sublag.clear();
    s->gapMax = s->launchCallMax = 0;
    s->firstArrival = s->lastDone = 0;
    s->resDone = s->batchesLaunched = s->slotsLaunched = s->srsDone = s->misses = s->missesLateSubmit = 0;
    return AERIAL_OK;
}
