// ffbf_serve.cu -- the scan server (ffbf_server_* in include/ffbf.h): resident pattern sets, admission of
// requests by free slots and free device memory, and continuous batching of the admitted requests.
//
// One host thread runs the loop. Per iteration it
//   1. takes new submissions into the FIFO of pending requests;
//   2. admits pending requests in order while a slot and a range of the text arena are free, and starts
//      each one's host-to-device copy on the copy stream (an event marks its end). The arena is a list of
//      device segments: when no segment has room, a new one is allocated only if the device's free memory
//      (cudaMemGetInfo, which sees every context's allocations) stays above a reserve afterwards and the
//      arena stays within its cap; otherwise the request waits, in order, until a finished request frees
//      room or other contexts free memory. Segments beyond the first are given back when the server idles;
//   3. moves requests whose copy has finished to the ready list;
//   4. when the previous launch sequence has finished, launches every ready request as one plan
//      (build_plan/launch_plan: one tuned launch per (LEN, configuration) group, one generic launch for
//      ragged ends) on the scan stream;
//   5. for each request of a finished batch (whose hit counts came back with the batch), enqueues line
//      resolution and the copy of its hits on the slot's own stream, overlapping the next batch's scan;
//      a request whose copy has landed is ordered on the host and its slot and arena range are freed.
//      A request with more hits than its slot's buffer takes the plain collect (regrow and rescan).
// A slot is a context with its own scan buffers whose filters are attached from the request's set.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ffbf_ctx.cuh"

using namespace ffbf_host;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    uint32_t set = 0;
    const uint8_t* h_text = nullptr;
    size_t len = 0;
    int seg = -1;       // arena segment holding the text
    uint64_t off = 0;   // offset in that segment
    uint64_t span = 0;  // arena bytes held
    int slot = -1;
    uint32_t nh = 0;  // hit windows, read back with the batch
    double t_submit = 0, t_admit = 0, t_launch = 0, t_done = 0;
    ffbf_status status = FFBF_OK;
    std::vector<uint64_t> hits, ls, le;
};

constexpr uint64_t kArenaAlign = 256;
constexpr uint64_t kSmallCopy = 4ull << 20;  // texts up to this size copy on the small-copy stream
constexpr uint32_t kMaxCtl = 64;  // control-word groups per plan (one per tuned launch, plus one)
constexpr uint64_t kPreallocText = 512ull << 20;  // request size the slots' scan buffers start out sized for
constexpr uint64_t kSegmentBytes = 1ull << 30;    // arena growth step (a larger request gets a segment its size)
constexpr uint64_t kHbmReserve = 1ull << 30;      // device memory the arena leaves free for others
constexpr double kGrowRetrySeconds = 1e-3;        // pause between growth attempts that found too little memory
constexpr double kShrinkIdleSeconds = 0.25;       // idle time after which grown segments are given back
constexpr uint32_t kPreallocHits = 16384;          // hit records each slot's pinned result copy starts with

}  // namespace

struct ffbf_server {
    int device = 0;
    int num_sms = 0;
    // request copies: texts of kSmallCopy bytes or less on st_copy_small, so that they do not queue behind
    // large texts on st_copy (the two copies share the link while both run)
    cudaStream_t st_scan = nullptr, st_copy = nullptr, st_copy_small = nullptr;
    Clock::time_point t0;
    std::string err;

    std::vector<ffbf_ctx*> sets;
    std::vector<ffbf_ctx*> slots;
    std::vector<cudaEvent_t> copy_done;  // per slot
    std::vector<int> free_slots;

    struct Segment {
        uint8_t* base = nullptr;
        uint64_t bytes = 0;
        std::map<uint64_t, uint64_t> free_ranges;  // offset -> length, coalesced
    };
    std::vector<Segment> segs;    // segs[0] is kept while the server idles (at its first size)
    uint64_t arena_cap = 0;       // most arena bytes the server holds (0: bounded by free device memory only)
    uint64_t arena_held = 0;      // bytes of all segments
    uint64_t device_bytes = 0;    // the device's memory
    double last_grow_fail = -1.0;
    double idle_since = -1.0;     // when the loop last found nothing admitted (segments shrink after a while)

    // plan tables on the device and their pinned staging
    ffbf::FastJob* d_fast = nullptr;
    ffbf::ScanArgs* d_args = nullptr;
    uint32_t** d_counters = nullptr;
    uint32_t* d_ctl = nullptr;
    uint2* d_tail = nullptr;
    size_t tail_cap = 0;
    ffbf::FastJob* h_fast = nullptr;
    ffbf::ScanArgs* h_args = nullptr;
    uint32_t** h_counters = nullptr;
    uint2* h_tail = nullptr;
    uint32_t* h_ctl = nullptr;  // error flags read back after each batch
    uint32_t* d_cnt = nullptr;  // every job's counters, gathered after each batch
    uint32_t* h_cnt = nullptr;
    struct SlotHost {
        HitRec* hr = nullptr;  // pinned copies of the slot's hit records and lines
        HitLine* hl = nullptr;
        uint32_t cap = 0;
        cudaEvent_t done = nullptr;
    };
    std::vector<SlotHost> slot_host;
    cudaEvent_t batch_done = nullptr;
    uint32_t batch_ctl = 0;

    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    bool started = false;
    std::deque<Request*> inbox;                    // guarded by mu
    std::deque<Request*> done;                     // guarded by mu
    std::unordered_map<uint64_t, Request*> owned;  // polled, not yet released (guarded by mu)
    uint64_t next_id = 1;
    ffbf_server_stats stats{};  // guarded by mu
    ffbf_status fatal = FFBF_OK;

    // worker-only state
    std::deque<Request*> pending;
    std::vector<Request*> copying, ready, running, resolving, slow;
    bool in_flight = false;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// The last error is written by the caller's thread and by the worker; both go through the mutex.
void set_err(ffbf_server* s, const std::string& msg) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = msg;
}

ffbf_status sfail(ffbf_server* s, ffbf_status st, const std::string& msg) {
    set_err(s, msg);
    return st;
}

bool seg_alloc(ffbf_server::Segment& g, uint64_t bytes, uint64_t* off) {
    for (auto it = g.free_ranges.begin(); it != g.free_ranges.end(); ++it) {
        if (it->second >= bytes) {
            *off = it->first;
            const uint64_t rest = it->second - bytes;
            const uint64_t at = it->first + bytes;
            g.free_ranges.erase(it);
            if (rest) g.free_ranges[at] = rest;
            return true;
        }
    }
    return false;
}

void seg_free(ffbf_server::Segment& g, uint64_t off, uint64_t bytes) {
    auto it = g.free_ranges.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != g.free_ranges.end() && it->first + it->second == next->first) {
        it->second += next->second;
        g.free_ranges.erase(next);
    }
    if (it != g.free_ranges.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            g.free_ranges.erase(it);
        }
    }
}

// A new segment of at least `bytes`, if the device's free memory stays above the reserve and the arena within
// its cap. cudaMemGetInfo counts every context's allocations, so memory other processes or libraries took
// since the last look is respected.
bool arena_grow(ffbf_server* s, uint64_t bytes) {
    const double t = s->now();
    if (s->last_grow_fail >= 0 && t - s->last_grow_fail < kGrowRetrySeconds) return false;
    uint64_t want = std::max(bytes, kSegmentBytes);
    if (s->arena_cap) {
        if (s->arena_held + bytes > s->arena_cap) return false;  // wait for a finished request's room
        want = std::min(want, s->arena_cap - s->arena_held);
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        s->last_grow_fail = t;
        return false;
    }
    if (free_b < want + kHbmReserve) want = bytes;  // take only what this request needs
    uint8_t* p = nullptr;
    if (free_b < want + kHbmReserve || cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        s->last_grow_fail = t;
        return false;
    }
    ffbf_server::Segment g;
    g.base = p;
    g.bytes = want;
    g.free_ranges[0] = want;
    s->segs.push_back(std::move(g));
    s->arena_held += want;
    s->last_grow_fail = -1.0;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.arena_bytes = s->arena_held;
    return true;
}

bool arena_alloc(ffbf_server* s, uint64_t bytes, int* seg, uint64_t* off) {
    for (size_t i = 0; i < s->segs.size(); i++) {
        if (seg_alloc(s->segs[i], bytes, off)) {
            *seg = (int)i;
            return true;
        }
    }
    if (!arena_grow(s, bytes)) return false;
    *seg = (int)s->segs.size() - 1;
    return seg_alloc(s->segs.back(), bytes, off);
}

void arena_free(ffbf_server* s, int seg, uint64_t off, uint64_t bytes) { seg_free(s->segs[seg], off, bytes); }

uint64_t first_segment_bytes(const ffbf_server* s) {
    return s->arena_cap ? std::min(s->arena_cap, kSegmentBytes) : kSegmentBytes;
}

// With nothing admitted, the segments grown for earlier requests go back to the device, and a first segment
// that was rebuilt larger for one request returns to its first size (cudaFree waits for the device, which is
// idle then).
void arena_shrink(ffbf_server* s) {
    bool freed = false;
    while (s->segs.size() > 1) {
        auto& g = s->segs.back();
        if (g.free_ranges.size() != 1 || g.free_ranges.begin()->second != g.bytes) break;
        cudaFree(g.base);
        s->arena_held -= g.bytes;
        s->segs.pop_back();
        freed = true;
    }
    if (s->segs.size() == 1 && s->segs[0].bytes > first_segment_bytes(s) && s->segs[0].free_ranges.size() == 1 &&
        s->segs[0].free_ranges.begin()->second == s->segs[0].bytes) {
        auto& g = s->segs[0];
        cudaFree(g.base);
        s->arena_held -= g.bytes;
        g.bytes = first_segment_bytes(s);
        g.free_ranges.clear();
        if (cudaMalloc(&g.base, g.bytes) != cudaSuccess) {
            cudaGetLastError();
            s->segs.clear();  // the next admission grows a segment as memory allows
        } else {
            g.free_ranges[0] = g.bytes;
            s->arena_held += g.bytes;
        }
        freed = true;
    }
    if (freed) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(s->mu);
        s->stats.arena_bytes = s->arena_held;
    }
}

// With nothing admitted (so every segment is free), the arena is replaced by one segment that holds `bytes`:
// free segments that are each too small, or a cap that the existing segments already fill, would otherwise
// keep a request that fits the cap waiting for good. The server's own segments count as free memory here.
bool arena_rebuild(ffbf_server* s, uint64_t bytes) {
    const double t = s->now();
    if (s->last_grow_fail >= 0 && t - s->last_grow_fail < kGrowRetrySeconds) return false;
    uint64_t want = std::max(bytes, first_segment_bytes(s));
    if (s->arena_cap) want = std::min(want, s->arena_cap);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b + s->arena_held < want + kHbmReserve) {
        cudaGetLastError();
        s->last_grow_fail = t;
        return false;
    }
    for (auto& g : s->segs) cudaFree(g.base);
    s->segs.clear();
    s->arena_held = 0;
    ffbf_server::Segment g;
    if (cudaMalloc(&g.base, want) != cudaSuccess) {
        cudaGetLastError();
        s->last_grow_fail = t;
        std::lock_guard<std::mutex> lk(s->mu);
        s->stats.arena_bytes = 0;
        return false;  // the next admission grows a segment as memory allows
    }
    g.bytes = want;
    g.free_ranges[0] = want;
    s->segs.push_back(std::move(g));
    s->arena_held = want;
    s->last_grow_fail = -1.0;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.arena_bytes = s->arena_held;
    return true;
}

// No request holds a slot: nothing is copying, ready, on the device or being collected.
bool nothing_admitted(const ffbf_server* s) {
    return s->copying.empty() && s->ready.empty() && !s->in_flight && s->resolving.empty() && s->slow.empty() &&
           s->running.empty();
}

// Ends a request: its slot and arena range return to the pools and it joins the finished queue.
void finish(ffbf_server* s, Request* r, ffbf_status st) {
    r->status = st;
    r->t_done = s->now();
    if (r->slot >= 0) s->free_slots.push_back(r->slot);
    if (r->span) arena_free(s, r->seg, r->off, r->span);
    r->slot = -1;
    r->span = 0;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.requests_done++;
    if (st == FFBF_OK) s->stats.bytes_scanned += r->len;
    s->done.push_back(r);
    s->cv_done.notify_all();
}

void admit(ffbf_server* s) {
    while (!s->pending.empty() && !s->free_slots.empty()) {
        Request* r = s->pending.front();
        const uint64_t span = (r->len + kArenaAlign - 1) / kArenaAlign * kArenaAlign;
        uint64_t off = 0;
        int seg = 0;
        if (span && !arena_alloc(s, span, &seg, &off) &&
            !(nothing_admitted(s) && arena_rebuild(s, span) && arena_alloc(s, span, &seg, &off)))
            break;  // in order: wait for room
        s->pending.pop_front();
        r->slot = s->free_slots.back();
        s->free_slots.pop_back();
        r->seg = seg;
        r->off = off;
        r->span = span;
        r->t_admit = s->now();
        cudaStream_t cs = r->len <= kSmallCopy ? s->st_copy_small : s->st_copy;
        if (r->len && cudaMemcpyAsync(s->segs[seg].base + off, r->h_text, r->len, cudaMemcpyHostToDevice, cs) !=
                          cudaSuccess) {
            cudaGetLastError();
            finish(s, r, FFBF_ECUDA);
            continue;
        }
        cudaEventRecord(s->copy_done[r->slot], cs);
        s->copying.push_back(r);
    }
}

bool ensure_tail(ffbf_server* s, size_t n) {
    if (n <= s->tail_cap) return true;
    size_t cap = std::max(n, 2 * s->tail_cap);
    if (s->d_tail) cudaFree(s->d_tail);
    if (s->h_tail) cudaFreeHost(s->h_tail);
    s->d_tail = nullptr;
    s->h_tail = nullptr;
    s->tail_cap = 0;
    if (cudaMalloc(&s->d_tail, cap * sizeof(uint2)) != cudaSuccess ||
        cudaMallocHost(&s->h_tail, cap * sizeof(uint2)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    s->tail_cap = cap;
    return true;
}

// Launches every ready request as one plan on the scan stream.
void launch_ready(ffbf_server* s) {
    NvtxRange nvtx_("server batch launch");
    std::vector<PlanJob> jobs;
    std::vector<Request*> batch;
    for (Request* r : s->ready) {
        ffbf_ctx* slot = s->slots[r->slot];
        attach_filters(slot, s->sets[r->set]);
        jobs.push_back({slot, s->segs[r->seg].base + r->off, r->len});
        batch.push_back(r);
    }
    s->ready.clear();
    ScanPlan plan;
    size_t bad = 0;
    ffbf_status st = build_plan(jobs, s->num_sms, plan, &bad);
    if (st == FFBF_OK && plan.launches.size() + 1 > kMaxCtl) st = FFBF_EINVAL;
    if (st == FFBF_OK && !ensure_tail(s, plan.tail.size() + 1)) st = FFBF_ENOMEM_DEVICE;
    if (st != FFBF_OK) {
        if (st != FFBF_EINVAL && bad < jobs.size()) set_err(s, jobs[bad].c->err);
        for (Request* r : batch) finish(s, r, st);
        return;
    }
    const uint32_t n = (uint32_t)jobs.size();
    const uint32_t n_ctl = (uint32_t)plan.launches.size() + 1;
    std::copy(plan.fast.begin(), plan.fast.end(), s->h_fast);
    std::copy(plan.args.begin(), plan.args.end(), s->h_args);
    std::copy(plan.tail.begin(), plan.tail.end(), s->h_tail);
    for (uint32_t i = 0; i < n; i++) s->h_counters[i] = jobs[i].c->d_counters;
    for (uint32_t i = 0; i < n_ctl; i++) s->h_counters[n + i] = s->d_ctl + 4 * i;
    PlanDevice d{s->d_fast, s->d_args, s->d_tail, s->d_counters, n + n_ctl, s->d_ctl};
    cudaError_t e = cudaSuccess;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->st_scan);
    };
    up(s->d_fast, s->h_fast, plan.fast.size() * sizeof(ffbf::FastJob));
    up(s->d_args, s->h_args, plan.args.size() * sizeof(ffbf::ScanArgs));
    up(s->d_tail, s->h_tail, plan.tail.size() * sizeof(uint2));
    up(s->d_counters, s->h_counters, (n + n_ctl) * sizeof(uint32_t*));
    const double t = s->now();
    if (e == cudaSuccess) e = launch_plan(plan, d, s->num_sms, s->st_scan);
    if (e == cudaSuccess) e = ffbf::gather_counters(s->d_counters, n, s->d_cnt, s->st_scan);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_cnt, s->d_cnt, 4 * ffbf::CNT_WORDS * n, cudaMemcpyDeviceToHost, s->st_scan);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_ctl, s->d_ctl, 16 * n_ctl, cudaMemcpyDeviceToHost, s->st_scan);
    if (e == cudaSuccess) e = cudaEventRecord(s->batch_done, s->st_scan);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_err(s, std::string("batch launch failed: ") + cudaGetErrorString(e));
        for (Request* r : batch) finish(s, r, FFBF_ECUDA);
        return;
    }
    for (Request* r : batch) r->t_launch = t;
    s->running = batch;
    s->batch_ctl = n_ctl;
    s->in_flight = true;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.batches++;
    s->stats.max_batch = std::max<uint64_t>(s->stats.max_batch, n);
}

// The plain collect: waits on the slot's stream, grows the hit buffer and rescans when needed.
void collect_slow(ffbf_server* s) {
    Request* r = s->slow.front();
    s->slow.erase(s->slow.begin());
    ffbf_ctx* slot = s->slots[r->slot];
    ffbf_scan_result res{};
    ffbf_status st = ffbf_scan_collect(slot, &res);
    if (st == FFBF_OK) {
        r->hits.assign(res.hit_offsets, res.hit_offsets + res.n_hits);
        r->ls.assign(res.line_start, res.line_start + res.n_lines);
        r->le.assign(res.line_end, res.line_end + res.n_lines);
    } else {
        set_err(s, slot->err);
    }
    finish(s, r, st);
}

// Enqueues line resolution and the copy of the hit records for a request of a finished batch.
ffbf_status start_resolve(ffbf_server* s, Request* r) {
    ffbf_ctx* c = s->slots[r->slot];
    auto& h = s->slot_host[r->slot];
    const uint32_t nh = r->nh;
    if (nh > h.cap) {
        if (h.hr) cudaFreeHost(h.hr);
        if (h.hl) cudaFreeHost(h.hl);
        h.hr = nullptr;
        h.hl = nullptr;
        h.cap = 0;
        const uint32_t cap = std::max<uint32_t>(nh, 4096);
        if (cudaMallocHost(&h.hr, cap * sizeof(HitRec)) != cudaSuccess ||
            cudaMallocHost(&h.hl, cap * sizeof(HitLine)) != cudaSuccess) {
            cudaGetLastError();
            return FFBF_ENOMEM_HOST;
        }
        h.cap = cap;
    }
    const uint64_t ntiles = (c->text_len + ffbf::kScanTile - 1) / ffbf::kScanTile;
    cudaError_t e = ffbf::resolve_lines(c->d_text, c->text_len, c->g.len, c->d_hits, nh, c->d_tiles,
                                        c->d_tiles + c->tiles_cap, c->d_tiles + 2 * c->tiles_cap,
                                        c->d_tiles + 3 * c->tiles_cap, ntiles, c->d_hitlines, c->st,
                                        c->d_tiles + 4 * c->tiles_cap);
    if (e == cudaSuccess && nh)
        e = cudaMemcpyAsync(h.hr, c->d_hits, nh * sizeof(HitRec), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess && nh)
        e = cudaMemcpyAsync(h.hl, c->d_hitlines, nh * sizeof(HitLine), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaEventRecord(h.done, c->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_err(s, std::string("result copy failed: ") + cudaGetErrorString(e));
        return FFBF_ECUDA;
    }
    return FFBF_OK;
}

// Finishes the requests whose result copies have landed.
bool finish_resolved(ffbf_server* s) {
    bool any = false;
    for (size_t i = 0; i < s->resolving.size();) {
        Request* r = s->resolving[i];
        auto& h = s->slot_host[r->slot];
        const cudaError_t q = cudaEventQuery(h.done);
        if (q == cudaErrorNotReady) {
            i++;
            continue;
        }
        s->resolving.erase(s->resolving.begin() + i);
        if (q == cudaSuccess) {
            order_hits(h.hr, h.hl, r->nh, r->hits, r->ls, r->le);
            finish(s, r, FFBF_OK);
        } else {
            cudaGetLastError();
            finish(s, r, FFBF_ECUDA);
        }
        any = true;
    }
    return any;
}

void worker_loop(ffbf_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            const bool idle = s->pending.empty() && s->copying.empty() && s->ready.empty() && !s->in_flight &&
                              s->resolving.empty() && s->slow.empty();
            if (idle && s->inbox.empty() && !s->stop) s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
            while (!s->inbox.empty()) {
                s->pending.push_back(s->inbox.front());
                s->inbox.pop_front();
            }
            if (s->stop) break;
        }
        bool progress = false;
        const size_t before = s->copying.size();
        admit(s);
        progress |= s->copying.size() != before;
        for (size_t i = 0; i < s->copying.size();) {
            Request* r = s->copying[i];
            cudaError_t q = cudaEventQuery(s->copy_done[r->slot]);
            if (q == cudaErrorNotReady) {
                i++;
                continue;
            }
            s->copying.erase(s->copying.begin() + i);
            if (q != cudaSuccess) {
                cudaGetLastError();
                finish(s, r, FFBF_ECUDA);
            } else {
                s->ready.push_back(r);
            }
            progress = true;
        }
        if (s->in_flight) {
            cudaError_t q = cudaEventQuery(s->batch_done);
            if (q != cudaErrorNotReady) {
                s->in_flight = false;
                uint32_t flags = 0;
                for (uint32_t i = 0; i < s->batch_ctl; i++) flags |= s->h_ctl[4 * i];
                const ffbf_status st = q != cudaSuccess ? FFBF_ECUDA : flags & 4u ? FFBF_ETIMEOUT : flags ? FFBF_ECUDA : FFBF_OK;
                if (q != cudaSuccess) cudaGetLastError();
                std::vector<Request*> done_batch;
                done_batch.swap(s->running);
                // hit counts first: the next batch's readback reuses the pinned buffer
                for (size_t i = 0; i < done_batch.size(); i++)
                    done_batch[i]->nh = s->h_cnt[ffbf::CNT_WORDS * i + ffbf::CNT_HITS];
                // the GPU is idle: start the next batch before resolving this one's results
                if (!s->ready.empty()) launch_ready(s);
                for (Request* r : done_batch) {
                    if (st != FFBF_OK) {
                        finish(s, r, st);
                        continue;
                    }
                    if (r->nh > s->slots[r->slot]->hits_cap) {
                        s->slow.push_back(r);
                        continue;
                    }
                    const ffbf_status rs = start_resolve(s, r);
                    if (rs == FFBF_OK) s->resolving.push_back(r);
                    else finish(s, r, rs);
                }
                progress = true;
            }
        }
        if (!s->in_flight && !s->ready.empty()) {
            launch_ready(s);
            progress = true;
        }
        progress |= finish_resolved(s);
        if (!s->slow.empty()) {
            collect_slow(s);
            progress = true;
        }
        // With nothing admitted for a while, segments grown for earlier requests go back to the device.
        const bool quiet = nothing_admitted(s);
        if (quiet && s->pending.empty()) {
            if (s->idle_since < 0) s->idle_since = s->now();
            else if ((s->segs.size() > 1 || (s->segs.size() == 1 && s->segs[0].bytes > first_segment_bytes(s))) &&
                     s->now() - s->idle_since > kShrinkIdleSeconds)
                arena_shrink(s);
        } else {
            s->idle_since = -1.0;
        }
        // Requests on the device or in copies: poll again at once (a sleep rounds up to tens of microseconds
        // on every stage of a request); with nothing in flight the loop waits on cv_work above. Pending requests
        // that wait for device memory other contexts hold are retried after a pause.
        if (!progress) {
            if (quiet && !s->pending.empty()) std::this_thread::sleep_for(std::chrono::microseconds(200));
            else std::this_thread::yield();
        }
    }
    // stopping: let the device finish what was issued, then drop what is left
    cudaStreamSynchronize(s->st_copy);
    cudaStreamSynchronize(s->st_copy_small);
    cudaStreamSynchronize(s->st_scan);
    for (auto* c : s->slots) cudaStreamSynchronize(c->st);
    cudaGetLastError();
}

void server_free(ffbf_server* s) {
    cudaSetDevice(s->device);
    for (auto* c : s->slots) ffbf_destroy(c);
    for (auto ev : s->copy_done) cudaEventDestroy(ev);
    for (auto& h : s->slot_host) {
        if (h.hr) cudaFreeHost(h.hr);
        if (h.hl) cudaFreeHost(h.hl);
        if (h.done) cudaEventDestroy(h.done);
    }
    if (s->batch_done) cudaEventDestroy(s->batch_done);
    for (auto& g : s->segs) cudaFree(g.base);
    s->segs.clear();
    for (void* p : {(void*)s->d_fast, (void*)s->d_args, (void*)s->d_counters, (void*)s->d_ctl,
                    (void*)s->d_tail, (void*)s->d_cnt})
        if (p) cudaFree(p);
    for (void* p : {(void*)s->h_fast, (void*)s->h_args, (void*)s->h_counters, (void*)s->h_tail, (void*)s->h_ctl,
                    (void*)s->h_cnt})
        if (p) cudaFreeHost(p);
    if (s->st_scan) cudaStreamDestroy(s->st_scan);
    if (s->st_copy) cudaStreamDestroy(s->st_copy);
    if (s->st_copy_small) cudaStreamDestroy(s->st_copy_small);
    auto drop = [](std::deque<Request*>& q) {
        for (auto* r : q) delete r;
        q.clear();
    };
    drop(s->inbox);
    drop(s->pending);
    drop(s->done);
    for (auto* v : {&s->copying, &s->ready, &s->running, &s->resolving, &s->slow}) {
        for (auto* r : *v) delete r;
        v->clear();
    }
    for (auto& kv : s->owned) delete kv.second;
    s->owned.clear();
    cudaGetLastError();
    delete s;
}

}  // namespace

extern "C" {

ffbf_status ffbf_server_create(int device, uint64_t arena_bytes, uint32_t slots, ffbf_server** out) {
    if (!out) return FFBF_EINVAL;
    *out = nullptr;
    ffbf_server* s = new (std::nothrow) ffbf_server();
    if (!s) return FFBF_ENOMEM_HOST;
    s->device = device;
    s->t0 = Clock::now();
    if (slots == 0) slots = 64;
    auto bail = [&](ffbf_status st) {
        server_free(s);
        return st;
    };
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess ||
        cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->st_scan, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->st_copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->st_copy_small, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->batch_done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return bail(FFBF_ECUDA);
    }
    // the arena starts as one segment and grows by free device memory up to the cap (0: no cap)
    s->arena_cap = arena_bytes / kArenaAlign * kArenaAlign;
    s->device_bytes = total_b;
    uint64_t first = s->arena_cap ? std::min(s->arena_cap, kSegmentBytes) : kSegmentBytes;
    if (first + kHbmReserve > free_b)
        first = free_b > kHbmReserve ? (free_b - kHbmReserve) / kArenaAlign * kArenaAlign : 0;
    if (first == 0) return bail(FFBF_ENOMEM_DEVICE);
    {
        ffbf_server::Segment g;
        if (cudaMalloc(&g.base, first) != cudaSuccess) {
            cudaGetLastError();
            return bail(FFBF_ENOMEM_DEVICE);
        }
        g.bytes = first;
        g.free_ranges[0] = first;
        s->segs.push_back(std::move(g));
        s->arena_held = first;
    }
    const size_t n_counters = slots + kMaxCtl;
    if (cudaMalloc(&s->d_fast, slots * sizeof(ffbf::FastJob)) != cudaSuccess ||
        cudaMalloc(&s->d_args, slots * sizeof(ffbf::ScanArgs)) != cudaSuccess ||
        cudaMalloc(&s->d_counters, n_counters * sizeof(uint32_t*)) != cudaSuccess ||
        cudaMalloc(&s->d_ctl, 16 * kMaxCtl) != cudaSuccess ||
        cudaMallocHost(&s->h_fast, slots * sizeof(ffbf::FastJob)) != cudaSuccess ||
        cudaMallocHost(&s->h_args, slots * sizeof(ffbf::ScanArgs)) != cudaSuccess ||
        cudaMallocHost(&s->h_counters, n_counters * sizeof(uint32_t*)) != cudaSuccess ||
        cudaMallocHost(&s->h_ctl, 16 * kMaxCtl) != cudaSuccess ||
        cudaMalloc(&s->d_cnt, 4 * ffbf::CNT_WORDS * (size_t)slots) != cudaSuccess ||
        cudaMallocHost(&s->h_cnt, 4 * ffbf::CNT_WORDS * (size_t)slots) != cudaSuccess || !ensure_tail(s, 4096)) {
        cudaGetLastError();
        return bail(FFBF_ENOMEM_DEVICE);
    }
    // Slots get their scan buffers up front, sized for requests of up to kPreallocText bytes (tile
    // summaries, 64k hit records, pinned copies for 16k hits), so that serving rarely allocates: an
    // allocation inside the loop would synchronise the device and stall every request in flight.
    const uint64_t prealloc_len = kPreallocText;
    for (uint32_t i = 0; i < slots; i++) {
        ffbf_ctx* c = nullptr;
        ffbf_status st = create_scan_slot(device, &c);
        if (st != FFBF_OK) return bail(st);
        s->slots.push_back(c);
        // (the pointer only sizes the buffers: nothing is read from it here)
        if ((st = setup_scan_state(c, s->segs[0].base, prealloc_len)) != FFBF_OK || (st = prepare_fast(c)) != FFBF_OK)
            return bail(st);
        reset_scan(c);
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return bail(FFBF_ECUDA);
        }
        s->copy_done.push_back(ev);
        s->slot_host.emplace_back();
        auto& h = s->slot_host.back();
        if (cudaEventCreateWithFlags(&h.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost(&h.hr, kPreallocHits * sizeof(HitRec)) != cudaSuccess ||
            cudaMallocHost(&h.hl, kPreallocHits * sizeof(HitLine)) != cudaSuccess) {
            cudaGetLastError();
            return bail(FFBF_ENOMEM_HOST);
        }
        h.cap = kPreallocHits;
        s->free_slots.push_back((int)(slots - 1 - i));
    }
    s->stats.arena_bytes = s->arena_held;
    s->stats.slots = slots;
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return FFBF_OK;
}

ffbf_status ffbf_server_add_set(ffbf_server* s, ffbf_ctx* set, uint32_t* set_id) {
    if (!s || !set || !set_id) return FFBF_EINVAL;
    if (set->device != s->device) return sfail(s, FFBF_EINVAL, "the set's context is on another device");
    bool started;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        started = s->started;
    }
    if (started) return sfail(s, FFBF_ESTATE, "sets are registered before the first submit");
    ffbf_status st = enter(set);
    if (st == FFBF_OK && ffbf::fast_scan_supported(set->g, ffbf::kScanTile) && !set->force_generic) st = prepare_fast(set);
    if (st == FFBF_OK) st = sync(set);
    if (st != FFBF_OK) return sfail(s, st, std::string("set preparation failed: ") + set->err);
    *set_id = (uint32_t)s->sets.size();
    s->sets.push_back(set);
    return FFBF_OK;
}

ffbf_status ffbf_server_submit(ffbf_server* s, uint32_t set_id, const uint8_t* text, size_t len, uint64_t* request_id) {
    if (!s || !request_id) return FFBF_EINVAL;
    if (set_id >= s->sets.size()) return sfail(s, FFBF_EINVAL, "unknown set");
    if (!text && len) return sfail(s, FFBF_EINVAL, "text is NULL");
    const uint64_t span = (len + kArenaAlign - 1) / kArenaAlign * kArenaAlign;
    if ((s->arena_cap && span > s->arena_cap) || span + kHbmReserve > s->device_bytes)
        return sfail(s, FFBF_EINVAL, "request text is larger than the server's text arena can grow");
    Request* r = new (std::nothrow) Request();
    if (!r) return FFBF_ENOMEM_HOST;
    r->set = set_id;
    r->h_text = text;
    r->len = len;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->started = true;
        r->id = s->next_id++;
        r->t_submit = s->now();
        s->inbox.push_back(r);
    }
    s->cv_work.notify_one();
    *request_id = r->id;
    return FFBF_OK;
}

ffbf_status ffbf_server_poll(ffbf_server* s, ffbf_request_result* out, uint32_t max, uint32_t* n_out,
                             uint32_t wait_us) {
    if (!s || !n_out || (max && !out)) return FFBF_EINVAL;
    *n_out = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_us)
        s->cv_done.wait_for(lk, std::chrono::microseconds(wait_us), [&] { return !s->done.empty(); });
    while (*n_out < max && !s->done.empty()) {
        Request* r = s->done.front();
        s->done.pop_front();
        s->owned[r->id] = r;
        ffbf_request_result& o = out[(*n_out)++];
        o.request_id = r->id;
        o.set_id = r->set;
        o.status = r->status;
        o.text_len = r->len;
        o.n_hits = r->hits.size();
        o.hit_offsets = r->hits.data();
        o.n_lines = r->ls.size();
        o.line_start = r->ls.data();
        o.line_end = r->le.data();
        o.t_submit = r->t_submit;
        o.t_admit = r->t_admit;
        o.t_launch = r->t_launch;
        o.t_done = r->t_done;
    }
    return FFBF_OK;
}

ffbf_status ffbf_server_release(ffbf_server* s, uint64_t request_id) {
    if (!s) return FFBF_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->owned.find(request_id);
    if (it == s->owned.end()) return FFBF_EINVAL;
    delete it->second;
    s->owned.erase(it);
    return FFBF_OK;
}

ffbf_status ffbf_server_get_stats(ffbf_server* s, ffbf_server_stats* out) {
    if (!s || !out) return FFBF_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    return FFBF_OK;
}

const char* ffbf_server_last_error(const ffbf_server* s) {
    if (!s) return "null server";
    // a copy per calling thread: the worker may set a new message meanwhile
    static thread_local std::string copy;
    std::lock_guard<std::mutex> lk(const_cast<ffbf_server*>(s)->mu);
    copy = s->err;
    return copy.c_str();
}

void ffbf_server_destroy(ffbf_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    server_free(s);
}

}  // extern "C"
