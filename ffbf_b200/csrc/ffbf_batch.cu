// ffbf_batch.cu -- many scans in one launch sequence: the job plan shared by the batch API and the server,
// the batch API (ffbf_batch_*: a fixed set of jobs captured once in a CUDA graph and launched repeatedly),
// and the autotuner of a context's scan configuration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "ffbf_ctx.cuh"

using namespace ffbf_host;

struct ffbf_batch {
    int device = 0;
    int num_sms = 0;
    cudaStream_t st = nullptr;
    std::string err;
    struct Job {
        ffbf_ctx* c;
        const uint8_t* text;
        size_t len;
    };
    // The device buffers and configuration each job's descriptors were built from. A context that has
    // since grown its hit buffer, reloaded its filter, added patterns or been retuned makes the batch
    // prepare again before its next launch.
    struct Key {
        const void *main, *ff, *hits, *counters, *tiles, *stage1;
        uint32_t hits_cap;
        uint64_t tiles_cap;
        int threads, mode;
        uint32_t rows;
        int order;
        bool operator==(const Key& o) const {
            return main == o.main && ff == o.ff && hits == o.hits && counters == o.counters && tiles == o.tiles &&
                   stage1 == o.stage1 && hits_cap == o.hits_cap && tiles_cap == o.tiles_cap && threads == o.threads &&
                   mode == o.mode && rows == o.rows && order == o.order;
        }
    };
    std::vector<Key> keys;
    std::vector<Job> jobs;
    bool prepared = false;
    std::vector<void*> allocs;
    uint32_t* d_error = nullptr;  // n_ctl groups of 4 words: error flags, work-queue counter
    uint32_t n_ctl = 0;
    uint64_t graph_kernels = 0;  // kernel nodes of the graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // branch streams and events used while capturing the graph's parallel branches
    std::vector<cudaStream_t> branches;
    std::vector<cudaEvent_t> events;
};


namespace ffbf_host {

ffbf_status build_plan(const std::vector<PlanJob>& jobs, int num_sms, ScanPlan& plan, size_t* bad) {
    plan = ScanPlan{};
    struct Group {
        uint32_t len;
        ffbf::FastConfig cfg;
        std::vector<std::pair<uint64_t, ffbf::FastJob>> jobs;  // (bytes, descriptor)
    };
    std::vector<Group> groups;
    for (size_t i = 0; i < jobs.size(); i++) {
        ffbf_ctx* c = jobs[i].c;
        *bad = i;
        TRY(enter(c));
        TRY(setup_scan_state(c, jobs[i].text, jobs[i].len));
        const ffbf::ScanArgs a = make_scan_args(c);
        plan.args.push_back(a);
        uint64_t covered = 0;
        if (use_fast(c, a.n)) {
            TRY(prepare_fast(c));
            const ffbf::FastConfig cfg = c->cfg;
            const int threads = ffbf::config_threads(cfg);
            // in a batch other jobs fill the GPU, so rows per stream follow this job's size alone
            const uint32_t rows = cfg.rows ? cfg.rows : ffbf::fast_rows(a.n, cfg, num_sms, true);
            ffbf::FastJob fj;
            cudaError_t e;
            covered = ffbf::fill_fast_job(a, c->d_stage1, cfg, rows, &fj, &e);
            if (e != cudaSuccess) return fail(c, FFBF_ECUDA, "tensor map encoding failed");
            if (fj.n_supertiles) {
                Group* gp = nullptr;
                for (auto& g : groups)
                    if (g.len == c->g.len && g.cfg.mode == cfg.mode && ffbf::config_threads(g.cfg) == threads &&
                        (cfg.mode != 1 || g.cfg.order == cfg.order))
                        gp = &g;
                if (!gp) {
                    groups.push_back(Group{c->g.len, cfg, {}});
                    gp = &groups.back();
                }
                gp->jobs.push_back({covered, fj});
            }
        }
        for (uint64_t t = covered / ffbf::kScanTile; t < a.ntiles; t++)
            plan.tail.push_back(make_uint2((uint32_t)i, (uint32_t)t));
        CUDA_TRY(c, cudaStreamSynchronize(c->st));  // stage-1 tables built on the context's stream
        c->scan_pending = true;
    }
    // descriptors: groups contiguous, largest jobs first within a group (the work queue hands out the
    // largest items first, so the last wave is made of small ones)
    for (auto& g : groups) {
        std::stable_sort(g.jobs.begin(), g.jobs.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        PlanLaunch L{g.len, g.cfg, plan.fast.size(), (uint32_t)g.jobs.size(), 0, 0};
        for (auto& jb : g.jobs) {
            jb.second.item_begin = L.n_items;
            L.n_items += jb.second.n_supertiles;
            L.max_s1 = std::max(L.max_s1, jb.second.stage1_nwords);
            plan.fast.push_back(jb.second);
        }
        plan.launches.push_back(L);
    }
    return FFBF_OK;
}

cudaError_t launch_plan(const ScanPlan& p, const PlanDevice& d, int num_sms, cudaStream_t st,
                        const cudaStream_t* branches, const cudaEvent_t* events) {
    cudaError_t e = ffbf::zero_counters(d.counters, d.n_counters, st);
    const size_t nl = p.launches.size();
    if (!branches) {
        for (size_t li = 0; li < nl && e == cudaSuccess; li++) {
            const PlanLaunch& L = p.launches[li];
            e = ffbf::launch_fast_jobs(L.len, L.cfg, d.fast + L.off, L.n_jobs, L.n_items, L.max_s1, d.ctl + 4 * li,
                                       num_sms, st);
        }
        if (e == cudaSuccess) e = ffbf::scan_generic_multi(d.args, d.tail, (uint32_t)p.tail.size(), num_sms, st);
        return e;
    }
    // fork: each tuned launch and the generic launch on its own branch (they touch disjoint tiles), join
    // back on st; a branch's kernel takes SMs as the others' work queues drain
    if (e == cudaSuccess) e = cudaEventRecord(events[0], st);
    for (size_t li = 0; li <= nl && e == cudaSuccess; li++) {
        cudaStream_t bs = branches[li];
        e = cudaStreamWaitEvent(bs, events[0], 0);
        if (e == cudaSuccess && li < nl) {
            const PlanLaunch& L = p.launches[li];
            e = ffbf::launch_fast_jobs(L.len, L.cfg, d.fast + L.off, L.n_jobs, L.n_items, L.max_s1, d.ctl + 4 * li,
                                       num_sms, bs);
        } else if (e == cudaSuccess) {
            e = ffbf::scan_generic_multi(d.args, d.tail, (uint32_t)p.tail.size(), num_sms, bs);
        }
        if (e == cudaSuccess) e = cudaEventRecord(events[1 + li], bs);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, events[1 + li], 0);
    }
    return e;
}

}  // namespace ffbf_host

namespace {

ffbf_status autotune_impl(ffbf_ctx* c, const uint8_t* d_text, size_t sample_len, bool per_sm, int* threads,
                          int* mode);

ffbf_batch::Key batch_key(const ffbf_ctx* c) {
    return ffbf_batch::Key{c->d_main, c->d_ff,          c->d_hits,      c->d_counters, c->d_tiles,
                           c->d_stage1, c->hits_cap,    c->tiles_cap,   c->cfg.threads, c->cfg.mode,
                           c->cfg.rows, c->cfg.order};
}

ffbf_status bfail(ffbf_batch* b, ffbf_status s, const std::string& msg) {
    b->err = msg;
    return s;
}

void batch_release(ffbf_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto s : b->branches) cudaStreamDestroy(s);
    for (auto e : b->events) cudaEventDestroy(e);
    b->branches.clear();
    b->events.clear();
    b->exec = nullptr;
    b->graph = nullptr;
    for (void* p : b->allocs) cudaFree(p);
    b->allocs.clear();
    b->d_error = nullptr;
    b->prepared = false;
    b->keys.clear();
    cudaGetLastError();
}

template <class T>
ffbf_status balloc(ffbf_batch* b, T** p, size_t count) {
    void* v = nullptr;
    if (cudaMalloc(&v, count * sizeof(T) + 16) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, FFBF_ENOMEM_DEVICE, "batch table allocation failed");
    }
    b->allocs.push_back(v);
    *p = static_cast<T*>(v);
    return FFBF_OK;
}

}  // namespace

extern "C" {

ffbf_status ffbf_batch_create(int device, ffbf_batch** out) {
    if (!out) return FFBF_EINVAL;
    *out = nullptr;
    ffbf_batch* b = new (std::nothrow) ffbf_batch();
    if (!b) return FFBF_ENOMEM_HOST;
    b->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return FFBF_ECUDA;
    }
    *out = b;
    return FFBF_OK;
}

void ffbf_batch_destroy(ffbf_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    batch_release(b);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

const char* ffbf_batch_last_error(const ffbf_batch* b) { return b ? b->err.c_str() : "null batch"; }

void* ffbf_batch_stream(ffbf_batch* b) { return b ? (void*)b->st : nullptr; }

ffbf_status ffbf_batch_add(ffbf_batch* b, ffbf_ctx* c, const uint8_t* d_text, size_t len) {
    if (!b || !c) return FFBF_EINVAL;
    if (c->device != b->device) return bfail(b, FFBF_EINVAL, "context and batch are on different devices");
    if (((uintptr_t)d_text & 15) != 0 || (!d_text && len)) return bfail(b, FFBF_EINVAL, "device text must be 16-byte aligned");
    for (auto& j : b->jobs)
        if (j.c == c) return bfail(b, FFBF_EINVAL, "a context may appear only once in a batch");
    if (b->prepared) batch_release(b);
    b->jobs.push_back({c, d_text, len});
    return FFBF_OK;
}

ffbf_status ffbf_batch_prepare(ffbf_batch* b) {
    NvtxRange nvtx_("ffbf_batch_prepare");
    if (!b) return FFBF_EINVAL;
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, FFBF_ECUDA, "cudaSetDevice failed");
    batch_release(b);
    std::vector<PlanJob> pj;
    for (const auto& j : b->jobs) pj.push_back({j.c, j.text, j.len});
    ScanPlan plan;
    size_t bad = 0;
    ffbf_status s = build_plan(pj, b->num_sms, plan, &bad);
    if (s != FFBF_OK) return bfail(b, s, "job " + std::to_string(bad) + ": " + b->jobs[bad].c->err);
    std::vector<uint32_t*> counters;
    for (const auto& j : b->jobs) {
        b->keys.push_back(batch_key(j.c));
        counters.push_back(j.c->d_counters);
    }
    PlanDevice d{};
    TRY(balloc(b, &d.fast, plan.fast.size() + 1));
    TRY(balloc(b, &d.args, plan.args.size() + 1));
    TRY(balloc(b, &d.tail, plan.tail.size() + 1));
    TRY(balloc(b, &b->d_error, 4 * (plan.launches.size() + 1)));
    b->n_ctl = (uint32_t)plan.launches.size() + 1;
    d.ctl = b->d_error;
    for (uint32_t i = 0; i < b->n_ctl; i++) counters.push_back(b->d_error + 4 * i);
    TRY(balloc(b, &d.counters, counters.size() + 1));
    d.n_counters = (uint32_t)counters.size();
    auto up = [](void* dst, const void* src, size_t bytes) {
        return bytes == 0 || cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!up(d.fast, plan.fast.data(), plan.fast.size() * sizeof(ffbf::FastJob)) ||
        !up(d.args, plan.args.data(), plan.args.size() * sizeof(ffbf::ScanArgs)) ||
        !up(d.tail, plan.tail.data(), plan.tail.size() * sizeof(uint2)) ||
        !up(d.counters, counters.data(), counters.size() * sizeof(uint32_t*)) ||
        cudaMemset(b->d_error, 0, 16 * b->n_ctl) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, FFBF_ECUDA, "batch table upload failed");
    }
    // one graph: zero the jobs' counters, one tuned launch per group, one generic launch for all tail tiles
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return bfail(b, FFBF_ECUDA, "stream capture failed to start");
    for (size_t i = 0; i <= plan.launches.size(); i++) {
        cudaStream_t bs;
        if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return bfail(b, FFBF_ECUDA, "branch stream creation failed");
        }
        b->branches.push_back(bs);
    }
    for (size_t i = 0; i <= plan.launches.size() + 1; i++) {
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return bfail(b, FFBF_ECUDA, "event creation failed");
        }
        b->events.push_back(ev);
    }
    const uint64_t launches0 = ffbf::launches_total();
    cudaError_t e = launch_plan(plan, d, b->num_sms, b->st, b->branches.data(), b->events.data());
    cudaError_t e2 = cudaStreamEndCapture(b->st, &b->graph);
    b->graph_kernels = ffbf::launches_total() - launches0;  // counted again at each graph launch
    ffbf::unnote_launches(b->graph_kernels);
    if (e != cudaSuccess || e2 != cudaSuccess || cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, FFBF_ECUDA,
                     std::string("batch graph capture failed: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    b->prepared = true;
    return FFBF_OK;
}

ffbf_status ffbf_batch_launch(ffbf_batch* b) {
    NvtxRange nvtx_("ffbf_batch_launch");
    if (!b) return FFBF_EINVAL;
    bool stale = !b->prepared || b->keys.size() != b->jobs.size();
    for (size_t i = 0; i < b->jobs.size() && !stale; i++)
        stale = !(batch_key(b->jobs[i].c) == b->keys[i]) ||
                (use_fast(b->jobs[i].c, b->jobs[i].len) && b->jobs[i].c->stage1_dirty);
    if (stale) TRY(ffbf_batch_prepare(b));
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, FFBF_ECUDA, "cudaSetDevice failed");
    for (auto& j : b->jobs) {
        reset_scan(j.c);
        j.c->d_text = j.text;
        j.c->text_len = j.len;
        j.c->scan_pending = true;
    }
    if (cudaGraphLaunch(b->exec, b->st) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, FFBF_ECUDA, "graph launch failed");
    }
    ffbf::note_launches(b->graph_kernels);
    return FFBF_OK;
}

ffbf_status ffbf_batch_wait(ffbf_batch* b) {
    if (!b) return FFBF_EINVAL;
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, FFBF_ECUDA, std::string("batch execution failed: ") + cudaGetErrorString(e));
    }
    uint32_t flag = 0;
    if (b->d_error) {
        std::vector<uint32_t> ctl(4 * b->n_ctl);
        if (cudaMemcpy(ctl.data(), b->d_error, 16 * b->n_ctl, cudaMemcpyDeviceToHost) != cudaSuccess)
            return bfail(b, FFBF_ECUDA, "error flag read failed");
        for (uint32_t i = 0; i < b->n_ctl; i++) flag |= ctl[4 * i];
    }
    if (flag) {
        char buf[96];
        snprintf(buf, sizeof buf, "batched scan error flags 0x%x (4: a bounded wait gave up; others: self-checks)", flag);
        return bfail(b, (flag & 4u) ? FFBF_ETIMEOUT : FFBF_ECUDA, buf);
    }
    return FFBF_OK;
}

ffbf_status ffbf_batch_autotune(ffbf_batch* b, size_t sample_bytes, uint32_t* n_classes) {
    NvtxRange nvtx_("ffbf_batch_autotune");
    if (!b) return FFBF_EINVAL;
    if (n_classes) *n_classes = 0;
    // classes: jobs with the same geometry whose stage-1 tables are about as full (1/16 steps) scan alike
    struct Class {
        size_t rep;  // the class's largest job
        std::vector<size_t> members;
    };
    std::map<std::vector<uint64_t>, Class> classes;
    for (size_t i = 0; i < b->jobs.size(); i++) {
        ffbf_ctx* c = b->jobs[i].c;
        TRY(enter(c));
        if (!use_fast(c, b->jobs[i].len)) continue;
        TRY(prepare_fast(c));  // builds the stage-1 table and measures its fill
        const std::vector<uint64_t> key = {c->g.len, c->g.k, c->g.s, c->g.cache_bits, c->g.nbits,
                                           (uint64_t)(c->stage1_fill * 16.0)};
        auto it = classes.find(key);
        if (it == classes.end()) {
            classes[key] = Class{i, {i}};
        } else {
            it->second.members.push_back(i);
            if (b->jobs[i].len > b->jobs[it->second.rep].len) it->second.rep = i;
        }
    }
    for (auto& kv : classes) {
        const auto& rep = b->jobs[kv.second.rep];
        size_t n = std::min(sample_bytes ? sample_bytes : (size_t)16 << 20, rep.len);
        n = n / ffbf::kScanTile * ffbf::kScanTile;
        if (n < ffbf::kScanTile) continue;
        int threads = 0, mode = 0;
        ffbf_status s = autotune_impl(rep.c, rep.text, n, true, &threads, &mode);
        if (s != FFBF_OK) return bfail(b, s, std::string("autotune: ") + rep.c->err);
        for (size_t m : kv.second.members) {
            ffbf_ctx* c = b->jobs[m].c;
            c->cfg = rep.c->cfg;
            c->cfg_tuned = true;
        }
    }
    if (n_classes) *n_classes = (uint32_t)classes.size();
    batch_release(b);  // the next launch prepares with the tuned configurations
    return FFBF_OK;
}

}  // extern "C"

namespace {

// Times the tuned scan's configurations on a sample and keeps the best. per_sm scores by SM-seconds per
// byte (time x SMs the launch occupies): in a batch many jobs share the GPU, so a configuration whose
// items fill fewer SMs on a small sample must not win by wall time alone. Otherwise by wall time.
ffbf_status autotune_impl(ffbf_ctx* c, const uint8_t* d_text, size_t sample_len, bool per_sm, int* threads,
                          int* mode) {
    TRY(enter(c));
    if (!d_text || ((uintptr_t)d_text & 15)) return fail(c, FFBF_EINVAL, "device text must be 16-byte aligned");
    if (!use_fast(c, sample_len)) return fail(c, FFBF_EINVAL, "the tuned scan does not cover this geometry or size");
    // keep the feed-forward filter: the trial scans set bits in it
    uint32_t* saved = nullptr;
    TRY(dalloc_t(c, &saved, c->filter_bytes / 4));
    CUDA_TRY(c, cudaMemcpyAsync(saved, c->d_ff, c->filter_bytes, cudaMemcpyDeviceToDevice, c->st));
    // shared-memory mode at three CTA sizes with candidates queued per byte (512 also with per-stage
    // barriers) and at two with candidates deferred to the end of each block, dense mode at three (its probe
    // order follows the filter's fills; 192 runs two CTAs per SM, and probe order 2 runs 192 as 384)
    const ffbf::FastConfig cands[] = {{512, 0, 0, 0}, {512, 3, 0, 0}, {384, 0, 0, 0}, {256, 0, 0, 0},
                                      {256, 2, 0, 0}, {192, 2, 0, 0}, {384, 1, 0, 0}, {192, 1, 0, 0},
                                      {256, 1, 0, 0}};
    ffbf::FastConfig best = c->cfg;
    double best_score = 1e300;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int saved_force = c->force_mode;
    c->force_mode = -1;
    ffbf_status s = FFBF_OK;
    for (const auto& cand : cands) {
        c->cfg = cand;
        c->cfg_tuned = true;
        if ((s = setup_scan_state(c, d_text, sample_len)) != FFBF_OK) break;
        float ms = 1e30f;
        for (int rep = 0; rep < 3 && s == FFBF_OK; rep++) {
            cudaEventRecord(e0, c->st);
            s = launch_scan(c);
            cudaEventRecord(e1, c->st);
            if (cudaEventSynchronize(e1) != cudaSuccess) s = fail(c, FFBF_ECUDA, "autotune timing failed");
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0) ms = std::min(ms, t);  // the first run also builds the stage-1 table
        }
        if (s != FFBF_OK) break;
        double score = ms;
        if (per_sm) {
            const int t = ffbf::config_threads(cand);
            const uint64_t bytes = sample_len / ffbf::kScanTile * ffbf::kScanTile;
            const uint64_t streams = bytes / ((uint64_t)ffbf::fast_rows(sample_len, cand, c->num_sms, false) * 128);
            const uint64_t items = (streams + t - 1) / t;
            score = ms * (double)std::min<uint64_t>(items, (uint64_t)c->num_sms);
        }
        if (score < best_score) {
            best_score = score;
            best = cand;
        }
    }
    c->force_mode = saved_force;
    c->cfg = best;
    c->cfg_tuned = true;
    reset_scan(c);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s == FFBF_OK) {
        CUDA_TRY(c, cudaMemcpyAsync(c->d_ff, saved, c->filter_bytes, cudaMemcpyDeviceToDevice, c->st));
        s = sync(c);
    }
    dfree(c, saved);
    if (s == FFBF_OK) s = prepare_fast(c);
    if (threads) *threads = ffbf::config_threads(best);
    if (mode) *mode = best.mode;
    return s;
}

}  // namespace

extern "C" {

ffbf_status ffbf_autotune(ffbf_ctx* c, const uint8_t* d_text, size_t sample_len, int* threads, int* mode) {
    return autotune_impl(c, d_text, sample_len, false, threads, mode);
}

}  // extern "C"
