// ffbf_ctx.cuh -- the context behind the C ABI's ffbf_ctx handle and the host helpers that the context,
// batch and server sources share. Internal to the library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/ffbf.h"
#include "ffbf_kernels.cuh"
#include "ffbf_scan_fast.cuh"

// A named NVTX range over a C-ABI call, for profilers (`ncu --nvtx`): the phases of the path show by name.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct ffbf_ctx {
    ffbf_params prm{};
    ffbf::Geom g{};
    int device = 0;
    int num_sms = 0;
    uint64_t device_mem = 0;  // the device's total memory
    cudaStream_t st = nullptr;
    uint64_t budget = 0, used = 0;
    std::map<void*, size_t> allocs;
    std::string err;

    uint32_t* d_main = nullptr;
    uint32_t* d_ff = nullptr;
    uint64_t filter_bytes = 0;
    uint32_t* d_counters = nullptr;
    uint32_t* h_counters = nullptr;  // pinned

    // patterns
    bool have_patterns = false;
    std::vector<uint8_t> h_pat;
    uint8_t* d_pat = nullptr;
    uint64_t npat = 0;
    uint64_t* d_pstart = nullptr;
    uint64_t* d_pend = nullptr;
    uint64_t* d_phash = nullptr;

    // scan
    uint8_t* d_text_own = nullptr;
    size_t text_cap = 0;
    const uint8_t* d_text = nullptr;
    uint64_t text_len = 0;
    bool scan_pending = false, have_scan = false;
    ffbf::HitRec* d_hits = nullptr;
    ffbf::HitLine* d_hitlines = nullptr;
    uint32_t hits_cap = 0;
    uint32_t nhits = 0;
    long long* d_tiles = nullptr;  // 4 arrays of tiles_cap (first, last, prev, next), then block aggregates
    uint64_t tiles_cap = 0;
    int scan_path = 0;             // 0 = generic, 1 = fast
    uint32_t* d_stage1 = nullptr;  // stage-1 table of the tuned scan (cache copy or its fold)
    bool stage1_dirty = true;
    int stage1_threads = 0;        // CTA size the table was sized for
    bool stage1_dense = false;     // sized for the dense kernel's room (its prefilter, probe order 2)
    uint32_t stage1_words = 0;
    unsigned long long* d_popc = nullptr;
    double stage1_fill = 0;
    ffbf::FastConfig cfg{512, 0, 0, 0};  // tuned-scan configuration (mode from the stage-1 fill, or the autotuner)
    bool cfg_tuned = false;
    int threads_env = 0;           // FFBF_SCAN_THREADS=256|384|512 in the environment
    int force_mode = -1;           // FFBF_SCAN_MODE=0|1 in the environment
    int force_order = -1;          // FFBF_SCAN_ORDER=0|1|2 in the environment (dense-mode probe order)
    int probe_order = 0;           // dense-mode probe order chosen from the region fills (0, 1, 2)
    bool force_generic = false;    // FFBF_FORCE_GENERIC_SCAN=1 in the environment
    // A context whose filters (main, feed-forward, stage-1 table) belong to another context: a served
    // request's scan state attached to a resident pattern set. It never frees or rebuilds them.
    bool borrowed = false;
    // host-text scans with the copy overlapped: a copy stream, one event per chunk, per-chunk descriptors
    cudaStream_t st_copy = nullptr;
    std::vector<cudaEvent_t> pipe_events;
    ffbf::FastJob* h_jobs = nullptr;  // pinned
    ffbf::FastJob* d_jobs = nullptr;
    uint32_t jobs_cap = 0;
    ffbf::FastJob* h_job = nullptr;  // pinned staging of a plain scan's job descriptor
    uint32_t* d_gate = nullptr;      // a publication word that stays zero (ffbf_debug_scan_unpublished)
    // a host text scanned in line-aligned segments (larger than the device holds): the text, the segments
    // and every hit record (absolute offsets, in segment order), which ffbf_verify uses segment by segment
    struct Segment {
        uint64_t pos, len, hr_begin, hr_end;
    };
    bool segmented = false, keep_records = false;
    const uint8_t* seg_text = nullptr;
    uint64_t seg_base = 0;
    std::vector<Segment> segs;
    std::vector<ffbf::HitRec> seg_hr;
    ffbf::FastJob* d_job = nullptr;
    std::vector<uint64_t> r_hits, r_ls, r_le;

    // prune
    bool have_prune = false;
    uint64_t* d_ids = nullptr;
    uint64_t nids = 0;
    std::vector<uint64_t> r_ids;

    // verify
    uint64_t* d_keys = nullptr;
    uint32_t* d_vals = nullptr;
    uint64_t table_cap = 0;
    uint64_t* d_moff = nullptr;
    uint32_t* d_mpid = nullptr;
    uint32_t match_cap = 0;
    std::vector<uint64_t> r_moff, r_mpid;

    // scratch for ordered compaction / codec
    uint64_t* d_tmp = nullptr;
    size_t tmp_words = 0;
    // scratch of the result ordering (sorts and selections), and the prune's per-pattern flags
    uint8_t* d_order = nullptr;
    size_t order_bytes = 0;
    uint8_t* d_pflags = nullptr;
    uint64_t pflags_cap = 0, ids_cap = 0;
    bool host_order = false;  // FFBF_HOST_ORDER: order results on the host (a check of the device ordering)
    uint8_t* d_small = nullptr;  // test_line input
    size_t small_cap = 0;
};


#define CUDA_TRY(c, expr)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (expr);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            cudaGetLastError();                                                                    \
            return fail((c), FFBF_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                 \
        }                                                                                          \
    } while (0)

#define TRY(expr)                       \
    do {                                \
        ffbf_status s_ = (expr);        \
        if (s_ != FFBF_OK) return s_;   \
    } while (0)

namespace ffbf_host {

using ffbf::Geom;
using ffbf::HitLine;
using ffbf::HitRec;

// Records a formatted message as the context's last error and returns s.
ffbf_status fail(ffbf_ctx* c, ffbf_status s, const char* fmt, ...);
// Device allocation charged to the context's HBM budget; dfree releases one.
ffbf_status dalloc(ffbf_ctx* c, void** p, size_t bytes);
template <class T>
ffbf_status dalloc_t(ffbf_ctx* c, T** p, size_t count) {
    void* v = nullptr;
    ffbf_status s = dalloc(c, &v, count * sizeof(T));
    *p = static_cast<T*>(v);
    return s;
}
template <class T>
void dfree(ffbf_ctx* c, T*& p) {
    if (!p) return;
    auto it = c->allocs.find((void*)p);
    if (it != c->allocs.end()) {
        c->used -= it->second;
        c->allocs.erase(it);
    }
    cudaFree((void*)p);
    p = nullptr;
}
ffbf_status enter(ffbf_ctx* c);  // clears the last error and makes the context's device current
ffbf_status sync(ffbf_ctx* c);   // waits for the context's stream
void reset_scan(ffbf_ctx* c);    // forgets the last scan's results
// Hit windows in text order and their lines, each line once (the hits come in any order).
void order_hits(const HitRec* hr, const HitLine* hl, uint32_t nh, std::vector<uint64_t>& hits,
                std::vector<uint64_t>& ls, std::vector<uint64_t>& le);
// Stage-1 table and probe mode of the tuned scan for the context's filter (no-op for borrowed filters).
ffbf_status prepare_fast(ffbf_ctx* c);
ffbf::ScanArgs make_scan_args(ffbf_ctx* c);
bool use_fast(const ffbf_ctx* c, uint64_t n);
ffbf_status launch_scan(ffbf_ctx* c);  // counters reset + scan of c->d_text on the context's stream
// Sizes the scan buffers for a device text of len bytes and resets the results, without launching.
ffbf_status setup_scan_state(ffbf_ctx* c, const uint8_t* d_text, size_t len);

// A context with no filters of its own (its own stream, counters and scan buffers), for attach_filters.
ffbf_status create_scan_slot(int device, ffbf_ctx** out);
// Points a slot at another context's filters, stage-1 table and scan configuration (all borrowed).
void attach_filters(ffbf_ctx* slot, const ffbf_ctx* owner);

// A scan of many (context, device text) jobs in a few launches: the tuned kernel's descriptors grouped by
// (LEN, configuration), one launch per group with its jobs largest first, and the generic kernel over every
// job's tiles that the tuned kernel does not cover (ragged ends, short texts, other geometries).
struct PlanLaunch {
    uint32_t len;
    ffbf::FastConfig cfg;
    size_t off;  // first descriptor of the group
    uint32_t n_jobs, n_items, max_s1;
};
struct PlanJob {
    ffbf_ctx* c;
    const uint8_t* text;
    size_t len;
};
struct ScanPlan {
    std::vector<ffbf::FastJob> fast;
    std::vector<PlanLaunch> launches;
    std::vector<ffbf::ScanArgs> args;  // per job, for the generic kernel
    std::vector<uint2> tail;           // (job, tile) items of the generic kernel
};
// Sets up every job's scan state (its buffers, its filter's stage-1 table) and fills the plan. On failure
// *bad is the job whose context holds the error message.
ffbf_status build_plan(const std::vector<PlanJob>& jobs, int num_sms, ScanPlan& plan, size_t* bad);
// Device copies of a plan's tables, in buffers the caller owns.
struct PlanDevice {
    ffbf::FastJob* fast;
    ffbf::ScanArgs* args;
    uint2* tail;
    uint32_t** counters;  // every job's counters, then one group of 4 control words per tuned launch
    uint32_t n_counters;
    uint32_t* ctl;        // 4 words per tuned launch: error flags, work-queue counter
};
// Enqueues a plan on st: zero every job's counters and control words, one tuned launch per group, one
// generic launch over all tail tiles. With `branches` (launches + 1 streams) and `events` (launches + 2),
// the launches run as parallel branches that fork from and join back to st.
cudaError_t launch_plan(const ScanPlan& p, const PlanDevice& d, int num_sms, cudaStream_t st,
                        const cudaStream_t* branches = nullptr, const cudaEvent_t* events = nullptr);

}  // namespace ffbf_host
