// ffbf_capi.cu -- host side of the C ABI declared in include/ffbf.h.
//
// Owns the per-context device state (the two bit arrays, the pattern file image and its line table, the
// scan/prune/verify buffers) and sequences the kernels on the context's stream. Host work is limited to
// argument checks, sorting the (few) hit and match records, and formatting the reference's output files.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/ffbf.h"
#include "ffbf_kernels.cuh"
#include "ffbf_scan_fast.cuh"

#include "ffbf_ctx.cuh"
#include "ffbf_order.cuh"

using ffbf::Geom;
using ffbf::HitLine;
using ffbf::HitRec;

namespace ffbf_host {

ffbf_status fail(ffbf_ctx* c, ffbf_status s, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return s;
}


ffbf_status dalloc(ffbf_ctx* c, void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (c->budget && c->used + bytes > c->budget)
        return fail(c, FFBF_ENOMEM_DEVICE, "device allocation of %zu bytes exceeds the HBM budget (%llu of %llu used)",
                    bytes, (unsigned long long)c->used, (unsigned long long)c->budget);
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(c, FFBF_ENOMEM_DEVICE, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    c->used += bytes;
    c->allocs[*p] = bytes;
    return FFBF_OK;
}

ffbf_status ensure_tmp(ffbf_ctx* c, size_t words) {
    if (c->tmp_words >= words) return FFBF_OK;
    dfree(c, c->d_tmp);
    c->tmp_words = 0;
    TRY(dalloc_t(c, &c->d_tmp, words));
    c->tmp_words = words;
    return FFBF_OK;
}

// Grows the result-ordering scratch to at least `bytes`.
ffbf_status ensure_order(ffbf_ctx* c, size_t bytes) {
    if (c->order_bytes >= bytes) return FFBF_OK;
    dfree(c, c->d_order);
    c->order_bytes = 0;
    TRY(dalloc_t(c, &c->d_order, bytes));
    c->order_bytes = bytes;
    return FFBF_OK;
}

ffbf_status enter(ffbf_ctx* c) {
    if (!c) return FFBF_EINVAL;
    c->err.clear();
    CUDA_TRY(c, cudaSetDevice(c->device));
    return FFBF_OK;
}

ffbf_status sync(ffbf_ctx* c) {
    CUDA_TRY(c, cudaStreamSynchronize(c->st));
    return FFBF_OK;
}

bool is_pow2(uint64_t x) { return x && !(x & (x - 1)); }

ffbf_status check_params(ffbf_ctx* c, const ffbf_params* p) {
    if (!p) return fail(c, FFBF_EINVAL, "params is NULL");
    if (p->len < 1 || p->len > 63) return fail(c, FFBF_EINVAL, "len must be in 1..63 (got %u)", p->len);
    if (p->k < 1 || p->k > 11) return fail(c, FFBF_EINVAL, "k must be in 1..11 (got %u)", p->k);
    if (p->s > p->k) return fail(c, FFBF_EINVAL, "s must be <= k (got s=%u k=%u)", p->s, p->k);
    if (p->reserved) return fail(c, FFBF_EINVAL, "reserved must be 0");
    if (!is_pow2(p->cache_bits) || !is_pow2(p->ext_bits))
        return fail(c, FFBF_EINVAL, "cache_bits and ext_bits must be powers of two");
    if (p->cache_bits < 32 || p->ext_bits < 32)
        return fail(c, FFBF_EINVAL, "cache_bits and ext_bits must be at least 32");
    if (p->cache_bits + p->ext_bits > (1ull << 31))
        return fail(c, FFBF_EINVAL, "cache_bits + ext_bits must be <= 2^31");
    return FFBF_OK;
}

// The reference prints a line as C strings (cut at the first NUL) and its carry buffer holds only the
// line's part in the previous read() chunk; see ffbf_format_lines in include/ffbf.h.
void put_cstr(std::vector<uint8_t>& out, const uint8_t* s, size_t n) {
    const void* z = memchr(s, 0, n);
    size_t m = z ? (size_t)((const uint8_t*)z - s) : n;
    out.insert(out.end(), s, s + m);
}

void format_line(std::vector<uint8_t>& out, const uint8_t* buf, uint64_t n, uint64_t s, uint64_t e, uint64_t chunk) {
    if (e < n) {
        // line ends with the '\n' at e, read in chunk ce
        uint64_t ce = e / chunk, cs = ce * chunk;
        if (s < cs) {
            uint64_t ps = std::max(s, cs - chunk);
            put_cstr(out, buf + ps, cs - ps);  // carry: the part in chunk ce-1
            put_cstr(out, buf + cs, e - cs);
        } else {
            put_cstr(out, buf + s, e - s);
        }
    } else {
        // final line without '\n': only the carry of the last chunk is printed (ffbf.cpp:385-388)
        uint64_t cl = (n - 1) / chunk, cs = cl * chunk;
        uint64_t ps = std::max(s, cs);
        put_cstr(out, buf + ps, n - ps);
    }
    out.push_back('\n');
}

ffbf_status to_host_buffer(ffbf_ctx* c, const std::vector<uint8_t>& v, uint8_t** out, size_t* out_len) {
    *out = (uint8_t*)malloc(v.size() ? v.size() : 1);
    if (!*out) return fail(c, FFBF_ENOMEM_HOST, "malloc(%zu) failed", v.size());
    if (!v.empty()) memcpy(*out, v.data(), v.size());
    *out_len = v.size();
    return FFBF_OK;
}

void order_hits(const HitRec* hr, const HitLine* hl, uint32_t nh, std::vector<uint64_t>& hits,
                std::vector<uint64_t>& ls, std::vector<uint64_t>& le) {
    std::vector<uint32_t> order(nh);
    for (uint32_t i = 0; i < nh; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return hr[a].off < hr[b].off; });
    hits.resize(nh);
    ls.clear();
    le.clear();
    for (uint32_t i = 0; i < nh; i++) {
        const uint32_t j = order[i];
        hits[i] = hr[j].off;
        if (ls.empty() || ls.back() != hl[j].start) {
            ls.push_back(hl[j].start);
            le.push_back(hl[j].end);
        }
    }
}

void reset_scan(ffbf_ctx* c) {
    c->have_scan = false;
    c->scan_pending = false;
    c->have_prune = false;
    c->r_hits.clear();
    c->r_ls.clear();
    c->r_le.clear();
    c->r_moff.clear();
    c->r_mpid.clear();
}

const uint64_t kInitialHitsCap = 1u << 16;

// Builds the stage-1 table for a CTA size and layout (the sparse mode's, or the dense mode's prefilter, which
// has the room the dense kernel leaves) unless the table on the device already is that one.
ffbf_status ensure_stage1(ffbf_ctx* c, int threads, bool dense, bool force) {
    if (!force && c->d_stage1 && c->stage1_threads == threads && c->stage1_dense == dense) return FFBF_OK;
    const uint32_t nw = ffbf::stage1_words_for(c->g, threads, dense);
    if (c->d_stage1 && c->stage1_words != nw) dfree(c, c->d_stage1);
    if (!c->d_stage1) TRY(dalloc_t(c, &c->d_stage1, nw));
    c->stage1_words = nw;
    c->stage1_threads = threads;
    c->stage1_dense = dense;
    CUDA_TRY(c, ffbf::build_stage1(c->d_main, c->g, threads, dense, c->d_stage1, c->st));
    return FFBF_OK;
}

// Makes the tuned scan ready for this context's filter: the stage-1 table the configured kernel reads and,
// unless the autotuner or the environment fixed them, the probe mode (from the sparse table's fill: the
// shared-memory stage only pays while it rejects most windows) and the dense mode's probe order (from the
// fills of the filter's regions).
ffbf_status prepare_fast(ffbf_ctx* c) {
    if (!c->d_popc) TRY(dalloc_t(c, &c->d_popc, 3));
    if (!c->h_job) {
        if (cudaMallocHost(&c->h_job, sizeof(ffbf::FastJob)) != cudaSuccess) {
            cudaGetLastError();
            c->h_job = nullptr;
            return fail(c, FFBF_ENOMEM_HOST, "pinned job descriptor");
        }
    }
    if (!c->d_job) TRY(dalloc_t(c, &c->d_job, 1));
    if (c->borrowed) return FFBF_OK;  // the filter's owner built the table and chose the configuration
    if (c->stage1_dirty || !c->d_stage1) {
        // measured on the sparse table of the configured CTA size (512 while the mode is open)
        const int tm = c->cfg.mode != 1 ? ffbf::config_threads(c->cfg) : 512;
        TRY(ensure_stage1(c, tm, false, true));
        CUDA_TRY(c, ffbf::popcount_words(c->d_stage1, c->stage1_words, c->d_popc, c->st));
        const uint32_t cw = c->g.cache_bits / 32, ew = (uint32_t)(((uint64_t)c->g.ext_mask + 1) / 32);
        CUDA_TRY(c, ffbf::popcount_words(c->d_main, cw, c->d_popc + 1, c->st));
        CUDA_TRY(c, ffbf::popcount_words(c->d_main + cw, ew, c->d_popc + 2, c->st));
        unsigned long long ones[3] = {0, 0, 0};
        CUDA_TRY(c, cudaMemcpyAsync(ones, c->d_popc, sizeof ones, cudaMemcpyDeviceToHost, c->st));
        TRY(sync(c));
        c->stage1_fill = (double)ones[0] / (32.0 * c->stage1_words);
        c->probe_order = ffbf::dense_probe_order(c->g, (double)ones[1] / (32.0 * cw), (double)ones[2] / (32.0 * ew));
        if (!c->cfg_tuned) {
            // the shared-memory stage passes about fill^2 of the windows (fill with S = 1); below 1 % the
            // warps rarely queue candidates and run apart through per-stage barriers (mode 3)
            const double pass = c->g.s > 1 ? c->stage1_fill * c->stage1_fill : c->stage1_fill;
            c->cfg.mode = c->force_mode >= 0 ? c->force_mode : c->stage1_fill > 0.3 ? 1 : pass < 0.01 ? 3 : 0;
            // default CTA sizes (measured best on the 10k- and 1M-pattern workloads): 512 threads for the
            // shared-memory stage, 2 x 192 per SM for dense filters
            // (dense: two 192-thread CTAs per SM; probe order 2 needs the 384-thread CTA's room for its table)
            c->cfg.threads = c->threads_env ? c->threads_env : c->cfg.mode == 1 ? 192 : c->cfg.mode == 2 ? 256 : 512;
        }
        c->stage1_dirty = false;
    }
    if (c->force_mode >= 0) c->cfg.mode = c->force_mode;
    // the dense mode pipelines two probes of distinct index functions: with K = 1 only the sparse mode applies
    if (c->g.k < 2 && c->cfg.mode == 1) c->cfg.mode = 0;
    // the dense mode's probe order is the filter's, unless the environment fixes it
    c->cfg.order = c->force_order >= 0 ? c->force_order : c->probe_order;
    if (c->g.k < 4 && c->cfg.order == 1) c->cfg.order = 0;  // order 1 probes f2 and f3 first
    // the table the configured kernel reads (a dense kernel without prefilter reads none)
    if (c->cfg.mode != 1) TRY(ensure_stage1(c, ffbf::config_threads(c->cfg), false, false));
    else if (c->cfg.order == 2) TRY(ensure_stage1(c, ffbf::config_threads(c->cfg), true, false));
    return FFBF_OK;
}


ffbf::ScanArgs make_scan_args(ffbf_ctx* c) {
    ffbf::ScanArgs a{};
    a.text = c->d_text;
    a.n = c->text_len;
    a.g = c->g;
    a.main_words = c->d_main;
    a.ff_words = c->d_ff;
    a.hits = c->d_hits;
    a.hits_cap = c->hits_cap;
    a.counters = c->d_counters;
    a.tile_first_nl = c->d_tiles;
    a.tile_last_nl = c->d_tiles + c->tiles_cap;
    a.ntiles = (c->text_len + ffbf::kScanTile - 1) / ffbf::kScanTile;
    a.tile_begin = 0;
    a.cache_in_smem = c->g.cache_bits <= ffbf::kSmemCacheMaxBits;
    return a;
}

bool use_fast(const ffbf_ctx* c, uint64_t n) { return ffbf::fast_scan_supported(c->g, n) && !c->force_generic; }

ffbf_status launch_scan(ffbf_ctx* c) {
    const uint64_t n = c->text_len;
    CUDA_TRY(c, cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * sizeof(uint32_t), c->st));
    if (n == 0) return FFBF_OK;
    ffbf::ScanArgs a = make_scan_args(c);
    if (use_fast(c, n)) {
        c->scan_path = 1;
        TRY(prepare_fast(c));
        CUDA_TRY(c, ffbf::scan_fast(a, c->d_stage1, c->cfg, c->num_sms, c->h_job, c->d_job, c->st));
    } else {
        c->scan_path = 0;
        int grid = ffbf::scan_generic_grid(c->g, a.cache_in_smem, a.ntiles);
        if (grid <= 0) return fail(c, FFBF_ECUDA, "scan kernel cannot be launched (occupancy query failed)");
        CUDA_TRY(c, ffbf::scan_generic(a, grid, c->st));
    }
    return FFBF_OK;
}

// Scan state for a text already on the device, without launching: buffers sized, results reset.
ffbf_status setup_scan_state(ffbf_ctx* c, const uint8_t* d_text, size_t len) {
    if (!d_text && len) return fail(c, FFBF_EINVAL, "text pointer is NULL");
    if (((uintptr_t)d_text & 15) != 0) return fail(c, FFBF_EINVAL, "device text must be 16-byte aligned");
    reset_scan(c);
    if (!c->keep_records) {  // a scan of one device text ends any segmented scan's state
        c->segmented = false;
        c->segs.clear();
        c->seg_hr.clear();
    }
    const uint64_t ntiles = (len + ffbf::kScanTile - 1) / ffbf::kScanTile;
    if (c->tiles_cap < ntiles) {
        dfree(c, c->d_tiles);
        c->tiles_cap = 0;
        // first, last, prev, next per tile, then the two-pass scan's block aggregates
        TRY(dalloc_t(c, &c->d_tiles, 4 * ntiles + 2 * ffbf::tile_agg_words(ntiles)));
        c->tiles_cap = ntiles;
    }
    if (!c->d_hits) {
        TRY(dalloc_t(c, &c->d_hits, kInitialHitsCap));
        TRY(dalloc_t(c, &c->d_hitlines, kInitialHitsCap));
        c->hits_cap = (uint32_t)kInitialHitsCap;
    }
    c->d_text = d_text;
    c->text_len = len;
    return FFBF_OK;
}

}  // namespace ffbf_host

using namespace ffbf_host;

extern "C" {

const char* ffbf_status_string(ffbf_status s) {
    switch (s) {
        case FFBF_OK: return "ok";
        case FFBF_EINVAL: return "invalid argument";
        case FFBF_ENOMEM_DEVICE: return "out of device memory";
        case FFBF_EIO: return "i/o error";
        case FFBF_ETIMEOUT: return "device wait timed out";
        case FFBF_ECUDA: return "CUDA error";
        case FFBF_ESTATE: return "call out of order";
        case FFBF_ENOMEM_HOST: return "out of host memory";
    }
    return "unknown status";
}

ffbf_status ffbf_params_default(ffbf_params* p) {
    if (!p) return FFBF_EINVAL;
    p->len = 19;
    p->k = 5;
    p->s = 2;
    p->reserved = 0;
    p->cache_bits = 0x1000000ull;
    p->ext_bits = 0x10000000ull;
    return FFBF_OK;
}

ffbf_status ffbf_create(const ffbf_params* p, int device, ffbf_ctx** out) {
    if (!out) return FFBF_EINVAL;
    *out = nullptr;
    ffbf_ctx* c = new (std::nothrow) ffbf_ctx();
    if (!c) return FFBF_ENOMEM_HOST;
    ffbf_status s = check_params(c, p);
    if (s != FFBF_OK) {
        delete c;
        return s;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        delete c;
        return FFBF_ECUDA;
    }
    c->prm = *p;
    c->device = device;
    c->g.len = p->len;
    c->g.k = p->k;
    c->g.s = p->s;
    c->g.cache_bits = (uint32_t)p->cache_bits;
    c->g.cache_mask = (uint32_t)(p->cache_bits - 1);
    c->g.ext_mask = (uint32_t)(p->ext_bits - 1);
    c->g.nbits = (uint32_t)(p->cache_bits + p->ext_bits);
    c->filter_bytes = (p->cache_bits + p->ext_bits) / 8;
    auto bail = [&](ffbf_status st) {
        ffbf_destroy(c);
        return st;
    };
    if ((e = cudaSetDevice(device)) != cudaSuccess || (e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
        cudaGetLastError();
        return bail(FFBF_ECUDA);
    }
    {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            return bail(FFBF_ECUDA);
        }
        c->device_mem = tot;
    }
    if (dalloc_t(c, &c->d_main, c->filter_bytes / 4) || dalloc_t(c, &c->d_ff, c->filter_bytes / 4) ||
        dalloc_t(c, &c->d_counters, ffbf::CNT_WORDS))
        return bail(FFBF_ENOMEM_DEVICE);
    if (cudaMallocHost(&c->h_counters, ffbf::CNT_WORDS * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        c->h_counters = nullptr;
        return bail(FFBF_ENOMEM_HOST);
    }
    if (cudaMemsetAsync(c->d_main, 0, c->filter_bytes, c->st) != cudaSuccess ||
        cudaMemsetAsync(c->d_ff, 0, c->filter_bytes, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
        cudaGetLastError();
        return bail(FFBF_ECUDA);
    }
    const char* th = getenv("FFBF_SCAN_THREADS");
    if (th && (atoi(th) == 192 || atoi(th) == 256 || atoi(th) == 384 || atoi(th) == 512))
        c->cfg.threads = c->threads_env = atoi(th);
    const char* fm = getenv("FFBF_SCAN_MODE");
    if (fm && fm[0] >= '0' && fm[0] <= '3') c->force_mode = fm[0] - '0';
    const char* fo = getenv("FFBF_SCAN_ORDER");
    if (fo && fo[0] >= '0' && fo[0] <= '2') c->force_order = fo[0] - '0';
    const char* fg = getenv("FFBF_FORCE_GENERIC_SCAN");
    c->force_generic = fg && fg[0] == '1';
    const char* ho = getenv("FFBF_HOST_ORDER");
    c->host_order = ho && ho[0] == '1';
    *out = c;
    return FFBF_OK;
}

}  // extern "C"

namespace ffbf_host {

ffbf_status create_scan_slot(int device, ffbf_ctx** out) {
    *out = nullptr;
    ffbf_ctx* c = new (std::nothrow) ffbf_ctx();
    if (!c) return FFBF_ENOMEM_HOST;
    c->device = device;
    c->borrowed = true;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        ffbf_destroy(c);
        return FFBF_ECUDA;
    }
    if (dalloc_t(c, &c->d_counters, ffbf::CNT_WORDS) != FFBF_OK) {
        ffbf_destroy(c);
        return FFBF_ENOMEM_DEVICE;
    }
    if (cudaMallocHost(&c->h_counters, ffbf::CNT_WORDS * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        c->h_counters = nullptr;
        ffbf_destroy(c);
        return FFBF_ENOMEM_HOST;
    }
    *out = c;
    return FFBF_OK;
}

void attach_filters(ffbf_ctx* slot, const ffbf_ctx* owner) {
    slot->prm = owner->prm;
    slot->g = owner->g;
    slot->filter_bytes = owner->filter_bytes;
    slot->d_main = owner->d_main;
    slot->d_ff = owner->d_ff;
    slot->d_stage1 = owner->d_stage1;
    slot->stage1_threads = owner->stage1_threads;
    slot->stage1_dense = owner->stage1_dense;
    slot->stage1_words = owner->stage1_words;
    slot->stage1_fill = owner->stage1_fill;
    slot->stage1_dirty = false;
    slot->cfg = owner->cfg;
    slot->cfg_tuned = true;
    slot->force_mode = owner->force_mode;
    slot->force_generic = owner->force_generic;
}

}  // namespace ffbf_host

extern "C" {

void ffbf_destroy(ffbf_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    for (auto& kv : c->allocs) cudaFree(kv.first);
    c->allocs.clear();
    if (c->h_counters) cudaFreeHost(c->h_counters);
    if (c->h_job) cudaFreeHost(c->h_job);
    if (c->h_jobs) cudaFreeHost(c->h_jobs);
    for (auto ev : c->pipe_events) cudaEventDestroy(ev);
    if (c->st_copy) {
        cudaStreamSynchronize(c->st_copy);
        cudaStreamDestroy(c->st_copy);
    }
    if (c->st) cudaStreamDestroy(c->st);
    cudaGetLastError();
    delete c;
}

const char* ffbf_last_error(const ffbf_ctx* c) { return c ? c->err.c_str() : "null context"; }

uint64_t ffbf_filter_bytes(const ffbf_ctx* c) { return c ? c->filter_bytes : 0; }

void ffbf_free(void* p) { free(p); }

void* ffbf_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void ffbf_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

void* ffbf_stream(ffbf_ctx* c) { return c ? (void*)c->st : nullptr; }

uint64_t ffbf_kernel_launches(void) { return ffbf::launches_total(); }

ffbf_status ffbf_set_hbm_budget(ffbf_ctx* c, uint64_t bytes) {
    if (!c) return FFBF_EINVAL;
    c->budget = bytes;
    return FFBF_OK;
}

ffbf_status ffbf_set_patterns(ffbf_ctx* c, const uint8_t* file, size_t len) {
    TRY(enter(c));
    if (!file && len) return fail(c, FFBF_EINVAL, "pattern buffer is NULL");
    c->have_patterns = false;
    c->have_prune = false;
    dfree(c, c->d_pat);
    dfree(c, c->d_pstart);
    dfree(c, c->d_pend);
    dfree(c, c->d_phash);
    c->npat = 0;
    try {
        c->h_pat.assign(file, file + len);
    } catch (...) {
        return fail(c, FFBF_ENOMEM_HOST, "host copy of %zu pattern bytes failed", len);
    }
    TRY(dalloc_t(c, &c->d_pat, len + 16));
    if (len) CUDA_TRY(c, cudaMemcpyAsync(c->d_pat, file, len, cudaMemcpyHostToDevice, c->st));
    const uint64_t nb = ffbf::compact_blocks(len);
    TRY(ensure_tmp(c, nb + 1));
    CUDA_TRY(c, ffbf::count_bytes(c->d_pat, len, '\n', c->d_tmp, c->st));
    uint64_t m = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&m, c->d_tmp + nb, sizeof m, cudaMemcpyDeviceToHost, c->st));
    TRY(sync(c));
    const int tail = len > 0 && file[len - 1] != '\n';
    const uint64_t npat = m + (tail ? 1 : 0);
    uint64_t* d_nl = nullptr;
    TRY(dalloc_t(c, &d_nl, m + 1));
    ffbf_status s = FFBF_OK;
    do {
        if (ffbf::emit_bytes(c->d_pat, len, '\n', d_nl, c->d_tmp, c->st) != cudaSuccess) {
            s = fail(c, FFBF_ECUDA, "newline compaction failed");
            break;
        }
        if ((s = dalloc_t(c, &c->d_pstart, npat + 1)) || (s = dalloc_t(c, &c->d_pend, npat + 1)) ||
            (s = dalloc_t(c, &c->d_phash, npat + 1)))
            break;
        if (ffbf::lines_from_newlines(d_nl, m, len, tail, c->d_pstart, c->d_pend, c->st) != cudaSuccess ||
            ffbf::hash_patterns(c->d_pat, c->d_pstart, c->d_pend, npat, c->g, c->d_phash, c->d_main, 0, c->st) !=
                cudaSuccess) {
            s = fail(c, FFBF_ECUDA, "pattern hashing failed: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        s = sync(c);
    } while (0);
    dfree(c, d_nl);
    if (s != FFBF_OK) return s;
    c->npat = npat;
    c->have_patterns = true;
    return FFBF_OK;
}

ffbf_status ffbf_build(ffbf_ctx* c) {
    NvtxRange nvtx_("ffbf_build");
    TRY(enter(c));
    if (!c->have_patterns) return fail(c, FFBF_ESTATE, "ffbf_build needs ffbf_set_patterns first");
    CUDA_TRY(c, ffbf::hash_patterns(c->d_pat, c->d_pstart, c->d_pend, c->npat, c->g, c->d_phash, c->d_main, 1, c->st));
    c->stage1_dirty = true;
    return sync(c);
}

ffbf_status ffbf_add_patterns(ffbf_ctx* c, const uint8_t* file, size_t len) {
    TRY(ffbf_set_patterns(c, file, len));
    return ffbf_build(c);
}

ffbf_status ffbf_load_filter(ffbf_ctx* c, const uint8_t* data, size_t len) {
    TRY(enter(c));
    if (!data && len) return fail(c, FFBF_EINVAL, "filter buffer is NULL");
    const uint64_t nd = len / 4;
    if (!nd) return FFBF_OK;
    uint32_t *d_d = nullptr, *d_idx = nullptr;
    TRY(dalloc_t(c, &d_d, nd));
    ffbf_status s = dalloc_t(c, &d_idx, nd);
    if (s == FFBF_OK) s = ensure_tmp(c, ffbf::decode_blocks(nd) + 1);
    if (s == FFBF_OK) {
        uint32_t err = 0;
        if (cudaMemcpyAsync(d_d, data, nd * 4, cudaMemcpyHostToDevice, c->st) != cudaSuccess ||
            cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * 4, c->st) != cudaSuccess ||
            ffbf::filter_decode(d_d, nd, c->g.nbits, d_idx, c->d_tmp, c->d_counters, c->st) != cudaSuccess ||
            cudaMemcpyAsync(&err, c->d_counters + ffbf::CNT_ERROR, 4, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
            cudaStreamSynchronize(c->st) != cudaSuccess) {
            s = fail(c, FFBF_ECUDA, "filter decode failed: %s", cudaGetErrorString(cudaGetLastError()));
        } else if (err) {
            s = fail(c, FFBF_EINVAL, "filter file holds a bit index at or beyond N = %u", c->g.nbits);
        } else if ((c->stage1_dirty = true, ffbf::filter_set_indices(d_idx, nd, c->d_main, c->st) != cudaSuccess) ||
                   cudaStreamSynchronize(c->st) != cudaSuccess) {
            s = fail(c, FFBF_ECUDA, "filter load failed: %s", cudaGetErrorString(cudaGetLastError()));
        }
    }
    dfree(c, d_d);
    dfree(c, d_idx);
    return s;
}

ffbf_status ffbf_save_filter(ffbf_ctx* c, uint8_t** data, size_t* len) {
    TRY(enter(c));
    if (!data || !len) return fail(c, FFBF_EINVAL, "NULL output pointer");
    *data = nullptr;
    *len = 0;
    const uint32_t nwords = c->g.nbits / 32;
    const uint64_t nb = ffbf::enc_blocks(nwords);
    TRY(ensure_tmp(c, nb + 1));
    CUDA_TRY(c, ffbf::filter_count(c->d_main, nwords, c->d_tmp, c->st));
    uint64_t total = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&total, c->d_tmp + nb, 8, cudaMemcpyDeviceToHost, c->st));
    TRY(sync(c));
    uint8_t* h = (uint8_t*)malloc(total * 4 + 1);
    if (!h) return fail(c, FFBF_ENOMEM_HOST, "malloc(%llu) failed", (unsigned long long)(total * 4));
    if (total) {
        uint32_t *d_idx = nullptr, *d_del = nullptr;
        ffbf_status s = dalloc_t(c, &d_idx, total);
        if (s == FFBF_OK) s = dalloc_t(c, &d_del, total);
        if (s == FFBF_OK && (ffbf::filter_encode(c->d_main, nwords, c->d_tmp, d_idx, c->st) != cudaSuccess ||
                             ffbf::filter_deltas(d_idx, total, d_del, c->st) != cudaSuccess ||
                             cudaMemcpyAsync(h, d_del, total * 4, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
                             cudaStreamSynchronize(c->st) != cudaSuccess))
            s = fail(c, FFBF_ECUDA, "filter encode failed: %s", cudaGetErrorString(cudaGetLastError()));
        dfree(c, d_idx);
        dfree(c, d_del);
        if (s != FFBF_OK) {
            free(h);
            return s;
        }
    }
    *data = h;
    *len = total * 4;
    return FFBF_OK;
}

ffbf_status ffbf_load_filter_file(ffbf_ctx* c, const char* path) {
    if (!c) return FFBF_EINVAL;
    if (!path) return fail(c, FFBF_EINVAL, "path is NULL");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(c, FFBF_EIO, "cannot open %s", path);
    std::vector<uint8_t> buf;
    uint8_t tmp[1 << 16];
    size_t r;
    while ((r = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + r);
    bool bad = ferror(f);
    fclose(f);
    if (bad) return fail(c, FFBF_EIO, "error while reading the filter file %s", path);
    return ffbf_load_filter(c, buf.data(), buf.size());
}

ffbf_status ffbf_save_filter_file(ffbf_ctx* c, const char* path) {
    if (!c) return FFBF_EINVAL;
    if (!path) return fail(c, FFBF_EINVAL, "path is NULL");
    uint8_t* data = nullptr;
    size_t len = 0;
    TRY(ffbf_save_filter(c, &data, &len));
    FILE* f = fopen(path, "wb");
    if (!f) {
        ffbf_free(data);
        return fail(c, FFBF_EIO, "cannot create %s", path);
    }
    bool ok = fwrite(data, 1, len, f) == len;
    ok = (fclose(f) == 0) && ok;
    ffbf_free(data);
    if (!ok) return fail(c, FFBF_EIO, "error while writing to the filter file %s", path);
    return FFBF_OK;
}

ffbf_status ffbf_scan_device(ffbf_ctx* c, const uint8_t* d_text, size_t len) {
    NvtxRange nvtx_("ffbf_scan_device");
    TRY(enter(c));
    TRY(setup_scan_state(c, d_text, len));
    TRY(launch_scan(c));
    c->scan_pending = true;
    return FFBF_OK;
}

ffbf_status ffbf_scan_collect(ffbf_ctx* c, ffbf_scan_result* out) {
    NvtxRange nvtx_("ffbf_scan_collect");
    TRY(enter(c));
    if (!c->scan_pending && !c->have_scan) return fail(c, FFBF_ESTATE, "no scan to collect");
    if (c->scan_pending) {
        CUDA_TRY(c, cudaMemcpyAsync(c->h_counters, c->d_counters, ffbf::CNT_WORDS * 4, cudaMemcpyDeviceToHost, c->st));
        TRY(sync(c));
        uint32_t nh = c->h_counters[ffbf::CNT_HITS];
        if (nh > c->hits_cap) {
            // Too many hits for the buffer: grow it and scan again. Setting feed-forward bits is
            // idempotent, so the second pass leaves the same filter.
            uint64_t cap = (uint64_t)nh + nh / 4 + 1024;
            if (cap > 0xffffffffull) return fail(c, FFBF_EINVAL, "more than 2^32 hit windows in one scan");
            dfree(c, c->d_hits);
            dfree(c, c->d_hitlines);
            c->hits_cap = 0;
            TRY(dalloc_t(c, &c->d_hits, cap));
            TRY(dalloc_t(c, &c->d_hitlines, cap));
            c->hits_cap = (uint32_t)cap;
            TRY(launch_scan(c));
            CUDA_TRY(c, cudaMemcpyAsync(c->h_counters, c->d_counters, ffbf::CNT_WORDS * 4, cudaMemcpyDeviceToHost, c->st));
            TRY(sync(c));
            nh = c->h_counters[ffbf::CNT_HITS];
        }
        c->nhits = nh;
        const uint64_t ntiles = (c->text_len + ffbf::kScanTile - 1) / ffbf::kScanTile;
        CUDA_TRY(c, ffbf::resolve_lines(c->d_text, c->text_len, c->g.len, c->d_hits, nh, c->d_tiles,
                                        c->d_tiles + c->tiles_cap, c->d_tiles + 2 * c->tiles_cap,
                                        c->d_tiles + 3 * c->tiles_cap, ntiles, c->d_hitlines, c->st,
                                        c->d_tiles + 4 * c->tiles_cap));
        // Text order on the device: sorted window starts, then the distinct lines of the sorted windows. When
        // the device has no room for the sort's scratch (about 60 bytes per hit window), or FFBF_HOST_ORDER is
        // set, the records are ordered on the host instead; the results are the same.
        const int kb = ffbf::key_bits_for(c->text_len);
        const size_t scratch = ffbf::order_hits_scratch(nh, kb);
        const size_t off_bytes = ((size_t)nh * 8 + 255) / 256 * 256, line_bytes = ((size_t)nh * 16 + 255) / 256 * 256;
        const bool on_device = !c->host_order && ensure_order(c, off_bytes + line_bytes + 256 + scratch) == FFBF_OK;
        if (!on_device) c->err.clear();
        std::vector<HitRec> hr;
        if (nh && (c->keep_records || !on_device)) {
            hr.resize(nh);
            CUDA_TRY(c, cudaMemcpyAsync(hr.data(), c->d_hits, nh * sizeof(HitRec), cudaMemcpyDeviceToHost, c->st));
            TRY(sync(c));
        }
        if (c->keep_records)  // a segment of a larger text: ffbf_verify needs its records again
            for (uint32_t i = 0; i < nh; i++) c->seg_hr.push_back(HitRec{hr[i].off + c->seg_base, hr[i].h});
        if (!on_device) {
            std::vector<HitLine> hl(nh);
            if (nh)
                CUDA_TRY(c, cudaMemcpyAsync(hl.data(), c->d_hitlines, nh * sizeof(HitLine), cudaMemcpyDeviceToHost,
                                            c->st));
            TRY(sync(c));
            order_hits(hr.data(), hl.data(), nh, c->r_hits, c->r_ls, c->r_le);
        } else {
            uint64_t* d_off = reinterpret_cast<uint64_t*>(c->d_order);
            HitLine* d_lu = reinterpret_cast<HitLine*>(c->d_order + off_bytes);
            uint64_t* d_nl = reinterpret_cast<uint64_t*>(c->d_order + off_bytes + line_bytes);
            CUDA_TRY(c, ffbf::order_hits(c->d_hits, c->d_hitlines, nh, kb, c->d_order + off_bytes + line_bytes + 256,
                                         scratch, d_off, d_lu, d_nl, c->st));
            uint64_t n_lines = 0;
            c->r_hits.resize(nh);
            if (nh)
                CUDA_TRY(c, cudaMemcpyAsync(c->r_hits.data(), d_off, nh * 8ull, cudaMemcpyDeviceToHost, c->st));
            CUDA_TRY(c, cudaMemcpyAsync(&n_lines, d_nl, 8, cudaMemcpyDeviceToHost, c->st));
            TRY(sync(c));
            if (n_lines > nh) return fail(c, FFBF_ECUDA, "line reduction returned %llu lines for %u hits",
                                          (unsigned long long)n_lines, nh);
            std::vector<HitLine> lines(n_lines);
            if (n_lines) {
                CUDA_TRY(c, cudaMemcpyAsync(lines.data(), d_lu, n_lines * sizeof(HitLine), cudaMemcpyDeviceToHost,
                                            c->st));
                TRY(sync(c));
            }
            c->r_ls.resize(n_lines);
            c->r_le.resize(n_lines);
            for (uint64_t i = 0; i < n_lines; i++) {
                c->r_ls[i] = lines[i].start;
                c->r_le[i] = lines[i].end;
            }
        }
        c->scan_pending = false;
        c->have_scan = true;
    }
    if (out) {
        out->text_len = c->text_len;
        out->n_hits = c->r_hits.size();
        out->hit_offsets = c->r_hits.data();
        out->n_lines = c->r_ls.size();
        out->line_start = c->r_ls.data();
        out->line_end = c->r_le.data();
    }
    return FFBF_OK;
}

}  // extern "C"

namespace {

// Host texts of kPipeMinText bytes or more are copied in chunks that the scan follows; a chunk is about an
// eighth of the text, between 8 and 128 MiB.
constexpr uint64_t kPipeMinText = 32ull << 20;
constexpr uint64_t kPipeChunkMin = 8ull << 20, kPipeChunkMax = 128ull << 20;

uint64_t pipe_chunk(uint64_t len) {
    return std::min(kPipeChunkMax, std::max(kPipeChunkMin, len / 8 >> 20 << 20));
}

// The scan of a host text whose copy to the device overlaps the scan: the text goes over in chunks of
// about pipe_chunk(len) bytes on the context's copy stream, and after each chunk the tuned kernel runs over
// the work items whose bytes (and halos) have landed. The rows per stream suit one chunk, whose launch
// then spreads over the SMs and ends soon after its copy; the copy is the bound. Every chunk's launch uses
// the whole text's tensor map and absolute positions; its descriptor only shifts the item numbering
// (item_begin = -first item).
ffbf_status scan_host_pipelined(ffbf_ctx* c, const uint8_t* text, size_t len) {
    TRY(setup_scan_state(c, c->d_text_own, len));
    CUDA_TRY(c, cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * sizeof(uint32_t), c->st));
    TRY(prepare_fast(c));
    c->scan_path = 1;
    const ffbf::ScanArgs a = make_scan_args(c);
    const int threads = ffbf::config_threads(c->cfg);
    const uint64_t chunk = pipe_chunk(len);
    const uint32_t rows = c->cfg.rows ? c->cfg.rows : ffbf::fast_rows(chunk, c->cfg, c->num_sms, false);
    ffbf::FastJob job;
    cudaError_t e;
    const uint64_t covered = ffbf::fill_fast_job(a, c->d_stage1, c->cfg, rows, &job, &e);
    if (e != cudaSuccess) return fail(c, FFBF_ECUDA, "tensor map encoding failed");
    const uint64_t item_bytes = (uint64_t)threads * rows * 128;
    const uint32_t per_chunk = (uint32_t)std::max<uint64_t>(1, chunk / item_bytes);
    const uint32_t n_chunks = (job.n_supertiles + per_chunk - 1) / per_chunk;
    if (!c->st_copy) CUDA_TRY(c, cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
    while (c->pipe_events.size() < (size_t)n_chunks + 2) {
        cudaEvent_t ev;
        CUDA_TRY(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        c->pipe_events.push_back(ev);
    }
    if (c->jobs_cap < n_chunks) {
        TRY(sync(c));  // the old staging may still feed a copy
        if (c->h_jobs) cudaFreeHost(c->h_jobs);
        c->h_jobs = nullptr;
        dfree(c, c->d_jobs);
        c->jobs_cap = 0;
        if (cudaMallocHost(&c->h_jobs, n_chunks * sizeof(ffbf::FastJob)) != cudaSuccess) {
            cudaGetLastError();
            c->h_jobs = nullptr;
            return fail(c, FFBF_ENOMEM_HOST, "pinned chunk descriptors");
        }
        TRY(dalloc_t(c, &c->d_jobs, n_chunks));
        c->jobs_cap = n_chunks;
    }
    TRY(sync(c));  // the staging array is rewritten below; earlier uploads must be done
    for (uint32_t i = 0; i < n_chunks; i++) {
        c->h_jobs[i] = job;
        c->h_jobs[i].item_begin = 0u - i * per_chunk;  // item k of chunk i is supertile i * per_chunk + k
    }
    CUDA_TRY(c, cudaMemcpyAsync(c->d_jobs, c->h_jobs, n_chunks * sizeof(ffbf::FastJob), cudaMemcpyHostToDevice,
                                c->st));
    // the copies overwrite the text buffer: start them after what the context's stream already holds
    CUDA_TRY(c, cudaEventRecord(c->pipe_events[n_chunks + 1], c->st));
    CUDA_TRY(c, cudaStreamWaitEvent(c->st_copy, c->pipe_events[n_chunks + 1], 0));
    uint64_t copied = 0;
    for (uint32_t i = 0; i < n_chunks; i++) {
        const uint32_t first = i * per_chunk;
        const uint32_t count = std::min(per_chunk, job.n_supertiles - first);
        const uint64_t end = std::min<uint64_t>(len, (uint64_t)(first + count) * item_bytes);
        if (end > copied) {
            CUDA_TRY(c, cudaMemcpyAsync(c->d_text_own + copied, text + copied, end - copied, cudaMemcpyHostToDevice,
                                        c->st_copy));
            copied = end;
        }
        CUDA_TRY(c, cudaEventRecord(c->pipe_events[i], c->st_copy));
        CUDA_TRY(c, cudaStreamWaitEvent(c->st, c->pipe_events[i], 0));
        CUDA_TRY(c, cudaMemsetAsync(c->d_counters + ffbf::CNT_QUEUE, 0, sizeof(uint32_t), c->st));
        CUDA_TRY(c, ffbf::launch_fast_jobs(c->g.len, c->cfg, c->d_jobs + i, 1, count, job.stage1_nwords,
                                           c->d_counters + ffbf::CNT_ERROR, c->num_sms, c->st));
    }
    if (copied < len) {
        CUDA_TRY(c, cudaMemcpyAsync(c->d_text_own + copied, text + copied, len - copied, cudaMemcpyHostToDevice,
                                    c->st_copy));
    }
    CUDA_TRY(c, cudaEventRecord(c->pipe_events[n_chunks], c->st_copy));
    CUDA_TRY(c, cudaStreamWaitEvent(c->st, c->pipe_events[n_chunks], 0));
    CUDA_TRY(c, ffbf::scan_tail(a, covered, c->st));
    return FFBF_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// One host text that fits the device: copied (overlapped with the scan when large) and scanned.
ffbf_status scan_one(ffbf_ctx* c, const uint8_t* text, size_t len, ffbf_scan_result* out) {
    if (c->text_cap < len + 64) {
        dfree(c, c->d_text_own);
        c->text_cap = 0;
        TRY(dalloc_t(c, &c->d_text_own, len + 64));
        c->text_cap = len + 64;
    }
    if (len >= kPipeMinText && use_fast(c, len)) {
        TRY(scan_host_pipelined(c, text, len));
        c->scan_pending = true;
        return ffbf_scan_collect(c, out);
    }
    if (len) CUDA_TRY(c, cudaMemcpyAsync(c->d_text_own, text, len, cudaMemcpyHostToDevice, c->st));
    TRY(ffbf_scan_device(c, c->d_text_own, len));
    return ffbf_scan_collect(c, out);
}

// Device bytes a scan of `len` text bytes needs beyond what the context holds: the text buffer, the tile
// summaries and, the first time, the hit buffers.
uint64_t scan_need(const ffbf_ctx* c, uint64_t len) {
    const uint64_t ntiles = (len + ffbf::kScanTile - 1) / ffbf::kScanTile;
    uint64_t need = len + 64 + 8 * (4 * ntiles + 2 * ffbf::tile_agg_words(ntiles));
    if (!c->d_hits) need += 2 * kInitialHitsCap * 16;
    return need;
}

// The largest segment a scan may put on the device: what the HBM budget (or the device's free memory, less
// 1 GiB) leaves after everything but the text buffer, three quarters of it; 0 when the whole text fits.
ffbf_status segment_size(ffbf_ctx* c, uint64_t len, uint64_t* seg) {
    *seg = 0;
    uint64_t avail;
    if (c->budget) {
        avail = c->budget > c->used ? c->budget - c->used : 0;
    } else {
        // asking the driver for free memory costs about a millisecond: only texts of a quarter of the
        // device or more can fail to fit, so smaller ones skip the query
        if (scan_need(c, len) < c->device_mem / 4) return FFBF_OK;
        size_t fr = 0, tot = 0;
        CUDA_TRY(c, cudaMemGetInfo(&fr, &tot));
        avail = fr > (1ull << 30) ? fr - (1ull << 30) : 0;
    }
    avail += c->text_cap;  // the current text buffer is given back first
    if (scan_need(c, len) <= avail) return FFBF_OK;
    *seg = avail / 4 * 3 / 65536 * 65536;
    if (*seg < (1u << 20)) return fail(c, FFBF_ENOMEM_DEVICE, "no room on the device for a 1 MiB text segment");
    return FFBF_OK;
}

}  // namespace

extern "C" {

ffbf_status ffbf_scan(ffbf_ctx* c, const uint8_t* text, size_t len, ffbf_scan_result* out) {
    NvtxRange nvtx_("ffbf_scan");
    TRY(enter(c));
    if (!text && len) return fail(c, FFBF_EINVAL, "text is NULL");
    c->segmented = false;
    c->keep_records = false;
    c->segs.clear();
    c->seg_hr.clear();
    uint64_t seg = 0;
    TRY(segment_size(c, len, &seg));
    if (seg == 0) return scan_one(c, text, len, out);
    // A text larger than the device holds: scan it in segments that end just after a '\n'. A valid window
    // never spans a '\n', so the segments' scans are independent; their results are offset and joined, and
    // the feed-forward filter accumulates over them as over successive scans.
    dfree(c, c->d_text_own);
    c->text_cap = 0;
    std::vector<uint64_t> hits, ls, le;
    c->keep_records = true;
    for (uint64_t pos = 0; pos < len;) {
        uint64_t end = std::min<uint64_t>(len, pos + seg);
        if (end < len) {
            const void* nl = memrchr(text + pos, '\n', end - pos);
            if (!nl) {
                c->keep_records = false;
                return fail(c, FFBF_EINVAL, "a line longer than the device's text segment (%llu bytes) at offset %llu",
                            (unsigned long long)seg, (unsigned long long)pos);
            }
            end = (uint64_t)((const uint8_t*)nl - text) + 1;
        }
        c->seg_base = pos;
        c->segs.push_back({pos, end - pos, (uint64_t)c->seg_hr.size(), 0});
        ffbf_scan_result r{};
        ffbf_status st = scan_one(c, text + pos, end - pos, &r);
        if (st != FFBF_OK) {
            c->keep_records = false;
            return st;
        }
        c->segs.back().hr_end = c->seg_hr.size();
        for (uint64_t i = 0; i < r.n_hits; i++) hits.push_back(r.hit_offsets[i] + pos);
        for (uint64_t i = 0; i < r.n_lines; i++) {
            ls.push_back(r.line_start[i] + pos);
            le.push_back(r.line_end[i] + pos);
        }
        pos = end;
    }
    c->keep_records = false;
    c->segmented = true;
    c->seg_text = text;
    c->r_hits.swap(hits);
    c->r_ls.swap(ls);
    c->r_le.swap(le);
    c->nhits = (uint32_t)c->r_hits.size();
    c->text_len = len;
    c->have_scan = true;
    c->scan_pending = false;
    if (out) {
        out->text_len = len;
        out->n_hits = c->r_hits.size();
        out->hit_offsets = c->r_hits.data();
        out->n_lines = c->r_ls.size();
        out->line_start = c->r_ls.data();
        out->line_end = c->r_le.data();
    }
    return FFBF_OK;
}

ffbf_status ffbf_format_lines(ffbf_ctx* c, const uint8_t* text, size_t len, size_t chunk, uint8_t** out,
                              size_t* out_len) {
    if (!c) return FFBF_EINVAL;
    if (!out || !out_len || (!text && len)) return fail(c, FFBF_EINVAL, "NULL argument");
    if (!c->have_scan) return fail(c, FFBF_ESTATE, "ffbf_format_lines needs a collected scan");
    if (len != c->text_len) return fail(c, FFBF_EINVAL, "text length differs from the scanned text");
    if (chunk == 0) return fail(c, FFBF_EINVAL, "chunk must be > 0");
    std::vector<uint8_t> v;
    for (size_t i = 0; i < c->r_ls.size(); i++) format_line(v, text, len, c->r_ls[i], c->r_le[i], chunk);
    return to_host_buffer(c, v, out, out_len);
}

ffbf_status ffbf_format_spans(const uint8_t* buf, size_t len, const uint64_t* start, const uint64_t* end, size_t n,
                              size_t chunk, uint8_t** out, size_t* out_len) {
    if (!out || !out_len || (!buf && len) || (n && (!start || !end)) || chunk == 0) return FFBF_EINVAL;
    *out = nullptr;
    *out_len = 0;
    for (size_t i = 0; i < n; i++)
        if (start[i] > end[i] || end[i] > len || (i && start[i] <= end[i - 1]))
            return FFBF_EINVAL;
    std::vector<uint8_t> v;
    try {
        for (size_t i = 0; i < n; i++) format_line(v, buf, len, start[i], end[i], chunk);
    } catch (...) {
        return FFBF_ENOMEM_HOST;
    }
    return to_host_buffer(nullptr, v, out, out_len);
}

ffbf_status ffbf_prune(ffbf_ctx* c, ffbf_prune_result* out) {
    NvtxRange nvtx_("ffbf_prune");
    TRY(enter(c));
    if (!c->have_patterns) return fail(c, FFBF_ESTATE, "ffbf_prune needs ffbf_set_patterns first");
    if (c->scan_pending) TRY(ffbf_scan_collect(c, nullptr));
    const uint64_t n = c->npat;
    const uint64_t nb = ffbf::compact_blocks(n);
    TRY(ensure_tmp(c, nb + 1));
    // the flags and id buffers are kept between calls: a cudaFree would wait for the whole device
    if (c->pflags_cap < n + 1) {
        dfree(c, c->d_pflags);
        c->pflags_cap = 0;
        TRY(dalloc_t(c, &c->d_pflags, n + 1));
        c->pflags_cap = n + 1;
    }
    uint8_t* d_flags = c->d_pflags;
    ffbf_status s = FFBF_OK;
    uint64_t cnt = 0;
    if (ffbf::prune_flags(c->d_pstart, c->d_pend, c->d_phash, n, c->g, c->d_ff, d_flags, c->st) != cudaSuccess ||
        ffbf::count_flags(d_flags, n, c->d_tmp, c->st) != cudaSuccess ||
        cudaMemcpyAsync(&cnt, c->d_tmp + nb, 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess)
        s = fail(c, FFBF_ECUDA, "prune failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (s == FFBF_OK && c->ids_cap < cnt + 1) {
        dfree(c, c->d_ids);
        c->ids_cap = 0;
        s = dalloc_t(c, &c->d_ids, cnt + 1);
        if (s == FFBF_OK) c->ids_cap = cnt + 1;
    }
    if (s == FFBF_OK) {
        c->r_ids.resize(cnt);
        if (ffbf::emit_flags(d_flags, n, c->d_ids, c->d_tmp, c->st) != cudaSuccess ||
            (cnt && cudaMemcpyAsync(c->r_ids.data(), c->d_ids, cnt * 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess) ||
            cudaStreamSynchronize(c->st) != cudaSuccess)
            s = fail(c, FFBF_ECUDA, "prune compaction failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    if (s != FFBF_OK) return s;
    c->nids = cnt;
    c->have_prune = true;
    if (out) {
        out->n_ids = cnt;
        out->ids = c->r_ids.data();
    }
    return FFBF_OK;
}

ffbf_status ffbf_format_pruned(ffbf_ctx* c, size_t chunk, uint8_t** out, size_t* out_len, uint8_t** index,
                               size_t* index_len) {
    if (!c) return FFBF_EINVAL;
    if (!out || !out_len || !index || !index_len) return fail(c, FFBF_EINVAL, "NULL argument");
    if (!c->have_prune) return fail(c, FFBF_ESTATE, "ffbf_format_pruned needs ffbf_prune first");
    if (chunk == 0) return fail(c, FFBF_EINVAL, "chunk must be > 0");
    const std::vector<uint8_t>& f = c->h_pat;
    // line spans of the pattern file, walked in step with the ascending ids
    std::vector<uint8_t> o, ix;
    uint64_t line = 0, pos = 0;
    char num[32];
    for (uint64_t id : c->r_ids) {
        while (line < id) {
            const void* nl = memchr(f.data() + pos, '\n', f.size() - pos);
            pos = nl ? (uint64_t)((const uint8_t*)nl - f.data()) + 1 : f.size();
            line++;
        }
        const void* nl = memchr(f.data() + pos, '\n', f.size() - pos);
        uint64_t e = nl ? (uint64_t)((const uint8_t*)nl - f.data()) : f.size();
        format_line(o, f.data(), f.size(), pos, e, chunk);
        int k = snprintf(num, sizeof num, "%llu\n", (unsigned long long)id);
        ix.insert(ix.end(), num, num + k);
    }
    TRY(to_host_buffer(c, o, out, out_len));
    ffbf_status s = to_host_buffer(c, ix, index, index_len);
    if (s != FFBF_OK) {
        free(*out);
        *out = nullptr;
    }
    return s;
}

}  // extern "C"

namespace {

// Verifies nh hit records already in c->d_hits against a device text, appending (offset + base, pattern)
// pairs. The match buffers grow and the pass reruns when they overflow.
ffbf_status verify_pass(ffbf_ctx* c, uint32_t nh, const uint8_t* d_text, uint64_t text_len, uint64_t tsize,
                        uint64_t base, std::vector<uint64_t>& off_out, std::vector<uint32_t>& pid_out) {
    if (c->match_cap < std::max<uint32_t>(1024, nh)) {
        dfree(c, c->d_moff);
        dfree(c, c->d_mpid);
        c->match_cap = 0;
        uint32_t cap = std::max<uint32_t>(1024, nh);
        TRY(dalloc_t(c, &c->d_moff, cap));
        TRY(dalloc_t(c, &c->d_mpid, cap));
        c->match_cap = cap;
    }
    for (int attempt = 0; attempt < 2; attempt++) {
        CUDA_TRY(c, cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * 4, c->st));
        CUDA_TRY(c, ffbf::verify_hits(c->d_hits, nh, d_text, text_len, c->d_keys, c->d_vals, tsize - 1, c->d_pat,
                                      c->d_pstart, c->d_pend, c->d_moff, c->d_mpid, c->match_cap, c->d_counters, c->st));
        CUDA_TRY(c, cudaMemcpyAsync(c->h_counters, c->d_counters, ffbf::CNT_WORDS * 4, cudaMemcpyDeviceToHost, c->st));
        TRY(sync(c));
        uint32_t nm = c->h_counters[ffbf::CNT_MATCHES];
        if (nm <= c->match_cap) break;
        uint64_t cap = (uint64_t)nm + nm / 4 + 1024;
        if (cap > 0xffffffffull) return fail(c, FFBF_EINVAL, "more than 2^32 matches");
        dfree(c, c->d_moff);
        dfree(c, c->d_mpid);
        c->match_cap = 0;
        TRY(dalloc_t(c, &c->d_moff, cap));
        TRY(dalloc_t(c, &c->d_mpid, cap));
        c->match_cap = (uint32_t)cap;
    }
    const uint32_t nm = c->h_counters[ffbf::CNT_MATCHES];
    // (offset, pattern id) order on the device, or on the host as the hits' order is (see ffbf_scan_collect)
    const int kb = ffbf::key_bits_for(text_len);
    const size_t scratch = ffbf::order_matches_scratch(nm, kb);
    const bool on_device = !c->host_order && ensure_order(c, scratch) == FFBF_OK;
    if (!on_device) c->err.clear();
    if (on_device) CUDA_TRY(c, ffbf::order_matches(c->d_moff, c->d_mpid, nm, kb, c->d_order, scratch, c->st));
    const size_t at = off_out.size();
    off_out.resize(at + nm);
    pid_out.resize(at + nm);
    if (nm) {
        CUDA_TRY(c, cudaMemcpyAsync(off_out.data() + at, c->d_moff, nm * 8ull, cudaMemcpyDeviceToHost, c->st));
        CUDA_TRY(c, cudaMemcpyAsync(pid_out.data() + at, c->d_mpid, nm * 4ull, cudaMemcpyDeviceToHost, c->st));
    }
    TRY(sync(c));
    if (!on_device) {
        std::vector<std::pair<uint64_t, uint32_t>> m(nm);
        for (size_t i = 0; i < nm; i++) m[i] = {off_out[at + i], pid_out[at + i]};
        std::sort(m.begin(), m.end());
        for (size_t i = 0; i < nm; i++) {
            off_out[at + i] = m[i].first;
            pid_out[at + i] = m[i].second;
        }
    }
    for (size_t i = at; i < off_out.size(); i++) off_out[i] += base;
    return FFBF_OK;
}

}  // namespace

extern "C" {

ffbf_status ffbf_verify(ffbf_ctx* c, ffbf_matches* out) {
    NvtxRange nvtx_("ffbf_verify");
    TRY(enter(c));
    if (c->scan_pending) TRY(ffbf_scan_collect(c, nullptr));
    if (!c->have_scan) return fail(c, FFBF_ESTATE, "ffbf_verify needs a scan first");
    if (!c->have_prune) TRY(ffbf_prune(c, nullptr));
    uint64_t tsize = 64;
    while (tsize < 2 * c->nids + 2) tsize <<= 1;
    if (c->table_cap < tsize) {
        dfree(c, c->d_keys);
        dfree(c, c->d_vals);
        c->table_cap = 0;
        TRY(dalloc_t(c, &c->d_keys, tsize));
        TRY(dalloc_t(c, &c->d_vals, tsize));
        c->table_cap = tsize;
    }
    CUDA_TRY(c, cudaMemsetAsync(c->d_vals, 0xff, tsize * 4, c->st));
    CUDA_TRY(c, cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * 4, c->st));
    CUDA_TRY(c, ffbf::table_build(c->d_ids, c->nids, c->d_phash, c->d_keys, c->d_vals, tsize - 1, c->d_counters, c->st));
    CUDA_TRY(c, cudaMemcpyAsync(c->h_counters, c->d_counters, ffbf::CNT_WORDS * 4, cudaMemcpyDeviceToHost, c->st));
    TRY(sync(c));
    if (c->h_counters[ffbf::CNT_ERROR]) return fail(c, FFBF_ECUDA, "verification table overflow");
    std::vector<uint64_t> off;
    std::vector<uint32_t> pid;
    if (!c->segmented) {
        TRY(verify_pass(c, c->nhits, c->d_text, c->text_len, tsize, 0, off, pid));
    } else {
        // the text was scanned in segments: each segment's text goes back to the device with its hit records
        for (const auto& sg : c->segs) {
            const uint64_t nh = sg.hr_end - sg.hr_begin;
            if (!nh) continue;
            if (c->hits_cap < nh) {
                dfree(c, c->d_hits);
                dfree(c, c->d_hitlines);
                c->hits_cap = 0;
                TRY(dalloc_t(c, &c->d_hits, nh));
                TRY(dalloc_t(c, &c->d_hitlines, nh));
                c->hits_cap = (uint32_t)nh;
            }
            if (c->text_cap < sg.len + 64) {
                dfree(c, c->d_text_own);
                c->text_cap = 0;
                TRY(dalloc_t(c, &c->d_text_own, sg.len + 64));
                c->text_cap = sg.len + 64;
            }
            std::vector<HitRec> rel(c->seg_hr.begin() + sg.hr_begin, c->seg_hr.begin() + sg.hr_end);
            for (auto& h : rel) h.off -= sg.pos;
            CUDA_TRY(c, cudaMemcpyAsync(c->d_text_own, c->seg_text + sg.pos, sg.len, cudaMemcpyHostToDevice, c->st));
            CUDA_TRY(c, cudaMemcpyAsync(c->d_hits, rel.data(), nh * sizeof(HitRec), cudaMemcpyHostToDevice, c->st));
            TRY(verify_pass(c, (uint32_t)nh, c->d_text_own, sg.len, tsize, sg.pos, off, pid));
        }
    }
    // each pass's matches come sorted, and segments follow one another in the text
    const size_t nm = off.size();
    c->r_moff.swap(off);
    c->r_mpid.resize(nm);
    for (size_t i = 0; i < nm; i++) c->r_mpid[i] = pid[i];
    if (out) {
        out->n = nm;
        out->offsets = c->r_moff.data();
        out->pattern_ids = c->r_mpid.data();
    }
    return FFBF_OK;
}

ffbf_status ffbf_test_line(ffbf_ctx* c, const uint8_t* line, size_t len, int* hit) {
    TRY(enter(c));
    if (!hit || (!line && len)) return fail(c, FFBF_EINVAL, "NULL argument");
    if (c->small_cap < len + 16) {
        dfree(c, c->d_small);
        c->small_cap = 0;
        TRY(dalloc_t(c, &c->d_small, len + 16));
        c->small_cap = len + 16;
    }
    if (len) CUDA_TRY(c, cudaMemcpyAsync(c->d_small, line, len, cudaMemcpyHostToDevice, c->st));
    CUDA_TRY(c, ffbf::test_line(c->d_small, len, c->g, c->d_main, c->d_counters + 3, c->st));
    uint32_t r = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&r, c->d_counters + 3, 4, cudaMemcpyDeviceToHost, c->st));
    TRY(sync(c));
    *hit = r ? 1 : 0;
    return FFBF_OK;
}

ffbf_status ffbf_debug_scan_unpublished(ffbf_ctx* c, const uint8_t* d_text, size_t len, uint32_t spins) {
    TRY(enter(c));
    if (!use_fast(c, len)) return fail(c, FFBF_EINVAL, "the tuned scan does not cover this geometry or size");
    TRY(setup_scan_state(c, d_text, len));
    if (!c->d_gate) TRY(dalloc_t(c, &c->d_gate, 1));
    CUDA_TRY(c, cudaMemsetAsync(c->d_gate, 0, sizeof(uint32_t), c->st));  // never published
    CUDA_TRY(c, cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * sizeof(uint32_t), c->st));
    TRY(prepare_fast(c));
    const ffbf::ScanArgs a = make_scan_args(c);
    const int threads = ffbf::config_threads(c->cfg);
    const uint32_t rows = c->cfg.rows ? c->cfg.rows : ffbf::fast_rows(len, c->cfg, c->num_sms, false);
    cudaError_t e;
    ffbf::fill_fast_job(a, c->d_stage1, c->cfg, rows, c->h_job, &e);
    if (e != cudaSuccess) return fail(c, FFBF_ECUDA, "tensor map encoding failed");
    c->h_job->ready = c->d_gate;
    c->h_job->ready_spins = spins;
    CUDA_TRY(c, cudaMemcpyAsync(c->d_job, c->h_job, sizeof(ffbf::FastJob), cudaMemcpyHostToDevice, c->st));
    CUDA_TRY(c, ffbf::launch_fast_jobs(c->g.len, c->cfg, c->d_job, 1, c->h_job->n_supertiles, c->h_job->stage1_nwords,
                                       c->d_counters + ffbf::CNT_ERROR, c->num_sms, c->st));
    CUDA_TRY(c, cudaMemcpyAsync(c->h_counters, c->d_counters, ffbf::CNT_WORDS * 4, cudaMemcpyDeviceToHost, c->st));
    TRY(sync(c));
    reset_scan(c);
    if (c->h_counters[ffbf::CNT_ERROR] & 4u)
        return fail(c, FFBF_ETIMEOUT, "the scan's publication gate stayed closed for %u polls", spins);
    return fail(c, FFBF_ESTATE, "the unpublished scan did not time out");
}

ffbf_status ffbf_get_scan_config(const ffbf_ctx* c, int* threads, int* mode) {
    if (!c) return FFBF_EINVAL;
    if (threads) *threads = ffbf::config_threads(c->cfg);
    if (mode) *mode = c->cfg.mode;
    return FFBF_OK;
}

ffbf_status ffbf_get_probe_order(const ffbf_ctx* c, int* order) {
    if (!c || !order) return FFBF_EINVAL;
    *order = c->cfg.order;
    return FFBF_OK;
}

ffbf_status ffbf_clear_ff(ffbf_ctx* c) {
    TRY(enter(c));
    CUDA_TRY(c, cudaMemsetAsync(c->d_ff, 0, c->filter_bytes, c->st));
    c->have_prune = false;
    return FFBF_OK;
}

ffbf_status ffbf_get_filters(ffbf_ctx* c, uint8_t* main_bits, uint8_t* ff_bits) {
    TRY(enter(c));
    if (c->scan_pending) TRY(ffbf_scan_collect(c, nullptr));
    if (main_bits) CUDA_TRY(c, cudaMemcpyAsync(main_bits, c->d_main, c->filter_bytes, cudaMemcpyDeviceToHost, c->st));
    if (ff_bits) CUDA_TRY(c, cudaMemcpyAsync(ff_bits, c->d_ff, c->filter_bytes, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

}  // extern "C"

