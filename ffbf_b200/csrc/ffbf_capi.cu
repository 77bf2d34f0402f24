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

using ffbf::Geom;
using ffbf::HitLine;
using ffbf::HitRec;

struct ffbf_ctx {
    ffbf_params prm{};
    Geom g{};
    int device = 0;
    int num_sms = 0;
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
    HitRec* d_hits = nullptr;
    HitLine* d_hitlines = nullptr;
    uint32_t hits_cap = 0;
    uint32_t nhits = 0;
    long long* d_tiles = nullptr;  // 4 arrays of tiles_cap: first, last, prev, next
    uint64_t tiles_cap = 0;
    int scan_path = 0;             // 0 = generic, 1 = fast
    uint32_t* d_stage1 = nullptr;  // stage-1 table of the tuned scan (cache copy or its fold)
    bool stage1_dirty = true;
    int stage1_threads = 0;        // CTA size the table was sized for
    unsigned long long* d_popc = nullptr;
    double stage1_fill = 0;
    ffbf::FastConfig cfg{512, 0, 0};  // tuned-scan configuration (mode from the stage-1 fill, or the autotuner)
    bool cfg_tuned = false;
    int force_mode = -1;           // FFBF_SCAN_MODE=0|1 in the environment
    bool force_generic = false;    // FFBF_FORCE_GENERIC_SCAN=1 in the environment
    ffbf::FastJob* h_job = nullptr;  // pinned staging of a plain scan's job descriptor
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
    uint8_t* d_small = nullptr;  // test_line input
    size_t small_cap = 0;
};

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
        bool operator==(const Key& o) const {
            return main == o.main && ff == o.ff && hits == o.hits && counters == o.counters && tiles == o.tiles &&
                   stage1 == o.stage1 && hits_cap == o.hits_cap && tiles_cap == o.tiles_cap && threads == o.threads &&
                   mode == o.mode && rows == o.rows;
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
    std::function<cudaError_t()> direct;  // the same launches without a graph (FFBF_BATCH_NOGRAPH=1)
};

namespace {

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

ffbf_status ensure_tmp(ffbf_ctx* c, size_t words) {
    if (c->tmp_words >= words) return FFBF_OK;
    dfree(c, c->d_tmp);
    c->tmp_words = 0;
    TRY(dalloc_t(c, &c->d_tmp, words));
    c->tmp_words = words;
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

// Makes the tuned scan ready for this context's filter: the stage-1 table for the configured CTA size and,
// unless the autotuner or the environment fixed it, the probe mode from the table's fill (the shared-memory
// stage only pays while it rejects most windows).
ffbf_status prepare_fast(ffbf_ctx* c) {
    const int sparse_threads = c->cfg.mode == 1 && c->cfg_tuned ? ffbf::fast_scan_threads() : c->cfg.threads;
    if (c->d_stage1 && c->stage1_threads != sparse_threads) {
        dfree(c, c->d_stage1);
        c->stage1_dirty = true;
    }
    if (!c->d_popc) TRY(dalloc_t(c, &c->d_popc, 1));
    if (!c->h_job) {
        if (cudaMallocHost(&c->h_job, sizeof(ffbf::FastJob)) != cudaSuccess) {
            cudaGetLastError();
            c->h_job = nullptr;
            return fail(c, FFBF_ENOMEM_HOST, "pinned job descriptor");
        }
    }
    if (!c->d_job) TRY(dalloc_t(c, &c->d_job, 1));
    if (!c->d_stage1) {
        TRY(dalloc_t(c, &c->d_stage1, ffbf::stage1_words_for(c->g, sparse_threads)));
        c->stage1_threads = sparse_threads;
        c->stage1_dirty = true;
    }
    if (c->stage1_dirty) {
        CUDA_TRY(c, ffbf::build_stage1(c->d_main, c->g, sparse_threads, c->d_stage1, c->st));
        const uint32_t nw = ffbf::stage1_words_for(c->g, sparse_threads);
        CUDA_TRY(c, ffbf::popcount_words(c->d_stage1, nw, c->d_popc, c->st));
        unsigned long long ones = 0;
        CUDA_TRY(c, cudaMemcpyAsync(&ones, c->d_popc, sizeof ones, cudaMemcpyDeviceToHost, c->st));
        TRY(sync(c));
        c->stage1_fill = (double)ones / (32.0 * nw);
        if (!c->cfg_tuned) c->cfg.mode = c->stage1_fill > 0.3 ? 1 : 0;
        c->stage1_dirty = false;
    }
    if (c->force_mode >= 0) c->cfg.mode = c->force_mode;
    return FFBF_OK;
}

ffbf_batch::Key batch_key(const ffbf_ctx* c) {
    return ffbf_batch::Key{c->d_main, c->d_ff,          c->d_hits,      c->d_counters, c->d_tiles,
                           c->d_stage1, c->hits_cap,    c->tiles_cap,   c->cfg.threads, c->cfg.mode,
                           c->cfg.rows};
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
    const uint64_t ntiles = (len + ffbf::kScanTile - 1) / ffbf::kScanTile;
    if (c->tiles_cap < ntiles) {
        dfree(c, c->d_tiles);
        c->tiles_cap = 0;
        TRY(dalloc_t(c, &c->d_tiles, 4 * ntiles));
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

}  // namespace

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
    if (th) ffbf::set_fast_scan_threads(atoi(th));
    c->cfg.threads = ffbf::fast_scan_threads();
    const char* fm = getenv("FFBF_SCAN_MODE");
    if (fm && (fm[0] == '0' || fm[0] == '1')) c->force_mode = fm[0] - '0';
    const char* fg = getenv("FFBF_FORCE_GENERIC_SCAN");
    c->force_generic = fg && fg[0] == '1';
    *out = c;
    return FFBF_OK;
}

void ffbf_destroy(ffbf_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    for (auto& kv : c->allocs) cudaFree(kv.first);
    c->allocs.clear();
    if (c->h_counters) cudaFreeHost(c->h_counters);
    if (c->h_job) cudaFreeHost(c->h_job);
    if (c->st) cudaStreamDestroy(c->st);
    cudaGetLastError();
    delete c;
}

const char* ffbf_last_error(const ffbf_ctx* c) { return c ? c->err.c_str() : "null context"; }

uint64_t ffbf_filter_bytes(const ffbf_ctx* c) { return c ? c->filter_bytes : 0; }

void ffbf_free(void* p) { free(p); }

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
    TRY(enter(c));
    TRY(setup_scan_state(c, d_text, len));
    TRY(launch_scan(c));
    c->scan_pending = true;
    return FFBF_OK;
}

ffbf_status ffbf_scan_collect(ffbf_ctx* c, ffbf_scan_result* out) {
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
                                        c->d_tiles + 3 * c->tiles_cap, ntiles, c->d_hitlines, c->st));
        std::vector<HitRec> hr(nh);
        std::vector<HitLine> hl(nh);
        if (nh) {
            CUDA_TRY(c, cudaMemcpyAsync(hr.data(), c->d_hits, nh * sizeof(HitRec), cudaMemcpyDeviceToHost, c->st));
            CUDA_TRY(c, cudaMemcpyAsync(hl.data(), c->d_hitlines, nh * sizeof(HitLine), cudaMemcpyDeviceToHost, c->st));
        }
        TRY(sync(c));
        std::vector<uint32_t> order(nh);
        for (uint32_t i = 0; i < nh; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return hr[a].off < hr[b].off; });
        c->r_hits.resize(nh);
        c->r_ls.clear();
        c->r_le.clear();
        for (uint32_t i = 0; i < nh; i++) {
            const uint32_t j = order[i];
            c->r_hits[i] = hr[j].off;
            if (c->r_ls.empty() || c->r_ls.back() != hl[j].start) {
                c->r_ls.push_back(hl[j].start);
                c->r_le.push_back(hl[j].end);
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

ffbf_status ffbf_scan(ffbf_ctx* c, const uint8_t* text, size_t len, ffbf_scan_result* out) {
    TRY(enter(c));
    if (!text && len) return fail(c, FFBF_EINVAL, "text is NULL");
    if (c->text_cap < len + 64) {
        dfree(c, c->d_text_own);
        c->text_cap = 0;
        TRY(dalloc_t(c, &c->d_text_own, len + 64));
        c->text_cap = len + 64;
    }
    if (len) CUDA_TRY(c, cudaMemcpyAsync(c->d_text_own, text, len, cudaMemcpyHostToDevice, c->st));
    TRY(ffbf_scan_device(c, c->d_text_own, len));
    return ffbf_scan_collect(c, out);
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
    TRY(enter(c));
    if (!c->have_patterns) return fail(c, FFBF_ESTATE, "ffbf_prune needs ffbf_set_patterns first");
    if (c->scan_pending) TRY(ffbf_scan_collect(c, nullptr));
    const uint64_t n = c->npat;
    const uint64_t nb = ffbf::compact_blocks(n);
    TRY(ensure_tmp(c, nb + 1));
    uint8_t* d_flags = nullptr;
    TRY(dalloc_t(c, &d_flags, n + 1));
    ffbf_status s = FFBF_OK;
    uint64_t cnt = 0;
    if (ffbf::prune_flags(c->d_pstart, c->d_pend, c->d_phash, n, c->g, c->d_ff, d_flags, c->st) != cudaSuccess ||
        ffbf::count_flags(d_flags, n, c->d_tmp, c->st) != cudaSuccess ||
        cudaMemcpyAsync(&cnt, c->d_tmp + nb, 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess)
        s = fail(c, FFBF_ECUDA, "prune failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (s == FFBF_OK) {
        dfree(c, c->d_ids);
        s = dalloc_t(c, &c->d_ids, cnt + 1);
    }
    if (s == FFBF_OK) {
        c->r_ids.resize(cnt);
        if (ffbf::emit_flags(d_flags, n, c->d_ids, c->d_tmp, c->st) != cudaSuccess ||
            (cnt && cudaMemcpyAsync(c->r_ids.data(), c->d_ids, cnt * 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess) ||
            cudaStreamSynchronize(c->st) != cudaSuccess)
            s = fail(c, FFBF_ECUDA, "prune compaction failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    dfree(c, d_flags);
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

ffbf_status ffbf_verify(ffbf_ctx* c, ffbf_matches* out) {
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
    const uint32_t nh = c->nhits;
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
        CUDA_TRY(c, cudaMemsetAsync(c->d_vals, 0xff, tsize * 4, c->st));
        CUDA_TRY(c, cudaMemsetAsync(c->d_counters, 0, ffbf::CNT_WORDS * 4, c->st));
        CUDA_TRY(c, ffbf::table_build(c->d_ids, c->nids, c->d_phash, c->d_keys, c->d_vals, tsize - 1, c->d_counters, c->st));
        CUDA_TRY(c, ffbf::verify_hits(c->d_hits, nh, c->d_text, c->text_len, c->d_keys, c->d_vals, tsize - 1, c->d_pat,
                                      c->d_pstart, c->d_pend, c->d_moff, c->d_mpid, c->match_cap, c->d_counters, c->st));
        CUDA_TRY(c, cudaMemcpyAsync(c->h_counters, c->d_counters, ffbf::CNT_WORDS * 4, cudaMemcpyDeviceToHost, c->st));
        TRY(sync(c));
        if (c->h_counters[ffbf::CNT_ERROR]) return fail(c, FFBF_ECUDA, "verification table overflow");
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
    std::vector<uint64_t> off(nm);
    std::vector<uint32_t> pid(nm);
    if (nm) {
        CUDA_TRY(c, cudaMemcpyAsync(off.data(), c->d_moff, nm * 8ull, cudaMemcpyDeviceToHost, c->st));
        CUDA_TRY(c, cudaMemcpyAsync(pid.data(), c->d_mpid, nm * 4ull, cudaMemcpyDeviceToHost, c->st));
    }
    TRY(sync(c));
    std::vector<uint32_t> order(nm);
    for (uint32_t i = 0; i < nm; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return off[a] != off[b] ? off[a] < off[b] : pid[a] < pid[b];
    });
    c->r_moff.resize(nm);
    c->r_mpid.resize(nm);
    for (uint32_t i = 0; i < nm; i++) {
        c->r_moff[i] = off[order[i]];
        c->r_mpid[i] = pid[order[i]];
    }
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

// ---- batched scans ---------------------------------------------------------------------------------------
namespace {

ffbf_status bfail(ffbf_batch* b, ffbf_status s, const std::string& msg) {
    b->err = msg;
    return s;
}

void batch_release(ffbf_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
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
    if (!b) return FFBF_EINVAL;
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, FFBF_ECUDA, "cudaSetDevice failed");
    batch_release(b);
    struct Group {
        uint32_t len;
        ffbf::FastConfig cfg;
        std::vector<std::pair<uint64_t, ffbf::FastJob>> jobs;  // (bytes, descriptor)
    };
    std::vector<Group> groups;
    std::vector<ffbf::ScanArgs> args;
    std::vector<uint2> tail;
    std::vector<uint32_t*> counters;
    for (uint32_t i = 0; i < b->jobs.size(); i++) {
        ffbf_ctx* c = b->jobs[i].c;
        ffbf_status s = enter(c);
        if (s == FFBF_OK) s = setup_scan_state(c, b->jobs[i].text, b->jobs[i].len);
        if (s != FFBF_OK) return bfail(b, s, std::string("job setup: ") + c->err);
        const ffbf::ScanArgs a = make_scan_args(c);
        args.push_back(a);
        counters.push_back(c->d_counters);
        uint64_t covered = 0;
        if (use_fast(c, a.n)) {
            if ((s = prepare_fast(c)) != FFBF_OK) return bfail(b, s, std::string("job filter: ") + c->err);
            const ffbf::FastConfig cfg = c->cfg;
            const int threads = ffbf::config_threads(cfg);
            const uint32_t rows = cfg.rows ? cfg.rows : ffbf::fast_rows(a.n, threads, b->num_sms, true);
            ffbf::FastJob fj;
            cudaError_t e;
            covered = ffbf::fill_fast_job(a, c->d_stage1, cfg, rows, &fj, &e);
            if (e != cudaSuccess) return bfail(b, FFBF_ECUDA, "tensor map encoding failed");
            if (fj.n_supertiles) {
                Group* gp = nullptr;
                for (auto& g : groups)
                    if (g.len == c->g.len && g.cfg.mode == cfg.mode && ffbf::config_threads(g.cfg) == threads) gp = &g;
                if (!gp) {
                    groups.push_back(Group{c->g.len, cfg, {}});
                    gp = &groups.back();
                }
                gp->jobs.push_back({covered, fj});
            }
        }
        for (uint64_t t = covered / ffbf::kScanTile; t < a.ntiles; t++) tail.push_back(make_uint2(i, (uint32_t)t));
        if (cudaStreamSynchronize(c->st) != cudaSuccess) return bfail(b, FFBF_ECUDA, "context stream failed");
        c->scan_pending = true;
        b->keys.push_back(batch_key(c));
    }
    // descriptors: groups contiguous, largest jobs first within a group
    std::vector<ffbf::FastJob> fast;
    struct Launch {
        uint32_t len;
        ffbf::FastConfig cfg;
        size_t off;
        uint32_t n_jobs, n_items, max_s1;
    };
    std::vector<Launch> launches;
    for (auto& g : groups) {
        std::stable_sort(g.jobs.begin(), g.jobs.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        Launch L{g.len, g.cfg, fast.size(), (uint32_t)g.jobs.size(), 0, 0};
        for (auto& jb : g.jobs) {
            jb.second.item_begin = L.n_items;
            L.n_items += jb.second.n_supertiles;
            L.max_s1 = std::max(L.max_s1, jb.second.stage1_nwords);
            fast.push_back(jb.second);
        }
        launches.push_back(L);
    }
    ffbf::FastJob* d_fast = nullptr;
    ffbf::ScanArgs* d_args = nullptr;
    uint2* d_tail = nullptr;
    uint32_t** d_counters = nullptr;
    TRY(balloc(b, &d_fast, fast.size() + 1));
    TRY(balloc(b, &d_args, args.size() + 1));
    TRY(balloc(b, &d_tail, tail.size() + 1));
    // per tuned launch: 4 control words (error flags, work-queue counter), zeroed with the job counters
    TRY(balloc(b, &b->d_error, 4 * (launches.size() + 1)));
    b->n_ctl = (uint32_t)launches.size() + 1;
    for (uint32_t i = 0; i < b->n_ctl; i++) counters.push_back(b->d_error + 4 * i);
    TRY(balloc(b, &d_counters, counters.size() + 1));
    if ((fast.size() && cudaMemcpy(d_fast, fast.data(), fast.size() * sizeof(ffbf::FastJob), cudaMemcpyHostToDevice)) ||
        (args.size() && cudaMemcpy(d_args, args.data(), args.size() * sizeof(ffbf::ScanArgs), cudaMemcpyHostToDevice)) ||
        (tail.size() && cudaMemcpy(d_tail, tail.data(), tail.size() * sizeof(uint2), cudaMemcpyHostToDevice)) ||
        (counters.size() &&
         cudaMemcpy(d_counters, counters.data(), counters.size() * sizeof(uint32_t*), cudaMemcpyHostToDevice)) ||
        cudaMemset(b->d_error, 0, 16 * b->n_ctl))
        return bfail(b, FFBF_ECUDA, "batch table upload failed");
    const char* dbg = getenv("FFBF_BATCH_DEBUG");
    if (dbg && dbg[0] == '1') {
        // diagnostic: the same launches, uncaptured, each checked before the next
        auto check = [&](cudaError_t e, const char* what) -> ffbf_status {
            if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return bfail(b, FFBF_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
            }
            return FFBF_OK;
        };
        TRY(check(ffbf::zero_counters(d_counters, (uint32_t)counters.size(), b->st), "zero_counters"));
        for (size_t li = 0; li < launches.size(); li++) {
            const Launch& L = launches[li];
            char what[96];
            snprintf(what, sizeof what, "tuned launch len %u threads %d mode %d jobs %u items %u", L.len,
                     ffbf::config_threads(L.cfg), L.cfg.mode, L.n_jobs, L.n_items);
            TRY(check(ffbf::launch_fast_jobs(L.len, L.cfg, d_fast + L.off, L.n_jobs, L.n_items, L.max_s1,
                                             b->d_error + 4 * li, b->num_sms, b->st),
                      what));
        }
        TRY(check(ffbf::scan_generic_multi(d_args, d_tail, (uint32_t)tail.size(), b->num_sms, b->st), "generic tail"));
    }
    {
        const uint32_t n_counters = (uint32_t)counters.size(), n_tail = (uint32_t)tail.size();
        b->direct = [=]() {
            cudaError_t e = ffbf::zero_counters(d_counters, n_counters, b->st);
            for (size_t li = 0; li < launches.size() && e == cudaSuccess; li++) {
                const Launch& L = launches[li];
                e = ffbf::launch_fast_jobs(L.len, L.cfg, d_fast + L.off, L.n_jobs, L.n_items, L.max_s1,
                                           b->d_error + 4 * li, b->num_sms, b->st);
            }
            if (e == cudaSuccess) e = ffbf::scan_generic_multi(d_args, d_tail, n_tail, b->num_sms, b->st);
            return e;
        };
    }
    // one graph: zero the jobs' counters, one tuned launch per group, one generic launch for all tail tiles
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return bfail(b, FFBF_ECUDA, "stream capture failed to start");
    const uint64_t launches0 = ffbf::launches_total();
    cudaError_t e = ffbf::zero_counters(d_counters, (uint32_t)counters.size(), b->st);
    for (size_t li = 0; li < launches.size() && e == cudaSuccess; li++) {
        const Launch& L = launches[li];
        e = ffbf::launch_fast_jobs(L.len, L.cfg, d_fast + L.off, L.n_jobs, L.n_items, L.max_s1, b->d_error + 4 * li,
                                   b->num_sms, b->st);
    }
    if (e == cudaSuccess) e = ffbf::scan_generic_multi(d_args, d_tail, (uint32_t)tail.size(), b->num_sms, b->st);
    cudaError_t e2 = cudaStreamEndCapture(b->st, &b->graph);
    b->graph_kernels = ffbf::launches_total() - launches0;  // counted again at each graph launch
    ffbf::unnote_launches(b->graph_kernels);
    if (e != cudaSuccess || e2 != cudaSuccess || cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, FFBF_ECUDA, std::string("batch graph capture failed: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    b->prepared = true;
    return FFBF_OK;
}

ffbf_status ffbf_batch_launch(ffbf_batch* b) {
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
    const char* ng = getenv("FFBF_BATCH_NOGRAPH");
    if (ng && ng[0] == '1') {
        if (b->direct() != cudaSuccess) {
            cudaGetLastError();
            return bfail(b, FFBF_ECUDA, "direct batch launch failed");
        }
        return FFBF_OK;
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

ffbf_status ffbf_autotune(ffbf_ctx* c, const uint8_t* d_text, size_t sample_len, int* threads, int* mode) {
    TRY(enter(c));
    if (!d_text || ((uintptr_t)d_text & 15)) return fail(c, FFBF_EINVAL, "device text must be 16-byte aligned");
    if (!use_fast(c, sample_len)) return fail(c, FFBF_EINVAL, "the tuned scan does not cover this geometry or size");
    // keep the feed-forward filter: the trial scans set bits in it
    uint32_t* saved = nullptr;
    TRY(dalloc_t(c, &saved, c->filter_bytes / 4));
    CUDA_TRY(c, cudaMemcpyAsync(saved, c->d_ff, c->filter_bytes, cudaMemcpyDeviceToDevice, c->st));
    const ffbf::FastConfig cands[] = {{512, 0, 0}, {384, 0, 0}, {256, 0, 0}, {256, 1, 0}};
    ffbf::FastConfig best = c->cfg;
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int saved_force = c->force_mode;
    c->force_mode = -1;
    ffbf_status s = FFBF_OK;
    for (const auto& cand : cands) {
        c->cfg = cand;
        c->cfg_tuned = true;
        ffbf::set_fast_scan_threads(cand.mode == 0 ? cand.threads : 0);
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
        if (ms < best_ms) {
            best_ms = ms;
            best = cand;
        }
    }
    c->force_mode = saved_force;
    ffbf::set_fast_scan_threads(best.mode == 0 ? best.threads : 0);
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

}  // extern "C"
