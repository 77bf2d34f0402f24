/*
 * ffbf.h -- C ABI of the B200 feed-forward Bloom filter (FFBF) matcher.
 *
 * Drop-in for the x86 rabin-karp path of efficient/ffbf. The reference's interface for that path is the
 * C++ class Filter<H, LEN> (src/rabin-karp/ffbf.h:43-93) plus the `ffbf` CLI (src/rabin-karp/ffbf.cpp:529-601);
 * every entry point below names the member or step it replaces. Differences that are part of the contract:
 *
 *  - The filter geometry (LEN, K, S, cache and external region sizes) is a runtime ffbf_params value
 *    instead of compile-time macros (src/rabin-karp/Makefile.am:1-32, ffbf.cpp:55-83). The same values give
 *    bit-identical filters and outputs.
 *  - Errors are status codes, never exceptions. FilterError (ffbf.h:31-41) becomes a non-zero ffbf_status
 *    and ffbf_last_error() holds its message.
 *  - Inputs are byte buffers (a pattern file image, a text image) rather than file descriptors; the CLI
 *    (ffbf_b200/csrc/ffbf_cli.cpp) and the C++ mirror (include/ffbf.hpp) read files and call these.
 *  - All computation runs on one CUDA device. There is no CPU fallback: without a usable device,
 *    ffbf_create fails with FFBF_ECUDA.
 *
 * Threading: one context is used by one host thread at a time. Distinct contexts are independent and may
 * run concurrently on different streams. Result pointers returned in ffbf_*_result structs are owned by
 * the context and stay valid until the next call of the same kind on that context, or ffbf_destroy.
 */
#ifndef FFBF_B200_FFBF_H
#define FFBF_B200_FFBF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FFBF_OK = 0,
    FFBF_EINVAL = 1,          /* bad argument: geometry, NULL pointer, misaligned device pointer, bad file */
    FFBF_ENOMEM_DEVICE = 2,   /* device allocation failed or would exceed the context's HBM budget */
    FFBF_EIO = 3,             /* file open/read/write failed (the *_file entry points) */
    FFBF_ETIMEOUT = 4,        /* a bounded device-side wait gave up (batched/served forms) */
    FFBF_ECUDA = 5,           /* a CUDA runtime call failed; ffbf_last_error has the CUDA message */
    FFBF_ESTATE = 6,          /* call out of order, e.g. ffbf_build before ffbf_set_patterns */
    FFBF_ENOMEM_HOST = 7      /* host allocation failed */
} ffbf_status;

/* Filter geometry. Field <-> reference macro: len = DEF_PATT_LEN, k = DEF_K, s = DEF_S,
 * cache_bits = DEF_CACHE_SIZE, ext_bits = DEF_EXT_SIZE (ffbf.cpp:55-77, 79-83).
 * Constraints (those of the reference's uint32 arithmetic): 1 <= len <= 63, 1 <= k <= 11, 0 <= s <= k,
 * cache_bits and ext_bits powers of two, cache_bits + ext_bits <= 2^31. */
typedef struct {
    uint32_t len;
    uint32_t k;
    uint32_t s;
    uint32_t reserved;     /* must be 0 */
    uint64_t cache_bits;
    uint64_t ext_bits;
} ffbf_params;

typedef struct ffbf_ctx ffbf_ctx;

/* Fills the reference's compile-time defaults: LEN 19, K 5, S 2, 2^24 cache bits, 2^28 external bits
 * (ffbf.cpp:55-77). */
ffbf_status ffbf_params_default(ffbf_params* p);

/* Filter<H,LEN>::Filter() (ffbf.cpp:87-108): allocates the main and the feed-forward bit arrays, N/8 bytes
 * each with N = cache_bits + ext_bits, zeroed, on `device`. */
ffbf_status ffbf_create(const ffbf_params* p, int device, ffbf_ctx** out);

/* Filter<H,LEN>::~Filter() (ffbf.cpp:110-116). NULL is accepted. */
void ffbf_destroy(ffbf_ctx* ctx);

/* FilterError::what() (ffbf.h:37-40) of the last failing call on ctx ("" if none). */
const char* ffbf_last_error(const ffbf_ctx* ctx);
const char* ffbf_status_string(ffbf_status s);

/* Limits the device memory this context may allocate (bytes; 0 = no limit beyond the device's). */
ffbf_status ffbf_set_hbm_budget(ffbf_ctx* ctx, uint64_t bytes);

/* Pattern file image, split into lines on '\n' exactly as main()'s getline loop (ffbf.cpp:556-558) and
 * filterPhrases (ffbf.cpp:426-447) do: a final line without '\n' is a line; a trailing '\n' adds none.
 * Copies the image to the device and hashes every line's LEN-byte prefix there. Sets no filter bits. */
ffbf_status ffbf_set_patterns(ffbf_ctx* ctx, const uint8_t* file, size_t len);

/* `filter << phrase` for every pattern line (operator<<, ffbf.cpp:268-283): lines shorter than LEN are
 * skipped; otherwise K bits of the main filter are set in getHashValue order (ffbf.cpp:135-159). */
ffbf_status ffbf_build(ffbf_ctx* ctx);

/* ffbf_set_patterns followed by ffbf_build. */
ffbf_status ffbf_add_patterns(ffbf_ctx* ctx, const uint8_t* file, size_t len);

/* loadFilterFromFile (ffbf.cpp:487-506): ORs the bits of a __bloom_filter_* image (consecutive
 * little-endian uint32 deltas between set-bit indices) into the main filter. A trailing partial word is
 * ignored. An index at or beyond N gives FFBF_EINVAL and leaves the filter unchanged. */
ffbf_status ffbf_load_filter(ffbf_ctx* ctx, const uint8_t* data, size_t len);

/* saveFilterToFile (ffbf.cpp:508-527): encodes the main filter in the same delta format. *data is
 * allocated by the library; release it with ffbf_free. */
ffbf_status ffbf_save_filter(ffbf_ctx* ctx, uint8_t** data, size_t* len);

/* File-path forms of the two above, for the CLI's __bloom_filter_<patterns> cache (ffbf.cpp:545-575). */
ffbf_status ffbf_load_filter_file(ffbf_ctx* ctx, const char* path);
ffbf_status ffbf_save_filter_file(ffbf_ctx* ctx, const char* path);

/* Result of one scan. hit_offsets: start offset of every window whose K main bits are all set, ascending.
 * line_start/line_end: the lines holding at least one such window, in text order; a line is
 * [line_start, line_end) and excludes its '\n'. */
typedef struct {
    uint64_t text_len;
    uint64_t n_hits;
    const uint64_t* hit_offsets;
    uint64_t n_lines;
    const uint64_t* line_start;
    const uint64_t* line_end;
} ffbf_scan_result;

/* processFile (ffbf.cpp:310-392) over a host text image: the hash rolls over every line ('\n' resets it
 * and is not hashed); every window whose K main bits are set marks its line and sets K bits of the
 * feed-forward filter in getHashValue_2 order (ffbf.cpp:161-185). The feed-forward filter accumulates
 * over successive scans, as it does over one reference run; ffbf_clear_ff starts a new one.
 * A text of 32 MiB or more is copied in chunks while the chunks already on the device are scanned. A text
 * larger than the device can hold (its free memory, or the context's HBM budget) is scanned in segments
 * that each end after a '\n' (a line longer than a segment gives FFBF_EINVAL); the results are the same,
 * and ffbf_verify then copies the segments again, so the text must stay valid until ffbf_verify. */
ffbf_status ffbf_scan(ffbf_ctx* ctx, const uint8_t* text, size_t len, ffbf_scan_result* out);

/* The same scan over a text already in device memory (16-byte aligned), enqueued on the context's
 * stream; ffbf_scan_collect waits for it and fills `out`. */
ffbf_status ffbf_scan_device(ffbf_ctx* ctx, const uint8_t* d_text, size_t len);
ffbf_status ffbf_scan_collect(ffbf_ctx* ctx, ffbf_scan_result* out);

/* What processFile writes to stdout for the last scan: every flagged line followed by '\n', with the
 * reference's output rules reproduced byte for byte -- each line is printed as C strings (cut at its
 * first NUL), and a line crossing read() chunk boundaries of `chunk` bytes (512 KiB in the reference,
 * ffbf.cpp:313, when reading a regular file) prints only its last two chunks' parts (the carry buffer is
 * overwritten, ffbf.cpp:372-382); a flagged final line without '\n' prints only its last chunk's part.
 * Needs the host text image the scan ran on. *out is library-allocated; release with ffbf_free. */
ffbf_status ffbf_format_lines(ffbf_ctx* ctx, const uint8_t* text, size_t len, size_t chunk,
                              uint8_t** out, size_t* out_len);

/* The output rule above as a stand-alone host function: writes buf[start[i], end[i]) for each i, each
 * followed by '\n', exactly as processFile/filterPhrases print a flagged line of a `len`-byte input read in
 * `chunk`-byte pieces (C-string cut at NUL; carry of the previous chunk only; a final line without '\n'
 * prints only its last chunk's part). end[i] == len marks a final line without '\n'. Spans must be
 * ascending, non-overlapping lines of buf. Needs no context and no device. Library-allocated output. */
ffbf_status ffbf_format_spans(const uint8_t* buf, size_t len, const uint64_t* start, const uint64_t* end, size_t n,
                              size_t chunk, uint8_t** out, size_t* out_len);

/* Result of the feed-forward pass: 0-based line numbers of the surviving patterns, ascending. */
typedef struct {
    uint64_t n_ids;
    const uint64_t* ids;
} ffbf_prune_result;

/* filterPhrases (ffbf.cpp:394-485): a pattern line survives when it is at least LEN bytes long and its
 * prefix window has all K feed-forward bits set (getHashValue_2 order). */
ffbf_status ffbf_prune(ffbf_ctx* ctx, ffbf_prune_result* out);

/* The two files filterPhrases writes for the last prune: the pruned pattern file (each surviving line
 * then '\n', with the C-string and chunk-carry rules of ffbf.cpp:431-442,464-481 over `chunk`-byte reads of
 * the pattern file) and the __index_ file (one decimal line number per line). Library-allocated. */
ffbf_status ffbf_format_pruned(ffbf_ctx* ctx, size_t chunk, uint8_t** out, size_t* out_len,
                               uint8_t** index, size_t* index_len);

/* Exact matches: every (offset, pattern line number) where a pruned pattern's full bytes occur in the
 * last scanned text at a hit window's start. This is the `grep -Ff pruned candidates` step of the
 * reference workflow (src/rabin-karp/README:49-52) done on the device: candidates are looked up by their
 * 64-bit window hash in a table of the pruned patterns' prefix hashes, then byte-compared.
 * Sorted by offset, then pattern id. Patterns shorter than LEN are never reported (ffbf.cpp:271-275). */
typedef struct {
    uint64_t n;
    const uint64_t* offsets;
    const uint64_t* pattern_ids;
} ffbf_matches;
ffbf_status ffbf_verify(ffbf_ctx* ctx, ffbf_matches* out);

/* operator[] (ffbf.cpp:285-308): 1 when some LEN-byte window of `line` has all K main bits set. Like the
 * reference, '\n' inside `line` is hashed as an ordinary byte, and lines shorter than LEN give 0. */
ffbf_status ffbf_test_line(ffbf_ctx* ctx, const uint8_t* line, size_t len, int* hit);

/* ---- Batched scans ------------------------------------------------------------------------------------
 * Many (context, device text) jobs scanned together. The reference processes one text per run; batching
 * is this library's answer to many small jobs, which one launch per job leaves mostly idle: the tuned
 * kernel walks a combined list of all jobs' tiles, one persistent launch per group of jobs sharing LEN and
 * CTA shape, and all of a batch's launches are captured in one CUDA graph. Per job the tile size and the
 * filter placement (shared-memory stage 1 or pipelined L2 probes) are chosen by ffbf_autotune's rules.
 *
 * Each job writes into its own context as ffbf_scan_device would: after ffbf_batch_wait, call
 * ffbf_scan_collect (then ffbf_prune / ffbf_verify) on each context. A context may appear once per batch,
 * must not be used by other calls between ffbf_batch_prepare and ffbf_batch_wait, and its texts must stay
 * valid until then. ffbf_batch_launch may be called repeatedly (each launch zeroes the jobs' hit counters;
 * feed-forward filters accumulate, as for repeated scans). */
typedef struct ffbf_batch ffbf_batch;
ffbf_status ffbf_batch_create(int device, ffbf_batch** out);
ffbf_status ffbf_batch_add(ffbf_batch* b, ffbf_ctx* ctx, const uint8_t* d_text, size_t len);
ffbf_status ffbf_batch_prepare(ffbf_batch* b);   /* job tables, stage-1 tables, graph capture */
ffbf_status ffbf_batch_launch(ffbf_batch* b);    /* one graph launch on the batch's stream */
ffbf_status ffbf_batch_wait(ffbf_batch* b);
void* ffbf_batch_stream(ffbf_batch* b);
const char* ffbf_batch_last_error(const ffbf_batch* b);
void ffbf_batch_destroy(ffbf_batch* b);
/* Autotunes a batch's jobs by class: jobs with the same geometry and a similar stage-1 table fill form a
 * class; ffbf_autotune times the configurations on the first `sample_bytes` (0: 16 MiB) of the class's
 * largest text, and every job of the class takes the winner. The next launch prepares again. */
ffbf_status ffbf_batch_autotune(ffbf_batch* b, size_t sample_bytes, uint32_t* n_classes);

/* Scan server: pattern sets resident on the device, scan requests admitted while device memory allows,
 * and every admitted request whose text has reached the device scanned together in the next launch
 * sequence (continuous batching). The reference has no counterpart: it scans one corpus per process
 * (ffbf.cpp:529-601); a request here produces what ffbf_scan would for its text and set.
 *
 * ffbf_server_create caps the device memory it holds for request texts at `arena_bytes` (0: no cap) and
 * takes `slots` request slots (0: 64). The text arena starts as one segment (1 GiB, or the cap if smaller)
 * and grows in segments while the device's free memory (cudaMemGetInfo, which counts every context's and
 * process's allocations) stays 1 GiB above what it takes; segments grown beyond the first go back to the
 * device after a quarter second without admitted requests. A host thread runs the loop: admit requests
 * in arrival order while a slot and arena room are free (a request that finds neither room nor enough free
 * device memory waits, and the requests behind it with it, until finished requests or other contexts free
 * memory), copy each text to the arena on a copy stream,
 * launch every request whose copy has finished as soon as the previous launch sequence is done, and
 * collect each finished request's hits and lines (the line resolution of one batch overlaps the next
 * batch's scan). A request's feed-forward bits go into its set's filter, as successive ffbf_scan calls on
 * the set would.
 *
 * Register sets with ffbf_server_add_set before the first submit (the server borrows the context's filters;
 * the context must not be modified or used for other calls until the server is destroyed). A submitted
 * text must stay valid until the request is polled; pinned host memory lets its copy overlap other work.
 * ffbf_server_poll returns finished requests (waiting up to wait_us microseconds for the first one);
 * their arrays stay valid until ffbf_server_release. Times are seconds since the server's creation,
 * from the host's steady clock. A request longer than the cap, or than the device's memory less 1 GiB, is
 * refused with FFBF_EINVAL. */
typedef struct ffbf_server ffbf_server;
typedef struct {
    uint64_t request_id;
    uint32_t set_id;
    ffbf_status status;
    uint64_t text_len;
    uint64_t n_hits;
    const uint64_t* hit_offsets; /* ascending */
    uint64_t n_lines;
    const uint64_t* line_start;  /* candidate lines, as ffbf_scan_result */
    const uint64_t* line_end;
    double t_submit, t_admit, t_launch, t_done;
} ffbf_request_result;
typedef struct {
    uint64_t requests_done, batches, bytes_scanned, max_batch;
    uint64_t arena_bytes;
    uint32_t slots;
} ffbf_server_stats;
ffbf_status ffbf_server_create(int device, uint64_t arena_bytes, uint32_t slots, ffbf_server** out);
ffbf_status ffbf_server_add_set(ffbf_server* s, ffbf_ctx* set, uint32_t* set_id);
ffbf_status ffbf_server_submit(ffbf_server* s, uint32_t set_id, const uint8_t* text, size_t len, uint64_t* request_id);
ffbf_status ffbf_server_poll(ffbf_server* s, ffbf_request_result* out, uint32_t max, uint32_t* n_out,
                             uint32_t wait_us);
ffbf_status ffbf_server_release(ffbf_server* s, uint64_t request_id);
ffbf_status ffbf_server_get_stats(ffbf_server* s, ffbf_server_stats* out);
const char* ffbf_server_last_error(const ffbf_server* s);
void ffbf_server_destroy(ffbf_server* s);  /* waits for work on the device; unfinished requests are dropped */

/* Autotuner: times the tuned scan's configurations (CTA size, shared-memory vs L2 filter placement) on the
 * first `sample_len` bytes of a device text with this context's filter, keeps the fastest for later scans
 * of the context, and reports it (threads, mode: 0 shared-memory stage, 1 pipelined L2 probes). The
 * feed-forward filter is left unchanged. Without it, the placement follows the stage-1 table's fill. */
ffbf_status ffbf_autotune(ffbf_ctx* ctx, const uint8_t* d_text, size_t sample_len, int* threads, int* mode);

/* Failure-detection check (no counterpart in the reference, which has no device waits): runs the tuned
 * scan of d_text gated on a device word that is never published. The kernel polls the word `spins` times
 * (about a microsecond apart), records the timeout and ends before issuing any load; the call returns
 * FFBF_ETIMEOUT and the context stays usable. Nothing is scanned and no result is kept. */
ffbf_status ffbf_debug_scan_unpublished(ffbf_ctx* ctx, const uint8_t* d_text, size_t len, uint32_t spins);

/* The tuned scan's current configuration for this context (CTA threads; mode 0 shared-memory stage 1 with
 * candidates queued per byte, 1 pipelined L2 probes, 2 shared-memory stage 1 with candidates deferred to the
 * end of each 32-byte block, 3 mode 0 at 512 threads whose warps meet through per-stage barriers), as the
 * autotuner or the filter's fill chose it. Before the first scan or tuning
 * it reports the defaults. */
ffbf_status ffbf_get_scan_config(const ffbf_ctx* ctx, int* threads, int* mode);

/* The dense mode's probe plan for this context's filter: 0 pipelines the loads of index functions f0 = h1
 * and f1 = h2, 1 those of f2 = rot16(h1) and f3 = rot16(h2) (K >= 4), 2 those of f0 and f1 with f0's load
 * skipped where a folded copy of the cache region in shared memory has its bit clear. Chosen from the
 * fills of the filter's regions when the filter is prepared for a scan (FFBF_SCAN_ORDER=0|1|2 fixes it);
 * a window hits iff all K bits are set, so the plan changes the work, never the result. */
ffbf_status ffbf_get_probe_order(const ffbf_ctx* ctx, int* order);

/* Zeroes the feed-forward filter (a fresh reverseBitvector, ffbf.cpp:107). Enqueued on the context's
 * stream; later calls on the context see it done. */
ffbf_status ffbf_clear_ff(ffbf_ctx* ctx);

/* Copies the main and/or feed-forward bit arrays (N/8 bytes each, bit i = byte i>>3, mask 1<<(i&7), as
 * setBit at ffbf.cpp:187-193) to host memory. Either pointer may be NULL. */
ffbf_status ffbf_get_filters(ffbf_ctx* ctx, uint8_t* main_bits, uint8_t* ff_bits);

/* Size in bytes of one bit array (N/8). */
uint64_t ffbf_filter_bytes(const ffbf_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t). Every device operation of the context is ordered on it;
 * callers may record events on it or make other streams wait on it. */
void* ffbf_stream(ffbf_ctx* ctx);

/* Number of CUDA kernels this library has launched in the process so far (all contexts). */
uint64_t ffbf_kernel_launches(void);

/* ffbf_scan_static: processFile's scan, run without allocating any device or host memory. This entry
 * point has no counterpart in the reference; it exists for callers that may not call cudaMalloc -- a
 * program whose own allocator owns every byte of device memory, a plug-in host that forbids allocation
 * in callbacks, a latency-critical loop that cannot take an allocation's implicit synchronisation.
 *
 * The caller passes the geometry, the main filter d_main (N/8 bytes, the layout ffbf_get_filters
 * returns), a feed-forward filter d_ff to OR hits into, the text (device, 16-byte aligned, at most
 * FFBF_STATIC_MAX_TEXT bytes) and three device output arrays of FFBF_STATIC_MAX_HITS entries each. On
 * return *n_hits holds the number of hit windows; d_hit_offsets[i] is a window start and
 * [d_line_start[i], d_line_end[i]) its line, in no particular order. All scratch memory comes from one
 * fixed device array of FFBF_STATIC_SCRATCH_BYTES compiled into the library, which every GPU that loads
 * the library holds until the process exits. Every call looks up that array's address in the context
 * current at the call (a lookup allocates nothing): after a cudaDeviceReset the next call finds the
 * reloaded array, and a caller's own driver-API context on the device uses the array of that context.
 * The first call in a context loads the module that holds the array there; make it before any stream
 * capture begins in that context. Work is ordered on `stream` (a cudaStream_t, 0 for the default); the
 * call waits for it. The array keeps the last call's contents (the call clears what must start at zero).
 * Calls whose work overlaps on the GPU share the array and race: serialise them.
 * Returns FFBF_EINVAL for a text longer than FFBF_STATIC_MAX_TEXT, and FFBF_ENOMEM_DEVICE when more than
 * FFBF_STATIC_MAX_HITS windows hit (*n_hits then holds the full count, the arrays a subset of it). */
#define FFBF_STATIC_MAX_TEXT (1ull << 30)
#define FFBF_STATIC_MAX_HITS (1u << 16)
#define FFBF_STATIC_SCRATCH_BYTES (256ull + 32ull * FFBF_STATIC_MAX_HITS + 32ull * (FFBF_STATIC_MAX_TEXT / 16384ull))
ffbf_status ffbf_scan_static(const ffbf_params* p, const uint32_t* d_main, uint32_t* d_ff, const uint8_t* d_text,
                             uint64_t len, uint64_t* d_hit_offsets, uint64_t* d_line_start, uint64_t* d_line_end,
                             uint32_t* n_hits, void* stream);

/* The reference's hash benchmark (src/hashes/hashbench.cc:60-130) for the scan's hash,
 * hash_rot_sbox_pre_2<19>, with the hashing on `device`. Raw bytes are hashed (hashbench does not map bytes
 * >= 0x80 to 0 as the filter does).
 *
 * ffbf_hashbench_lines is `hashbench -l` (hash_lines, :108-127): for every piece fgets(buf, 4095, f) would
 * return (a line through its '\n', or the next 4094 bytes of a longer line) the hash restarts, the bytes up
 * to the first NUL or '\n' are hashed, and "%x %s\n" prints hval() (the hash's high 32 bits) and that
 * string. *out holds exactly the bytes the reference prints; release it with ffbf_free.
 *
 * ffbf_hashbench_file is `hashbench -f` (hash_file, :60-99): the hash rolls over every byte with no restart.
 * The reference prints only the byte count and the time; here *xor_of_hashes is the XOR of the 64-bit hash
 * after every byte (a checkable result) and *seconds the device time of that pass (copy excluded). */
ffbf_status ffbf_hashbench_lines(int device, const uint8_t* text, size_t len, uint8_t** out, size_t* out_len);
ffbf_status ffbf_hashbench_file(int device, const uint8_t* text, size_t len, uint64_t* xor_of_hashes,
                                double* seconds);

/* Page-locked host memory (cudaMallocHost) for texts that ffbf_scan copies to the device: copies from it run
 * at full PCIe speed and overlap the scan, where pageable memory is staged. NULL on failure; release it with
 * ffbf_host_free. No counterpart in the reference. */
void* ffbf_host_alloc(size_t bytes);
void ffbf_host_free(void* p);

/* Releases memory the library allocated for an out-parameter. */
void ffbf_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* FFBF_B200_FFBF_H */
