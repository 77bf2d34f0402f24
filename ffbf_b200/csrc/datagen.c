/*
 * datagen.c -- seeded synthetic pattern sets and texts for the FFBF workloads.
 *
 * efficient/ffbf ships no data; its workflow is `ffbf patterns out < corpus` (src/rabin-karp/README:49-52).
 * The workloads here are the shapes the matcher is measured on: printable-ASCII patterns and texts with
 * geometric line lengths, Zipf-lettered "word" text, and uniform binary signatures, each with planted
 * pattern occurrences. Everything derives from one uint64 seed through splitmix64 -> xoshiro256**, with
 * integer-only arithmetic, so the same seed gives the same bytes on every x86-64 host and any thread count.
 *
 * Draw order (per seed): patterns, then text bytes (with newlines folded in as a per-byte Bernoulli
 * draw, which gives geometric line lengths), then planted occurrences, which overwrite text bytes.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { FFBF_GEN_PRINTABLE = 0, FFBF_GEN_ZIPF_WORDS = 1, FFBF_GEN_BINARY = 2 };

typedef struct { uint64_t s[4]; } xo_t;

static inline uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t xo_next(xo_t* r) {
    uint64_t* s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return result;
}
static void xo_seed(xo_t* r, uint64_t seed, uint64_t stream) {
    uint64_t x = seed ^ (stream * 0xd1342543de82ef95ull);
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}
/* uniform integer in [0, n) from 32 random bits (multiply-shift; bias < n / 2^32) */
static inline uint32_t below(uint32_t r32, uint32_t n) { return (uint32_t)(((uint64_t)r32 * n) >> 32); }

/* Zipf(s=1) over 26 lowercase letters: cumulative thresholds on 2^32, P(k) = (1/k) / H_26.
 * Built with integer arithmetic only: weights 1/k scaled by lcm-free fixed point 2^40 / k. */
static uint32_t g_zipf_cdf[26];
static int g_zipf_ready = 0;
static void zipf_init(void) {
    if (g_zipf_ready) return;
    uint64_t w[26], tot = 0;
    for (int k = 0; k < 26; k++) { w[k] = (1ull << 40) / (uint64_t)(k + 1); tot += w[k]; }
    uint64_t acc = 0;
    for (int k = 0; k < 26; k++) {
        acc += w[k];
        /* threshold = floor(acc / tot * 2^32) without floating point */
        unsigned __int128 t = ((unsigned __int128)acc << 32) / tot;
        g_zipf_cdf[k] = t >= ((unsigned __int128)1 << 32) ? 0xffffffffu : (uint32_t)t;
    }
    g_zipf_cdf[25] = 0xffffffffu;
    g_zipf_ready = 1;
}
static inline uint8_t zipf_letter(uint32_t r32) {
    int k = 0;
    while (k < 25 && r32 >= g_zipf_cdf[k]) k++;
    return (uint8_t)('a' + k);
}

/* One non-newline byte of the given alphabet. For FFBF_GEN_ZIPF_WORDS a space follows a run of
 * letters with probability 1/7 per position, i.e. after geometric(mean 6) letters. */
static inline uint8_t draw_byte(xo_t* r, int kind, int no_newline) {
    uint64_t x = xo_next(r);
    switch (kind) {
        case FFBF_GEN_PRINTABLE:
            return (uint8_t)(0x20 + below((uint32_t)x, 95));
        case FFBF_GEN_ZIPF_WORDS:
            if ((uint32_t)x < 613566757u) return ' ';  /* floor(2^32 / 7) */
            return zipf_letter((uint32_t)(x >> 32));
        default: {
            uint8_t b = (uint8_t)x;
            while (no_newline && b == '\n') b = (uint8_t)xo_next(r);
            return b;
        }
    }
}

/*
 * Pattern file image: n_patterns lines, each of length uniform in [len_lo, len_hi], each followed by '\n'.
 * Binary patterns never contain '\n' (it is redrawn) so that every pattern stays one line of the file.
 * out must hold n_patterns * (len_hi + 1) bytes. Returns the number of bytes written.
 */
size_t ffbf_gen_patterns(uint64_t seed, int kind, uint64_t n_patterns, uint32_t len_lo, uint32_t len_hi, uint8_t* out) {
    zipf_init();
    xo_t r;
    xo_seed(&r, seed, 1);
    size_t o = 0;
    for (uint64_t i = 0; i < n_patterns; i++) {
        uint32_t len = len_lo + below((uint32_t)(xo_next(&r) >> 32), len_hi - len_lo + 1);
        for (uint32_t j = 0; j < len; j++) out[o++] = draw_byte(&r, kind, 1);
        out[o++] = '\n';
    }
    return o;
}

typedef struct {
    uint64_t seed; int kind; uint32_t nl_thresh; uint8_t* out; size_t n; size_t b0, b1;
} text_job;

#define GEN_BLOCK (1u << 20)

static void* text_worker(void* arg) {
    text_job* j = (text_job*)arg;
    for (size_t b = j->b0; b < j->b1; b++) {
        xo_t r;
        xo_seed(&r, j->seed, 0x1000000ull + b);
        size_t lo = b * (size_t)GEN_BLOCK, hi = lo + GEN_BLOCK < j->n ? lo + GEN_BLOCK : j->n;
        for (size_t i = lo; i < hi; i++) {
            if (j->nl_thresh && (uint32_t)(xo_next(&r) >> 32) < j->nl_thresh) { j->out[i] = '\n'; continue; }
            j->out[i] = draw_byte(&r, j->kind, 0);
        }
    }
    return NULL;
}

/*
 * Text of n bytes. With newline_mean > 0 every byte is '\n' with probability 1/newline_mean (geometric
 * line lengths); binary text gets its newlines from the uniform byte draw only. Each 1 MiB block has its
 * own stream, so the result does not depend on nthreads.
 */
int ffbf_gen_text(uint64_t seed, int kind, uint32_t newline_mean, uint8_t* out, size_t n, int nthreads) {
    zipf_init();
    uint32_t thresh = newline_mean ? (uint32_t)(0x100000000ull / newline_mean) : 0;
    size_t nblocks = (n + GEN_BLOCK - 1) / GEN_BLOCK;
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > nblocks) nthreads = nblocks ? (int)nblocks : 1;
    text_job jobs[64];
    pthread_t th[64];
    if (nthreads > 64) nthreads = 64;
    for (int t = 0; t < nthreads; t++) {
        jobs[t].seed = seed; jobs[t].kind = kind; jobs[t].nl_thresh = thresh; jobs[t].out = out; jobs[t].n = n;
        jobs[t].b0 = nblocks * t / nthreads; jobs[t].b1 = nblocks * (t + 1) / nthreads;
    }
    for (int t = 1; t < nthreads; t++)
        if (pthread_create(&th[t], NULL, text_worker, &jobs[t])) return -1;
    text_worker(&jobs[0]);
    for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
    return 0;
}

/*
 * Plant n_plant occurrences: each picks a pattern line uniformly and an offset uniformly among the
 * positions where it fits, and copies the pattern's bytes over the text (later plants may overwrite
 * earlier ones). Writes the chosen (offset, pattern id) pairs when offs/ids are non-NULL.
 */
int ffbf_gen_plant(uint64_t seed, const uint8_t* pats, size_t plen, uint8_t* text, size_t n, uint64_t n_plant,
                   uint64_t* offs, uint64_t* ids) {
    size_t npat = 0;
    for (size_t i = 0; i < plen; i++) npat += pats[i] == '\n';
    if (plen && pats[plen - 1] != '\n') npat++;
    if (!npat || !n) return 0;
    size_t* st = (size_t*)malloc((npat + 1) * sizeof(size_t));
    if (!st) return -1;
    size_t k = 0;
    st[k++] = 0;
    for (size_t i = 0; i < plen; i++)
        if (pats[i] == '\n' && k <= npat) st[k++] = i + 1;
    if (k == npat) st[k] = plen + 1; /* no trailing newline: sentinel one past the end */
    xo_t r;
    xo_seed(&r, seed, 2);
    for (uint64_t p = 0; p < n_plant; p++) {
        uint64_t x = xo_next(&r);
        size_t id = (size_t)(((unsigned __int128)x * npat) >> 64);
        size_t len = st[id + 1] - st[id] - 1;
        if (len > n) continue;
        uint64_t y = xo_next(&r);
        size_t o = (size_t)(((unsigned __int128)y * (n - len + 1)) >> 64);
        memcpy(text + o, pats + st[id], len);
        if (offs) offs[p] = o;
        if (ids) ids[p] = id;
    }
    free(st);
    return 0;
}

/* A raw stream of 64-bit draws, for job sizes and arrival times that callers derive themselves. */
void ffbf_gen_u64(uint64_t seed, uint64_t stream, uint64_t* out, size_t n) {
    xo_t r;
    xo_seed(&r, seed, 0x2000000ull + stream);
    for (size_t i = 0; i < n; i++) out[i] = xo_next(&r);
}
