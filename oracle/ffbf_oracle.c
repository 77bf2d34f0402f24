/*
 * ffbf_oracle.c -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A plain-C restatement of efficient/ffbf's x86 rabin-karp path (src/rabin-karp/ffbf.cpp and
 * src/hashes/hash_rot_sbox_pre_2.h). Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg load it, and only as the checker. The product library (ffbf_b200/libffbf.so) never links it.
 *
 * Parity of this restatement is pinned against the reference binary itself: oracle/Makefile compiles
 * the reference's ffbf.cpp in place (oracle/_ref/), tests/golden/make_golden.py runs it on seeded
 * inputs, and tests/test_oracle_golden.py checks every artefact of this file against those outputs
 * (the __bloom_filter_* file, stdout, the pruned pattern file, the __index_* file and the FF bit array).
 *
 * Every function follows the reference loop for loop, including its output quirks, because the
 * product's outputs are compared with these byte for byte.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../ffbf_b200/csrc/ffbf_sbox.h"
#include <stdio.h>

static const uint64_t ORC_SBOX[256] = {FFBF_SBOX_WORDS};

typedef struct {
    int len;              /* LEN / DEF_PATT_LEN: window length, 1..63 */
    int k;                /* DEF_K: number of hash functions, 1..11 */
    int s;                /* DEF_S: how many of them index the cache region, 0..k */
    uint64_t cache_bits;  /* DEF_CACHE_SIZE: power of two */
    uint64_t ext_bits;    /* DEF_EXT_SIZE: power of two */
} orc_params;

/* ---- growable byte / u64 buffers ------------------------------------------------------------ */
typedef struct { uint8_t* p; size_t n, cap; } obuf;
typedef struct { uint64_t* p; size_t n, cap; } u64buf;

static int ob_put(obuf* b, const void* src, size_t n) {
    if (b->n + n + 1 > b->cap) {
        size_t c = b->cap ? b->cap : 4096;
        while (c < b->n + n + 1) c *= 2;
        uint8_t* q = (uint8_t*)realloc(b->p, c);
        if (!q) return -1;
        b->p = q; b->cap = c;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
    return 0;
}
/* `cout << (char*)s` prints up to the first NUL (ffbf.cpp:350,353,387). */
static int ob_put_cstr(obuf* b, const uint8_t* s, size_t maxlen) {
    const void* z = memchr(s, 0, maxlen);
    return ob_put(b, s, z ? (size_t)((const uint8_t*)z - s) : maxlen);
}
static int u64_put(u64buf* b, uint64_t v) {
    if (b->n + 1 > b->cap) {
        size_t c = b->cap ? b->cap * 2 : 1024;
        uint64_t* q = (uint64_t*)realloc(b->p, c * sizeof(uint64_t));
        if (!q) return -1;
        b->p = q; b->cap = c;
    }
    b->p[b->n++] = v;
    return 0;
}

/* ---- rolling hash: hash_rot_sbox_pre_2<LEN> (src/hashes/hash_rot_sbox_pre_2.h:8-57) --------- */
typedef struct {
    uint64_t h;
    uint64_t b[64];
    int bufptr, full, len;
} orc_hash;

static inline uint64_t rol64(uint64_t w, int s) { return (w << s) | (w >> (64 - s)); } /* hash_common.h:13-16 */

static void hash_reset(orc_hash* x) { /* :30-37 */
    x->h = 0; x->bufptr = 0; x->full = 0;
    memset(x->b, 0, sizeof(x->b));
}
/* Filter::updateHashes (ffbf.cpp:124-133) folded with hash_rot_sbox_pre_2::update (:42-51). */
static inline void hash_update(orc_hash* x, uint8_t c) {
    if (c & 0x80) c = 0;
    x->h = rol64(x->h, 1);
    x->h ^= ORC_SBOX[c];
    x->h ^= x->b[x->bufptr];
    x->b[x->bufptr++] = rol64(ORC_SBOX[c], x->len);
    if (x->bufptr >= x->len) { x->bufptr = 0; x->full = 1; }
}

uint64_t orc_window_hash(const uint8_t* w, int len) {
    orc_hash x; x.len = len; hash_reset(&x);
    for (int i = 0; i < len; i++) hash_update(&x, w[i]);
    return x.h;
}

/* ---- index functions: getHashValue (ffbf.cpp:135-159) and getHashValue_2 (:161-185) --------- */
static uint32_t fn(uint32_t h1, uint32_t h2, int f) {
    switch (f) {
        case 0: return h1;
        case 1: return h2;
        case 2: return (h1 << 16) | (h1 >> 16);
        case 3: return (h2 << 16) | (h2 >> 16);
        case 4: return h1 + h2;
        case 5: return h1 + (h2 << 1);
        case 6: return h1 + (h2 << 2);
        case 7: return h1 + 3 * h2;
        case 8: return h1 + 5 * h2;
        case 9: return h1 + 6 * h2;
        case 10: return h1 + 7 * h2;
    }
    return 0;
}
/* getHashValue_2 case i uses the formula that getHashValue uses at case MAP2[i]. */
static const int MAP2[11] = {5, 6, 7, 8, 9, 10, 0, 1, 2, 3, 4};

uint32_t orc_index(const orc_params* p, uint64_t h, int i, int order) {
    uint32_t h1 = (uint32_t)h, h2 = (uint32_t)(h >> 32);
    uint32_t x = fn(h1, h2, order == 2 ? MAP2[i] : i);
    if (i < p->s) return x & (uint32_t)(p->cache_bits - 1);
    return (x & (uint32_t)(p->ext_bits - 1)) + (uint32_t)p->cache_bits;
}

static inline void set_bit(uint8_t* v, uint32_t i) { v[i >> 3] |= (uint8_t)(1u << (i & 7)); } /* :187-193 */
static inline int get_bit(const uint8_t* v, uint32_t i) { return (v[i >> 3] >> (i & 7)) & 1; }

/* checkInFilter / checkInFilter_2 (:214-266): all K bits set; probe order does not change the answer. */
static int check(const orc_params* p, const uint8_t* v, uint64_t h, int order) {
    for (int i = 0; i < p->k; i++)
        if (!get_bit(v, orc_index(p, h, i, order))) return 0;
    return 1;
}
static void set_bits(const orc_params* p, uint8_t* v, uint64_t h, int order) { /* :195-211 */
    for (int i = 0; i < p->k; i++) set_bit(v, orc_index(p, h, i, order));
}

/* ---- filter build: main() getline loop (:556-571) + operator<< (:268-283) ------------------ */
long orc_build(const orc_params* p, const uint8_t* pats, size_t n, uint8_t* bv) {
    long inserted = 0;
    size_t i = 0;
    while (i < n) {
        const uint8_t* nl = (const uint8_t*)memchr(pats + i, '\n', n - i);
        size_t e = nl ? (size_t)(nl - pats) : n;
        if (e - i >= (size_t)p->len) {
            set_bits(p, bv, orc_window_hash(pats + i, p->len), 1);
            inserted++;
        }
        i = e + 1; /* getline: a final line without '\n' still counts; a trailing '\n' adds no empty line */
    }
    return inserted;
}

/* ---- scan: Filter::processFile (:310-392), read() chunk by chunk ---------------------------- */
typedef struct {
    uint8_t* out; size_t out_len;          /* bytes the reference writes to stdout */
    uint64_t* hits; size_t n_hits;         /* start offset of every window that hits, ascending */
    uint64_t* line_start; uint64_t* line_end; size_t n_lines; /* flagged lines, [start, end) without '\n' */
} orc_scan_result;

int orc_scan(const orc_params* p, const uint8_t* bv, uint8_t* ffbv, const uint8_t* text, size_t n,
             size_t chunk, orc_scan_result* r) {
    obuf out = {0}, line = {0};
    u64buf hits = {0}, ls = {0}, le = {0};
    orc_hash x; x.len = p->len; hash_reset(&x);
    int printLine = 0, flagged = 0;
    uint64_t abs_line_start = 0;
    uint8_t z = 0;
    if (ob_put(&line, &z, 0)) return -1;
    line.p[0] = 0;
    size_t pos = 0;
    while (pos < n) {
        size_t rr = n - pos < chunk ? n - pos : chunk;
        const uint8_t* buff = text + pos;
        size_t lineStart = 0;
        for (size_t i = 0; i < rr; i++) {
            if (buff[i] == '\n') {
                if (printLine) {
                    printLine = 0;
                    if (line.p[0] != 0) ob_put_cstr(&out, line.p, line.n);
                    ob_put_cstr(&out, buff + lineStart, i - lineStart);
                    ob_put(&out, "\n", 1);
                }
                if (flagged) { u64_put(&ls, abs_line_start); u64_put(&le, pos + i); flagged = 0; }
                line.n = 0; line.p[0] = 0;
                hash_reset(&x);
                lineStart = i + 1;
                abs_line_start = pos + i + 1;
                continue;
            }
            hash_update(&x, buff[i]);
            if (x.full && check(p, bv, x.h, 1)) {
                set_bits(p, ffbv, x.h, 2);
                printLine = 1;
                flagged = 1;
                u64_put(&hits, pos + i + 1 - (size_t)p->len);
            }
        }
        if (buff[rr - 1] != '\n') { /* carry buffer is replaced, not appended (:372-382) */
            line.n = 0;
            ob_put(&line, buff + lineStart, rr - lineStart);
            line.p[line.n] = 0;
        }
        pos += rr;
    }
    if (printLine) {
        ob_put_cstr(&out, line.p, line.n);
        ob_put(&out, "\n", 1);
    }
    if (flagged) { u64_put(&ls, abs_line_start); u64_put(&le, n); }
    free(line.p);
    r->out = out.p; r->out_len = out.n;
    r->hits = hits.p; r->n_hits = hits.n;
    r->line_start = ls.p; r->line_end = le.p; r->n_lines = ls.n;
    return 0;
}

/* ---- FF prune: Filter::filterPhrases (:394-485) ------------------------------------------- */
typedef struct {
    uint8_t* out; size_t out_len;   /* the pruned pattern file */
    uint8_t* idx; size_t idx_len;   /* the __index_ file: decimal line numbers, one per line */
    uint64_t* ids; size_t n_ids;    /* the same line numbers */
} orc_prune_result;

static void put_dec(obuf* b, uint64_t v) {
    char tmp[24]; int k = 0;
    do { tmp[k++] = (char)('0' + v % 10); v /= 10; } while (v);
    while (k) ob_put(b, &tmp[--k], 1);
    ob_put(b, "\n", 1);
}

int orc_prune(const orc_params* p, const uint8_t* ffbv, const uint8_t* pats, size_t n, size_t chunk,
              orc_prune_result* r) {
    obuf out = {0}, idx = {0}, line = {0};
    u64buf ids = {0};
    orc_hash x; x.len = p->len; hash_reset(&x);
    uint8_t z = 0;
    ob_put(&line, &z, 0); line.p[0] = 0;
    int printLine = 0, skipRest = 0;
    uint64_t lineNumber = 0;
    size_t pos = 0;
    while (pos < n) {
        size_t rr = n - pos < chunk ? n - pos : chunk;
        const uint8_t* buff = pats + pos;
        size_t lineStart = 0;
        for (size_t i = 0; i < rr; i++) {
            if (buff[i] == '\n') {
                skipRest = 0;
                if (printLine) {
                    printLine = 0;
                    if (line.p[0] != 0) ob_put_cstr(&out, line.p, line.n);
                    ob_put_cstr(&out, buff + lineStart, i - lineStart);
                    ob_put(&out, "\n", 1);
                    put_dec(&idx, lineNumber);
                    u64_put(&ids, lineNumber);
                }
                line.n = 0; line.p[0] = 0;
                hash_reset(&x);
                lineStart = i + 1;
                lineNumber++;
                continue;
            }
            if (printLine || skipRest) continue;
            hash_update(&x, buff[i]);
            if (x.full) {
                if (check(p, ffbv, x.h, 2)) printLine = 1;
                skipRest = 1;
            }
        }
        if (buff[rr - 1] != '\n') {
            line.n = 0;
            ob_put(&line, buff + lineStart, rr - lineStart);
            line.p[line.n] = 0;
        }
        pos += rr;
    }
    if (printLine) {
        ob_put_cstr(&out, line.p, line.n);
        ob_put(&out, "\n", 1);
        put_dec(&idx, lineNumber);
        u64_put(&ids, lineNumber);
    }
    free(line.p);
    r->out = out.p; r->out_len = out.n;
    r->idx = idx.p; r->idx_len = idx.n;
    r->ids = ids.p; r->n_ids = ids.n;
    return 0;
}

/* ---- operator[] (:285-308): first hitting window of one string, no newline handling --------- */
int orc_test_line(const orc_params* p, const uint8_t* bv, const uint8_t* s, size_t n) {
    if (n < (size_t)p->len) return 0;
    orc_hash x; x.len = p->len; hash_reset(&x);
    for (size_t i = 0; i < n; i++) {
        hash_update(&x, s[i]);
        if (x.full && check(p, bv, x.h, 1)) return 1;
    }
    return 0;
}

/* ---- filter cache file: saveFilterToFile (:508-527) / loadFilterFromFile (:487-506) -------- */
int orc_save_filter(const orc_params* p, const uint8_t* bv, uint8_t** out, size_t* out_len) {
    obuf b = {0};
    uint32_t prev = 0;
    uint64_t nbits = p->cache_bits + p->ext_bits;
    for (uint64_t i = 0; i < nbits; i++) {
        if (get_bit(bv, (uint32_t)i)) {
            uint32_t delta = (uint32_t)i - prev;
            prev = (uint32_t)i;
            if (ob_put(&b, &delta, 4)) return -1;
        }
    }
    *out = b.p; *out_len = b.n;
    return 0;
}

/* Returns 0, or -1 when a decoded index falls outside the main filter (the reference would write
 * past its bit array there). A trailing partial word is ignored, as the reference's nr/4 does. */
int orc_load_filter(const orc_params* p, const uint8_t* file, size_t len, uint8_t* bv) {
    uint32_t prev = 0;
    uint64_t nbits = p->cache_bits + p->ext_bits;
    for (size_t i = 0; i + 4 <= len; i += 4) {
        uint32_t d;
        memcpy(&d, file + i, 4);
        prev += d;
        if (prev >= nbits) return -1;
        set_bit(bv, prev);
    }
    return 0;
}

/* ---- exact verification (the `grep -Ff pruned candidates` stage, src/rabin-karp/README:49-52) --
 * For every hit window start w and every pruned pattern q (length >= LEN), report (w, q) when the
 * text holds q's bytes at w. Output is sorted by (offset, pattern id). The prefix table is keyed by
 * the raw LEN prefix bytes, not by the rolling hash, so this check is independent of the hash. */
typedef struct { uint64_t* off; uint64_t* pid; size_t n; } orc_matches;

static uint64_t fnv(const uint8_t* s, int n) {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < n; i++) { h ^= s[i]; h *= 1099511628211ull; }
    return h;
}

int orc_verify(const orc_params* p, const uint8_t* pats, size_t plen, const uint64_t* ids, size_t n_ids,
               const uint8_t* text, size_t n, const uint64_t* hits, size_t n_hits, orc_matches* m) {
    const int L = p->len;
    /* line table of the pattern file */
    u64buf st = {0}, en = {0};
    size_t i = 0;
    while (i < plen) {
        const uint8_t* nl = (const uint8_t*)memchr(pats + i, '\n', plen - i);
        size_t e = nl ? (size_t)(nl - pats) : plen;
        u64_put(&st, i); u64_put(&en, e);
        i = e + 1;
    }
    size_t cap = 1; while (cap < 2 * n_ids + 2) cap <<= 1;
    int64_t* head = (int64_t*)malloc(cap * sizeof(int64_t));
    int64_t* next = (int64_t*)malloc((n_ids + 1) * sizeof(int64_t));
    if (!head || !next) return -1;
    for (size_t k = 0; k < cap; k++) head[k] = -1;
    for (size_t k = 0; k < n_ids; k++) {
        uint64_t id = ids[k];
        if (id >= st.n || en.p[id] - st.p[id] < (uint64_t)L) continue;
        size_t slot = fnv(pats + st.p[id], L) & (cap - 1);
        next[k] = head[slot]; head[slot] = (int64_t)k;
    }
    u64buf off = {0}, pid = {0};
    for (size_t h = 0; h < n_hits; h++) {
        uint64_t w = hits[h];
        if (w + L > n) continue;
        size_t slot = fnv(text + w, L) & (cap - 1);
        /* collect matches for this window, then emit in ascending id order */
        size_t first = pid.n;
        for (int64_t k = head[slot]; k >= 0; k = next[k]) {
            uint64_t id = ids[k];
            uint64_t ql = en.p[id] - st.p[id];
            if (w + ql > n) continue;
            if (memcmp(text + w, pats + st.p[id], ql) == 0) { u64_put(&off, w); u64_put(&pid, id); }
        }
        /* insertion sort of the few ids just added */
        for (size_t a = first + 1; a < pid.n; a++)
            for (size_t b = a; b > first && pid.p[b - 1] > pid.p[b]; b--) {
                uint64_t t = pid.p[b]; pid.p[b] = pid.p[b - 1]; pid.p[b - 1] = t;
            }
    }
    free(head); free(next); free(st.p); free(en.p);
    m->off = off.p; m->pid = pid.p; m->n = off.n;
    return 0;
}

/* ---- hashbench (src/hashes/hashbench.cc), HashTester<hash_rot_sbox_pre_2<19>, 19> -------------- */

/* hash_rot_sbox_pre_2::update (:42-51) on the raw byte: hashbench does not map bytes >= 0x80. */
static inline void hash_update_raw(orc_hash* x, uint8_t c) {
    x->h = rol64(x->h, 1);
    x->h ^= ORC_SBOX[c];
    x->h ^= x->b[x->bufptr];
    x->b[x->bufptr++] = rol64(ORC_SBOX[c], x->len);
    if (x->bufptr >= x->len) { x->bufptr = 0; x->full = 1; }
}

/* hash_lines (hashbench.cc:108-127): fgets(buf, 4095, f) returns a line with its '\n', or the next 4094
 * bytes of a longer line; per piece the hash is reset, every byte up to the first NUL is hashed except the
 * '\n' (which becomes the string's end), and "%x %s\n" prints hval() = h >> 32 and the string.
 * Writes the printed bytes to *out (malloc'd) and returns their count, or -1 on allocation failure. */
long orc_hashbench_lines(const uint8_t* text, size_t n, uint8_t** out) {
    size_t cap = n * 2 + 64, o = 0;
    uint8_t* buf = (uint8_t*)malloc(cap);
    if (!buf) return -1;
    for (size_t pos = 0; pos < n;) {
        size_t m = 0; /* fgets: up to 4094 bytes, through the first '\n' */
        while (m < 4094 && pos + m < n) {
            m++;
            if (text[pos + m - 1] == '\n') break;
        }
        orc_hash x; x.len = 19; hash_reset(&x);
        size_t e = 0; /* the C string: up to the first NUL or '\n' */
        while (e < m && text[pos + e] != 0 && text[pos + e] != '\n') hash_update_raw(&x, text[pos + e++]);
        if (o + e + 16 > cap) {
            cap = (o + e + 16) * 2;
            uint8_t* nb = (uint8_t*)realloc(buf, cap);
            if (!nb) { free(buf); return -1; }
            buf = nb;
        }
        o += (size_t)sprintf((char*)buf + o, "%x ", (uint32_t)(x.h >> 32));
        memcpy(buf + o, text + pos, e);
        o += e;
        buf[o++] = '\n';
        pos += m;
    }
    *out = buf;
    return (long)o;
}

/* hash_file (hashbench.cc:60-99) hashes every byte with no reset and prints only the byte count and the
 * time; as a checkable result, the XOR of the 64-bit hash after every byte. */
uint64_t orc_hash_xor(const uint8_t* text, size_t n, int len) {
    orc_hash x; x.len = len; hash_reset(&x);
    uint64_t acc = 0;
    for (size_t i = 0; i < n; i++) {
        hash_update_raw(&x, text[i]);
        acc ^= x.h;
    }
    return acc;
}

void orc_free(void* ptr) { free(ptr); }
