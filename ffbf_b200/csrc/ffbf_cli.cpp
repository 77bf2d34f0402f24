// ffbf_cli.cpp -- the `ffbf` command, a drop-in for efficient/ffbf's CLI (src/rabin-karp/ffbf.cpp:529-601).
//
//   ffbf [options] patterns_file filtered_patterns_out < corpus > candidate_lines
//
// Same positional arguments, files and streams as the reference:
//  * the main filter is loaded from ./__bloom_filter_<patterns_file> when that file opens, otherwise built
//    from the patterns and saved there (ffbf.cpp:545-575);
//  * candidate lines go to stdout, the pruned patterns to <filtered_patterns_out>, their 0-based line numbers
//    to ./__index_<filtered_patterns_out> (ffbf.cpp:537-540);
//  * "processFile time: %.5f" and "filterPhrases time: %.5f" (and "filter load time: %.5f") go to stderr
//    (ffbf.cpp:37-51, 551, 586-587);
//  * wrong argument count prints the usage line and returns -1 (ffbf.cpp:531-535).
// The filter geometry, compile-time in the reference (src/rabin-karp/Makefile.am:1-21), comes from options
// with the reference's defaults. --exact additionally runs verification and prints the lines that hold an
// exact pattern occurrence (what `grep -Ff filtered_patterns_out candidate_lines` prints) instead of the
// candidate lines.
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ffbf.h"

namespace {

double now() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + (double)tv.tv_usec / 1e6;
}

bool read_fd(int fd, std::vector<uint8_t>& out) {
    out.clear();
    std::vector<uint8_t> buf(1 << 20);
    for (;;) {
        ssize_t r = read(fd, buf.data(), buf.size());
        if (r < 0) return false;
        if (r == 0) return true;
        out.insert(out.end(), buf.begin(), buf.begin() + r);
    }
}

// A text buffer: page-locked (from the library) when stdin is a regular file of known size, so that the scan's
// copy to the device runs at full speed and overlaps the scan; a growing vector otherwise (pipes).
struct TextBuf {
    uint8_t* pinned = nullptr;
    size_t n = 0;
    std::vector<uint8_t> vec;
    const uint8_t* data() const { return pinned ? pinned : vec.data(); }
    size_t size() const { return pinned ? n : vec.size(); }
    ~TextBuf() {
        if (pinned) ffbf_host_free(pinned);
    }
};

bool read_stdin(TextBuf& t) {
    struct stat st;
    if (fstat(0, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
        const off_t here = lseek(0, 0, SEEK_CUR);
        const size_t want = (size_t)(st.st_size - (here > 0 ? here : 0));
        t.pinned = (uint8_t*)ffbf_host_alloc(want ? want : 1);
        if (t.pinned) {
            size_t got = 0;
            while (got < want) {
                ssize_t r = read(0, t.pinned + got, want - got);
                if (r < 0) return false;
                if (r == 0) break;
                got += (size_t)r;
            }
            t.n = got;
            return true;
        }
    }
    return read_fd(0, t.vec);
}

bool read_file(const char* path, std::vector<uint8_t>& out) {
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    out.clear();
    std::vector<uint8_t> buf(1 << 20);
    size_t r;
    while ((r = fread(buf.data(), 1, buf.size(), f)) > 0) out.insert(out.end(), buf.begin(), buf.begin() + r);
    bool ok = !ferror(f);
    fclose(f);
    return ok;
}

bool write_all(FILE* f, const uint8_t* p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }

void usage() {
    fprintf(stderr,
            "Usage: ffbf phrases phrases.out < corpus > filtered_corpus\n"
            "options: --len N --k N --s N --cache-bits N --ext-bits N --device N --chunk N --exact\n");
}

int die(ffbf_ctx* c, ffbf_status s, const char* what) {
    fprintf(stderr, "Exception %s: %s (%s)\n", what, ffbf_status_string(s), c ? ffbf_last_error(c) : "");
    return -1;
}

}  // namespace

int main(int argc, char** argv) {
    ffbf_params prm;
    ffbf_params_default(&prm);
    int device = 0, exact = 0;
    size_t chunk = 512 * 1024;
    std::vector<const char*> pos;
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        auto num = [&](unsigned long long& v) {
            if (i + 1 >= argc) return false;
            char* end = nullptr;
            v = strtoull(argv[++i], &end, 0);
            return end && *end == 0;
        };
        unsigned long long v = 0;
        if (!strcmp(a, "--exact")) exact = 1;
        else if (!strcmp(a, "--len") && num(v)) prm.len = (uint32_t)v;
        else if (!strcmp(a, "--k") && num(v)) prm.k = (uint32_t)v;
        else if (!strcmp(a, "--s") && num(v)) prm.s = (uint32_t)v;
        else if (!strcmp(a, "--cache-bits") && num(v)) prm.cache_bits = v;
        else if (!strcmp(a, "--ext-bits") && num(v)) prm.ext_bits = v;
        else if (!strcmp(a, "--device") && num(v)) device = (int)v;
        else if (!strcmp(a, "--chunk") && num(v) && v > 0) chunk = (size_t)v;
        else if (a[0] == '-' && a[1] == '-') {
            usage();
            return -1;
        } else pos.push_back(a);
    }
    if (pos.size() != 2) {
        usage();
        return -1;
    }
    const std::string patterns_path = pos[0], out_path = pos[1];
    const std::string index_path = "__index_" + out_path;
    const std::string cache_path = "__bloom_filter_" + patterns_path;

    FILE* out_f = fopen(out_path.c_str(), "wb");
    FILE* idx_f = fopen(index_path.c_str(), "wb");

    ffbf_ctx* c = nullptr;
    ffbf_status s = ffbf_create(&prm, device, &c);
    if (s != FFBF_OK) {
        fprintf(stderr, "Not able to initialize filter: %s\n", ffbf_status_string(s));
        return -1;
    }
    std::vector<uint8_t> pats;
    const bool have_pats = read_file(patterns_path.c_str(), pats);
    if (!have_pats) pats.clear();
    // The pattern lines are needed by the prune either way; the main filter comes from the cache if present.
    if ((s = ffbf_set_patterns(c, pats.data(), pats.size())) != FFBF_OK) return die(c, s, "while reading patterns");
    struct stat sb;
    if (stat(cache_path.c_str(), &sb) == 0) {
        double t0 = now();
        s = ffbf_load_filter_file(c, cache_path.c_str());
        fprintf(stderr, "filter load time: %.5f\n", now() - t0);
        if (s != FFBF_OK) return die(c, s, "while loading the filter");
    } else {
        if ((s = ffbf_build(c)) != FFBF_OK) return die(c, s, "while building the filter");
        if ((s = ffbf_save_filter_file(c, cache_path.c_str())) != FFBF_OK) return die(c, s, "while saving the filter");
    }
    if (!have_pats) {
        perror("Error while trying to open the phrases file");
        ffbf_destroy(c);
        return -1;
    }

    TextBuf text;
    double t0 = now();
    if (!read_stdin(text)) {
        perror("Error");
        return die(c, FFBF_EIO, "Error while reading from file");
    }
    ffbf_scan_result res;
    if ((s = ffbf_scan(c, text.data(), text.size(), &res)) != FFBF_OK) return die(c, s, "during the scan");
    if (!exact) {
        uint8_t* lines = nullptr;
        size_t nl = 0;
        if ((s = ffbf_format_lines(c, text.data(), text.size(), chunk, &lines, &nl)) != FFBF_OK)
            return die(c, s, "while formatting lines");
        write_all(stdout, lines, nl);
        ffbf_free(lines);
    }
    fflush(stdout);
    fprintf(stderr, "processFile time: %.5f\n", now() - t0);

    t0 = now();
    ffbf_prune_result pr;
    if ((s = ffbf_prune(c, &pr)) != FFBF_OK) return die(c, s, "during the prune");
    uint8_t *po = nullptr, *pi = nullptr;
    size_t pon = 0, pin = 0;
    if ((s = ffbf_format_pruned(c, chunk, &po, &pon, &pi, &pin)) != FFBF_OK) return die(c, s, "while writing patterns");
    if (out_f) write_all(out_f, po, pon);
    if (idx_f) write_all(idx_f, pi, pin);
    ffbf_free(po);
    ffbf_free(pi);
    fprintf(stderr, "filterPhrases time: %.5f\n", now() - t0);

    if (exact) {
        ffbf_matches m;
        if ((s = ffbf_verify(c, &m)) != FFBF_OK) return die(c, s, "during verification");
        // lines holding at least one exact occurrence, in text order, printed whole
        uint64_t j = 0;
        for (uint64_t i = 0; i < res.n_lines && j < m.n; i++) {
            while (j < m.n && m.offsets[j] < res.line_start[i]) j++;
            if (j < m.n && m.offsets[j] < res.line_end[i]) {
                write_all(stdout, text.data() + res.line_start[i], res.line_end[i] - res.line_start[i]);
                fputc('\n', stdout);
            }
        }
        fflush(stdout);
    }
    if (out_f) fclose(out_f);
    if (idx_f) fclose(idx_f);
    ffbf_destroy(c);
    return 0;
}
