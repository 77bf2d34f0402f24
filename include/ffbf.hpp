// ffbf.hpp -- C++ mirror of efficient/ffbf's Filter<H, LEN> (src/rabin-karp/ffbf.h:43-93) over the C ABI.
//
// A program written against the reference class switches by replacing
//     #include "ffbf.h"                                   (src/rabin-karp/ffbf.h)
//     Filter<hash_rot_sbox_pre_2<DEF_PATT_LEN>, DEF_PATT_LEN> filter;
// with
//     #include "ffbf.hpp"                                 (this file; link with -lffbf)
//     ffbf::Filter filter;                                (or ffbf::Filter filter(params, device))
// and keeps its calls: `filter << phrase`, `filter[line]`, processFile(fd), filterPhrases(pfd, out, outIndex),
// loadFilterFromFile(fd), saveFilterToFile(fd). Errors are thrown as FilterError (ffbf.h:31-41), whose what()
// carries the library's message. The geometry defaults to the reference's compile-time defaults.
//
// Differences, all documented in include/ffbf.h: the filter lives on a CUDA device; `filter << phrase` buffers
// patterns and the device build runs once, before the first operation that needs the filter; processFile
// reads the whole stream before scanning it.
#ifndef FFBF_B200_FFBF_HPP
#define FFBF_B200_FFBF_HPP

#include <unistd.h>

#include <fstream>
#include <string>
#include <vector>

#include "ffbf.h"

namespace ffbf {

class FilterError {
    std::string message;

public:
    explicit FilterError(const std::string& msg = "") : message(msg) {}
    const char* what() const { return message.c_str(); }
};

class Filter {
public:
    explicit Filter(const ffbf_params* p = nullptr, int device = 0) {
        ffbf_params d;
        ffbf_params_default(&d);
        ffbf_status s = ffbf_create(p ? p : &d, device, &ctx_);
        if (s != FFBF_OK) throw FilterError(std::string("Not able to initialize filter: ") + ffbf_status_string(s));
    }
    ~Filter() { ffbf_destroy(ctx_); }
    Filter(const Filter&) = delete;
    Filter& operator=(const Filter&) = delete;

    // operator<< (ffbf.cpp:268-283): queue one pattern line; lines shorter than LEN are ignored at build time.
    Filter& operator<<(const std::string& pattern) {
        pending_.insert(pending_.end(), pattern.begin(), pattern.end());
        pending_.push_back('\n');
        dirty_ = true;
        return *this;
    }

    // operator[] (ffbf.cpp:285-308): does some window of `line` hit the main filter?
    bool operator[](const std::string& line) {
        flush();
        int hit = 0;
        check(ffbf_test_line(ctx_, reinterpret_cast<const uint8_t*>(line.data()), line.size(), &hit));
        return hit != 0;
    }

    // processFile (ffbf.cpp:310-392): reads fd to its end, scans it, writes the candidate lines to stdout
    // with the reference's output rules (512 KiB read() chunks of a regular file).
    void processFile(int fd) {
        flush();
        std::vector<uint8_t> text;
        std::vector<uint8_t> buf(1 << 20);
        for (;;) {
            ssize_t r = ::read(fd, buf.data(), buf.size());
            if (r < 0) throw FilterError("Error while reading from file");
            if (r == 0) break;
            text.insert(text.end(), buf.begin(), buf.begin() + r);
        }
        ffbf_scan_result res;
        check(ffbf_scan(ctx_, text.data(), text.size(), &res));
        uint8_t* out = nullptr;
        size_t n = 0;
        check(ffbf_format_lines(ctx_, text.data(), text.size(), 512 * 1024, &out, &n));
        size_t off = 0;
        while (off < n) {
            ssize_t w = ::write(1, out + off, n - off);
            if (w <= 0) break;
            off += (size_t)w;
        }
        ffbf_free(out);
    }

    // filterPhrases (ffbf.cpp:394-485): re-reads the pattern file from pfd, writes the surviving lines to
    // `out` and their 0-based line numbers to `outIndex`.
    void filterPhrases(int pfd, std::ofstream& out, std::ofstream& outIndex) {
        flush();
        std::vector<uint8_t> pats;
        std::vector<uint8_t> buf(1 << 20);
        for (;;) {
            ssize_t r = ::read(pfd, buf.data(), buf.size());
            if (r < 0) throw FilterError("Error while reading from file");
            if (r == 0) break;
            pats.insert(pats.end(), buf.begin(), buf.begin() + r);
        }
        check(ffbf_set_patterns(ctx_, pats.data(), pats.size()));
        ffbf_prune_result pr;
        check(ffbf_prune(ctx_, &pr));
        uint8_t *o = nullptr, *ix = nullptr;
        size_t on = 0, in = 0;
        check(ffbf_format_pruned(ctx_, 512 * 1024, &o, &on, &ix, &in));
        out.write(reinterpret_cast<const char*>(o), (std::streamsize)on);
        outIndex.write(reinterpret_cast<const char*>(ix), (std::streamsize)in);
        ffbf_free(o);
        ffbf_free(ix);
    }

    // loadFilterFromFile / saveFilterToFile (ffbf.cpp:487-527): the __bloom_filter_ delta format.
    void loadFilterFromFile(int fd) {
        std::vector<uint8_t> data;
        std::vector<uint8_t> buf(1 << 20);
        for (;;) {
            ssize_t r = ::read(fd, buf.data(), buf.size());
            if (r < 0) throw FilterError("Error while reading from the filter file");
            if (r == 0) break;
            data.insert(data.end(), buf.begin(), buf.begin() + r);
        }
        check(ffbf_load_filter(ctx_, data.data(), data.size()));
    }

    void saveFilterToFile(int fd) {
        flush();
        uint8_t* data = nullptr;
        size_t n = 0;
        check(ffbf_save_filter(ctx_, &data, &n));
        size_t off = 0;
        while (off < n) {
            ssize_t w = ::write(fd, data + off, n - off);
            if (w < 0) {
                ffbf_free(data);
                throw FilterError("Error while writing to the filter file");
            }
            off += (size_t)w;
        }
        ffbf_free(data);
    }

    ffbf_ctx* handle() { return ctx_; }

    // The tuned scan's configuration as the filter's fills or ffbf_autotune chose it: CTA threads, mode (0
    // shared-memory stage, 1 pipelined L2 probes, 2 shared-memory stage with deferred candidates, 3 shared-memory
    // stage with per-stage barriers) and the
    // dense mode's probe order (0, 1 or 2).
    struct ScanConfig {
        int threads, mode, order;
    };
    ScanConfig scanConfig() {
        ScanConfig c{0, 0, 0};
        check(ffbf_get_scan_config(ctx_, &c.threads, &c.mode));
        check(ffbf_get_probe_order(ctx_, &c.order));
        return c;
    }

    // The context with every queued pattern built into its filter, for the batch and server wrappers below.
    ffbf_ctx* built_handle() {
        flush();
        return ctx_;
    }

    // The results of the last scan of this filter's context (a batch job's, once the batch is waited for).
    ffbf_scan_result collect() {
        ffbf_scan_result r;
        check(ffbf_scan_collect(ctx_, &r));
        return r;
    }

private:
    void check(ffbf_status s) {
        if (s != FFBF_OK) throw FilterError(std::string(ffbf_status_string(s)) + ": " + ffbf_last_error(ctx_));
    }
    // Builds the queued patterns into the main filter (the reference sets bits inside operator<<).
    void flush() {
        if (!dirty_) return;
        check(ffbf_set_patterns(ctx_, pending_.data(), pending_.size()));
        check(ffbf_build(ctx_));
        dirty_ = false;
    }

    ffbf_ctx* ctx_ = nullptr;
    std::vector<uint8_t> pending_;
    bool dirty_ = false;
};

// Many (filter, device text) jobs scanned in one graph launch (ffbf_batch_* in ffbf.h). The reference has no
// counterpart; each job's results come from its filter's collect() after wait().
class Batch {
public:
    explicit Batch(int device = 0) {
        ffbf_status s = ffbf_batch_create(device, &b_);
        if (s != FFBF_OK) throw FilterError(std::string("Not able to create a batch: ") + ffbf_status_string(s));
    }
    ~Batch() { ffbf_batch_destroy(b_); }
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    void add(Filter& f, const uint8_t* d_text, size_t len) { check(ffbf_batch_add(b_, f.built_handle(), d_text, len)); }
    uint32_t autotune(size_t sample_bytes = 0) {
        uint32_t n = 0;
        check(ffbf_batch_autotune(b_, sample_bytes, &n));
        return n;
    }
    void launch() { check(ffbf_batch_launch(b_)); }
    void wait() { check(ffbf_batch_wait(b_)); }

private:
    void check(ffbf_status s) {
        if (s != FFBF_OK) throw FilterError(std::string(ffbf_status_string(s)) + ": " + ffbf_batch_last_error(b_));
    }
    ffbf_batch* b_ = nullptr;
};

// Resident pattern sets and a request loop with continuous batching (ffbf_server_* in ffbf.h). No counterpart
// in the reference. Register the filters before the first submit; a result's arrays stay valid until
// release(request_id).
class Server {
public:
    explicit Server(int device = 0, uint64_t arena_bytes = 0, uint32_t slots = 0) {
        ffbf_status s = ffbf_server_create(device, arena_bytes, slots, &s_);
        if (s != FFBF_OK) throw FilterError(std::string("Not able to create a server: ") + ffbf_status_string(s));
    }
    ~Server() { ffbf_server_destroy(s_); }
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    uint32_t add_set(Filter& f) {
        uint32_t id = 0;
        check(ffbf_server_add_set(s_, f.built_handle(), &id));
        return id;
    }
    uint64_t submit(uint32_t set, const uint8_t* text, size_t len) {
        uint64_t id = 0;
        check(ffbf_server_submit(s_, set, text, len, &id));
        return id;
    }
    std::vector<ffbf_request_result> poll(uint32_t max = 64, uint32_t wait_us = 0) {
        std::vector<ffbf_request_result> out(max);
        uint32_t n = 0;
        check(ffbf_server_poll(s_, out.data(), max, &n, wait_us));
        out.resize(n);
        return out;
    }
    void release(uint64_t request_id) { check(ffbf_server_release(s_, request_id)); }

private:
    void check(ffbf_status s) {
        if (s != FFBF_OK) throw FilterError(std::string(ffbf_status_string(s)) + ": " + ffbf_server_last_error(s_));
    }
    ffbf_server* s_ = nullptr;
};

}  // namespace ffbf

#endif  // FFBF_B200_FFBF_HPP
