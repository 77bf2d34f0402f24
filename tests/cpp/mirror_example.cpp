// A program written the way the reference's main (src/rabin-karp/ffbf.cpp:529-601) drives Filter<H,LEN>, built
// against the C++ mirror (include/ffbf.hpp): patterns go in with operator<<, the text is scanned with
// processFile(0) (candidate lines to stdout), and filterPhrases writes the pruned patterns and their indexes.
// With the argument "server", the same text is also scanned as one request through ffbf::Server and the
// hit count is printed to stderr beside the direct scan's.
//
//   mirror_example <len> <patterns> <pruned_out> [server] < text > candidate_lines
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "ffbf.hpp"

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <len> <patterns> <pruned_out> [server]\n", argv[0]);
        return 2;
    }
    try {
        ffbf_params p;
        ffbf_params_default(&p);
        p.len = (uint32_t)atoi(argv[1]);
        ffbf::Filter filter(&p);
        std::ifstream pats(argv[2]);
        std::string line;
        while (std::getline(pats, line)) filter << line;
        std::vector<uint8_t> text;
        if (argc > 4 && !strcmp(argv[4], "server")) {
            // read the text once for the server request, then scan it through processFile from a copy
            char buf[1 << 16];
            ssize_t r;
            while ((r = read(0, buf, sizeof buf)) > 0) text.insert(text.end(), buf, buf + r);
            {
                ffbf::Filter set(&p);
                std::ifstream pats2(argv[2]);
                while (std::getline(pats2, line)) set << line;
                ffbf::Server server(0, 64 << 20, 4);
                const uint32_t sid = server.add_set(set);
                const uint64_t rid = server.submit(sid, text.data(), text.size());
                std::vector<ffbf_request_result> got;
                while (got.empty()) got = server.poll(4, 100000);
                fprintf(stderr, "server request %llu: status %d, %llu hits\n", (unsigned long long)rid,
                        (int)got[0].status, (unsigned long long)got[0].n_hits);
                server.release(got[0].request_id);
            }
            char tmpl[] = "/tmp/mirror_textXXXXXX";
            int fd = mkstemp(tmpl);
            if (fd < 0 || write(fd, text.data(), text.size()) != (ssize_t)text.size()) return 3;
            lseek(fd, 0, SEEK_SET);
            dup2(fd, 0);
            close(fd);
            unlink(tmpl);
        }
        filter.processFile(0);
        ffbf_scan_result r = filter.collect();
        fprintf(stderr, "direct scan: %llu hits\n", (unsigned long long)r.n_hits);
        const ffbf::Filter::ScanConfig sc = filter.scanConfig();
        fprintf(stderr, "scan config: %d threads, mode %d, probe order %d\n", sc.threads, sc.mode, sc.order);
        std::ofstream out(argv[3]), idx(std::string("__index_") + argv[3]);
        int pfd = open(argv[2], O_RDONLY);
        filter.filterPhrases(pfd, out, idx);
        close(pfd);
    } catch (const ffbf::FilterError& e) {
        fprintf(stderr, "FilterError: %s\n", e.what());
        return 1;
    }
    return 0;
}
