// hashbench_cli.cpp -- drop-in for the reference's hash benchmark CLI (src/hashes/hashbench.cc:19-196),
// built for the scan's hash, hash_rot_sbox_pre_2<19>, with the hashing on GPU 0 (ffbf_hashbench_* in
// include/ffbf.h).
//
//   hashbench [-fl] <input file>     ("-" reads stdin)
//     -l   print each line's final hash (default): the same bytes the reference prints
//     -f   hash the whole file silently, print time: the reference's header and "<bytes> <seconds>", where
//          the seconds are the device's hashing time (the reference times its read() loop)
#include <getopt.h>
#include <sys/param.h>
#include <sys/time.h>
#include <time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ffbf.h"

namespace {

void usage() { fprintf(stderr, "hashbench [-fl] <input file>\n"); }

void help() {
    usage();
    fprintf(stderr,
            "  -l   print each line's final hash (default)\n"
            "  -f   hash the whole file silently, print time\n");
}

bool read_all(const char* path, std::vector<uint8_t>& out) {
    FILE* f = strcmp(path, "-") ? fopen(path, "rb") : stdin;
    if (!f) return false;
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) out.insert(out.end(), buf, buf + n);
    if (f != stdin) fclose(f);
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    const int orig_argc = argc;
    char** orig_argv = argv;
    bool file_mode = false;
    int ch;
    while ((ch = getopt(argc, argv, "hfl")) != -1) {
        switch (ch) {
            case 'h': help(); exit(0);
            case 'l': file_mode = false; break;
            case 'f': file_mode = true; break;
            default: usage(); exit(-1);
        }
    }
    argc -= optind;
    argv += optind;
    if (argc < 1) {
        usage();
        exit(-1);
    }
    std::vector<uint8_t> text;
    if (!read_all(argv[0], text)) {
        perror(argv[0]);
        exit(-1);
    }
    if (!file_mode) {
        uint8_t* out = nullptr;
        size_t out_len = 0;
        ffbf_status s = ffbf_hashbench_lines(0, text.data(), text.size(), &out, &out_len);
        if (s != FFBF_OK) {
            fprintf(stderr, "hashbench: %s\n", ffbf_status_string(s));
            exit(-1);
        }
        fwrite(out, 1, out_len, stdout);
        ffbf_free(out);
        return 0;
    }
    struct timeval tv_start;
    gettimeofday(&tv_start, nullptr);
    uint64_t x = 0;
    double secs = 0;
    ffbf_status s = ffbf_hashbench_file(0, text.data(), text.size(), &x, &secs);
    if (s != FFBF_OK) {
        fprintf(stderr, "hashbench: %s\n", ffbf_status_string(s));
        exit(-1);
    }
    // the reference's report (hashbench.cc:82-98)
    char tfmtbuf[32];
    char curpath[MAXPATHLEN + 1];
    if (!getcwd(curpath, MAXPATHLEN)) curpath[0] = 0;
    ctime_r(&tv_start.tv_sec, tfmtbuf);
    printf("# hashbench.c %s", tfmtbuf);
    printf("# hashfn: %s\n", "hash_rot_sbox_pre_2");
    printf("# input file: %s\n", argv[0]);
    printf("# command line: ");
    for (int i = 0; i < orig_argc; i++) printf(" %s", orig_argv[i]);
    printf("\n");
    const char* user = getlogin();
    printf("# user: %s\n", user ? user : "(null)");
    printf("# path: %s\n", curpath);
    printf("#\n");
    printf("# bytes     execution time (seconds)\n");
    printf("%lld %.3f\n", (long long)text.size(), secs);
    return 0;
}
