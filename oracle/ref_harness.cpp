// ref_harness.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
// Compiles efficient/ffbf's own src/rabin-karp/ffbf.cpp, in place and unmodified, into oracle/_ref/.
// The file is pulled in with #include from the reference checkout (FFBF_REF_SOURCE); no reference
// source is copied into this repository. Three shims make it build and run here without changing
// what it computes:
//
//  * ffbf.cpp:501 reads `if (read < 0)`, an ordered comparison of the function `read` with 0, which
//    g++ 13 rejects. `read` is renamed to a function object that forwards calls to ::read and whose
//    `< 0` is false -- what the comparison of a non-null function address evaluates to.
//  * The filter memory comes from mmap(MAP_SHARED) of a hugetlbfs file (ffbf.cpp:91-107). There is
//    no hugetlbfs here, and an empty regular file would SIGBUS, so mmap is redirected to anonymous
//    zero-filled memory of the same size. The empty file the constructor creates is still unlinked
//    by the destructor.
//  * When FFBF_REF_DUMP names a file, the destructor's munmap first writes the whole mapping there
//    (main bit array then feed-forward bit array, N/8 bytes each), so tests can compare the
//    feed-forward filter, which the reference never saves.
//  * When FFBF_REF_FF_IN names a file of N/8 bytes, the mapping's feed-forward half starts with that
//    file's contents instead of zeros. Run over an empty stdin, processFile then sets no bit and
//    filterPhrases (ffbf.cpp:394-485) prunes the patterns with the given feed-forward array: the OR
//    of the arrays that runs over line-aligned shards of one text dumped, which equals the array a
//    single run over the whole text builds (a window never spans a '\n').
#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>
#include <xmmintrin.h>

#include <fstream>
#include <iostream>
#include <queue>
#include <string>
#include <vector>

namespace ffbf_ref_shim {
struct read_fn {
    ssize_t operator()(int fd, void* buf, size_t n) const { return ::read(fd, buf, n); }
};
static inline bool operator<(const read_fn&, int) { return false; }
static const read_fn read_obj = {};

static void* map_fn(void*, size_t len, int prot, int, int, off_t) {
    void* p = ::mmap(NULL, len, prot, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    const char* ff_in = getenv("FFBF_REF_FF_IN");
    if (p != MAP_FAILED && ff_in && *ff_in) {
        FILE* f = fopen(ff_in, "rb");
        const size_t half = len / 2;
        if (!f || fread((char*)p + half, 1, half, f) != half) {
            fprintf(stderr, "FFBF_REF_FF_IN: cannot read %zu bytes from %s\n", half, ff_in);
            exit(3);
        }
        fclose(f);
    }
    return p;
}

static int unmap_fn(void* addr, size_t len) {
    const char* path = getenv("FFBF_REF_DUMP");
    if (path && *path) {
        FILE* f = fopen(path, "wb");
        if (f) {
            fwrite(addr, 1, len, f);
            fclose(f);
        }
    }
    return ::munmap(addr, len);
}
}  // namespace ffbf_ref_shim

#define read ffbf_ref_shim::read_obj
#define mmap ffbf_ref_shim::map_fn
#define munmap ffbf_ref_shim::unmap_fn

#include FFBF_REF_SOURCE
