// Host-only checks of the tuned scan's sizing rules, linked against libffbf.so (no device is touched):
// rows per stream alone on the GPU (waves of equal items over the CTA slots, a stream's 32-byte halo
// costing a quarter row) and in a batch (at least four items of the job's own), the CTA size of each
// configuration, and the key width of the result sorts. Prints each failure and exits non-zero on any.
#include <cstdio>

#include "ffbf_order.cuh"
#include "ffbf_scan_fast.cuh"

namespace {

int failures = 0;

void expect(const char* what, unsigned long long got, unsigned long long want) {
    if (got != want) {
        std::printf("FAIL %s: got %llu, want %llu\n", what, got, want);
        failures++;
    }
}

}  // namespace

int main() {
    using ffbf::FastConfig;
    const unsigned long long M = 1ull << 20, G = 1ull << 30;
    const int sms = 148;
    const FastConfig dense192{192, 1, 0, 1};   // two 192-thread CTAs per SM
    const FastConfig sparse512{512, 0, 0, 0};  // one CTA per SM
    const FastConfig staged512{0, 3, 0, 0};    // per-stage barriers: always 512 threads

    expect("dense 4 GiB", ffbf::fast_rows(4 * G, dense192, sms, false), 16);
    expect("dense 8 GiB", ffbf::fast_rows(8 * G, dense192, sms, false), 16);
    expect("dense 1 GiB", ffbf::fast_rows(1 * G, dense192, sms, false), 8);
    expect("dense 256 MiB", ffbf::fast_rows(256 * M, dense192, sms, false), 8);
    expect("dense 128 MiB chunk", ffbf::fast_rows(128 * M, dense192, sms, false), 4);
    expect("sparse 1 GiB", ffbf::fast_rows(1 * G, sparse512, sms, false), 16);
    expect("sparse 256 MiB", ffbf::fast_rows(256 * M, sparse512, sms, false), 4);
    expect("sparse 64 MiB", ffbf::fast_rows(64 * M, sparse512, sms, false), 8);
    expect("sparse 8 MiB chunk", ffbf::fast_rows(8 * M, sparse512, sms, false), 4);
    expect("staged 1 GiB", ffbf::fast_rows(1 * G, staged512, sms, false), 16);
    expect("batch 1 MiB", ffbf::fast_rows(1 * M, sparse512, sms, true), 4);
    expect("batch 64 MiB", ffbf::fast_rows(64 * M, sparse512, sms, true), 16);

    expect("CTAs per SM, dense 192", ffbf::fast_ctas_per_sm(dense192), 2);
    expect("CTAs per SM, sparse 512", ffbf::fast_ctas_per_sm(sparse512), 1);
    expect("threads, staged", ffbf::config_threads(staged512), 512);
    expect("threads, dense 192 order 2", ffbf::config_threads(FastConfig{192, 1, 0, 2}), 384);
    expect("threads, deferred 512", ffbf::config_threads(FastConfig{512, 2, 0, 0}), 256);

    expect("key bits of 1", ffbf::key_bits_for(1), 1);
    expect("key bits of 2", ffbf::key_bits_for(2), 2);
    expect("key bits of 2^32 - 1", ffbf::key_bits_for((1ull << 32) - 1), 32);
    expect("key bits of 2^32", ffbf::key_bits_for(1ull << 32), 33);

    if (failures == 0) std::printf("row model: all checks passed\n");
    return failures ? 1 : 0;
}
