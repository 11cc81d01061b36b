// ORACLE — test infrastructure only (the timed CPU baseline of bench.py).  Builds against the
// reference's own decoder header where it lies in the reference tree, untouched, in a namespace as
// tests/test_tile_matrix_40tile_lockstep_stepper_sfpi_5cw_performance.cpp:33-36 does, and runs the
// reference's Monte Carlo worker run_ldpc_worker (engines/scalar_5w/ldpc_decoder_core.h:214-586) on
// every host thread:
//
//   ref_mc <matrix.bin> mu sigma max_iter max_frames time_budget_s seed threads
//
// Work is handed out one codeword pair at a time from a shared counter; pair p starts its xoshiro128+
// stream from the reference's splitmix32 seeding of (seed ^ p*0x9E3779B1) (ldpc_sim_scalar.cpp:46-63),
// like the per-pair derived seeds of the reference's golden-model runner (the 5cw test, :904-907).
// A thread stops when max_frames are claimed or the time budget is spent.  Prints one JSON line.
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

// The header's own includes must be seen first, outside the namespace.
#include <stdint.h>
#include <string.h>
#include <cstring>

namespace ref {
#include "engines/scalar_5w/ldpc_decoder_core.h"
}

static void seed_state(uint32_t seed, uint32_t s[4]) {
    uint32_t sm = seed;
    for (int i = 0; i < 4; i++) {
        uint32_t z = (sm += 0x9e3779b9u);
        z ^= z >> 16; z *= 0x21f0aaadu;
        z ^= z >> 15; z *= 0x735a2d97u;
        z ^= z >> 15;
        s[i] = z;
    }
}

int main(int argc, char** argv) {
    if (argc != 9) {
        fprintf(stderr, "usage: ref_mc matrix.bin mu sigma max_iter max_frames time_budget_s seed threads\n");
        return 2;
    }
    FILE* fm = fopen(argv[1], "rb");
    if (!fm) { perror("matrix"); return 2; }
    uint32_t hdr[4];
    if (fread(hdr, 4, 4, fm) != 4) return 2;
    const uint32_t N = hdr[0], M = hdr[1], P = hdr[2], dmax = hdr[3];
    std::vector<uint16_t> h((size_t)M * (dmax + 1));
    if (fread(h.data(), 2, h.size(), fm) != h.size()) return 2;
    fclose(fm);
    if (dmax > ref::MAX_DEG_STRIDE) { fprintf(stderr, "degree above the reference's stride\n"); return 2; }
    const float mu = strtof(argv[2], nullptr), sigma = strtof(argv[3], nullptr);
    const uint32_t max_iter = (uint32_t)strtoul(argv[4], nullptr, 0);
    const uint64_t max_frames = strtoull(argv[5], nullptr, 0);
    const double budget = strtod(argv[6], nullptr);
    const uint32_t seed = (uint32_t)strtoul(argv[7], nullptr, 0);
    int threads = atoi(argv[8]);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();

    std::atomic<uint64_t> next_pair{0};
    std::atomic<uint64_t> frames{0}, be{0}, be2{0}, fe{0}, it0{0}, n0{0};
    const uint64_t max_pairs = (max_frames + 1) / 2;
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        std::vector<uint32_t> llr(N), rmsg((size_t)M * ref::MAX_DEG_STRIDE);
        for (;;) {
            double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (budget > 0 && el >= budget) break;
            uint64_t p = next_pair.fetch_add(1);
            if (p >= max_pairs) break;
            uint32_t s[4];
            seed_state(seed ^ (uint32_t)(p * 0x9E3779B1ull), s);
            uint32_t st[4];
            ref::run_ldpc_worker(0, 2, N, M, dmax, P, max_iter, mu, sigma, 0.0f, 0.0f, 0.0f,
                                 s[0], s[1], s[2], s[3], h.data(), llr.data(), rmsg.data(), st);
            frames += 2;
            be += st[0];
            be2 += (uint64_t)st[0] * st[0];
            fe += st[1];
            it0 += st[2];
            n0 += 1;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("{\"frames\": %llu, \"bit_errors\": %llu, \"bit_errors_sq_pairs\": %llu, \"frame_errors\": %llu, "
           "\"cw0_iter_sum\": %llu, \"cw0_count\": %llu, \"elapsed_s\": %.6f, \"threads\": %d}\n",
           (unsigned long long)frames.load(), (unsigned long long)be.load(), (unsigned long long)be2.load(),
           (unsigned long long)fe.load(), (unsigned long long)it0.load(),
           (unsigned long long)n0.load(), el, threads);
    return 0;
}
