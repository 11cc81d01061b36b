// ORACLE — test infrastructure only.  Builds against the reference's own decoder header, where it
// lies in the reference tree (-I <reference root>), untouched, inside a namespace the way the
// reference's own 5-codeword performance test does
// (tests/test_tile_matrix_40tile_lockstep_stepper_sfpi_5cw_performance.cpp:33-36).
//
// Runs the reference's run_ldpc_worker (engines/scalar_5w/ldpc_decoder_core.h:214-586) on one
// worker's batch and records what it saw and produced, to pin the CPU restatement and the GPU kernels:
//
//   ref_golden <matrix.bin> <out.bin> mu sigma l_max r_max l_post_max max_iter n_codewords s0 s1 s2 s3
//
// matrix.bin: u32 N, M, P, max_check_deg, then M*(max_check_deg+1) u16 rows [deg, v0.., 0xFFFF pad]
// (the flattened layout of ldpc_sim_scalar.cpp:193-199).
// out.bin, per codeword pair: u32 in[N] (packed bf16 channel LLRs, cw0 in bits 15:0, as the worker
// fills them at ldpc_decoder_core.h:262-297), u32 out[N] (the same buffer after decoding), u32
// stats[4] of that pair (bit errors, frame errors, cw0 iterations, sample LLR); then u32 stats[4]
// summed over pairs (iterations and sample of the first pair).
//
// The channel is replayed by calling the reference's own generator functions in the worker's order
// (one generate_awgn_llr_pair for codeword 0 then one for codeword 1 per position pair); the decoder
// call is a single run_ldpc_worker per pair so that the buffer after the call is that pair's result.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

// The header's own includes must be seen first, outside the namespace.
#include <stdint.h>
#include <string.h>
#include <cstring>

namespace ref {
#include "engines/scalar_5w/ldpc_decoder_core.h"
}

static uint32_t rd32(FILE* f) {
    uint32_t v = 0;
    if (fread(&v, 4, 1, f) != 1) { fprintf(stderr, "short matrix file\n"); exit(2); }
    return v;
}

int main(int argc, char** argv) {
    if (argc != 14) {
        fprintf(stderr, "usage: ref_golden matrix.bin out.bin mu sigma l_max r_max l_post_max max_iter "
                        "n_codewords s0 s1 s2 s3\n");
        return 2;
    }
    FILE* fm = fopen(argv[1], "rb");
    if (!fm) { perror("matrix"); return 2; }
    uint32_t N = rd32(fm), M = rd32(fm), P = rd32(fm), dmax = rd32(fm);
    std::vector<uint16_t> h((size_t)M * (dmax + 1));
    if (fread(h.data(), 2, h.size(), fm) != h.size()) { fprintf(stderr, "short rows\n"); return 2; }
    fclose(fm);
    float mu = strtof(argv[3], nullptr), sigma = strtof(argv[4], nullptr);
    float l_max = strtof(argv[5], nullptr), r_max = strtof(argv[6], nullptr);
    float l_post_max = strtof(argv[7], nullptr);
    uint32_t max_iter = (uint32_t)strtoul(argv[8], nullptr, 0);
    uint32_t ncw = (uint32_t)strtoul(argv[9], nullptr, 0);
    uint32_t s[4];
    for (int i = 0; i < 4; i++) s[i] = (uint32_t)strtoul(argv[10 + i], nullptr, 0);
    if (dmax > ref::MAX_DEG_STRIDE) { fprintf(stderr, "degree above the reference's stride\n"); return 2; }

    FILE* fo = fopen(argv[2], "wb");
    if (!fo) { perror("out"); return 2; }
    std::vector<uint32_t> llr(N), rmsg((size_t)M * ref::MAX_DEG_STRIDE);
    ref::Xoshiro128Plus rng;
    rng.init_state(s[0], s[1], s[2], s[3]);
    uint32_t total[4] = {0, 0, 0, 0};
    const uint32_t ntx = N - P;
    for (uint32_t cw = 0; cw < ncw; cw += 2) {
        const uint32_t here = (ncw - cw) >= 2 ? 2 : 1;
        ref::Xoshiro128Plus start = rng;
        // Replay of the worker's channel fill (ldpc_decoder_core.h:262-297) with its own functions.
        std::vector<uint32_t> in(N, 0);
        if (sigma > 0.0f) {
            for (uint32_t i = 0; i < ntx; i += 2) {
                float a0, a1, b0, b1;
                ref::generate_awgn_llr_pair(rng, mu, sigma, a0, a1);
                if (l_max > 0.0f) {
                    if (a0 > l_max) a0 = l_max; else if (a0 < -l_max) a0 = -l_max;
                    if (a1 > l_max) a1 = l_max; else if (a1 < -l_max) a1 = -l_max;
                }
                ref::generate_awgn_llr_pair(rng, mu, sigma, b0, b1);
                if (l_max > 0.0f) {
                    if (b0 > l_max) b0 = l_max; else if (b0 < -l_max) b0 = -l_max;
                    if (b1 > l_max) b1 = l_max; else if (b1 < -l_max) b1 = -l_max;
                }
                in[i] = ref::fp32_to_bf16(a0) | ((uint32_t)ref::fp32_to_bf16(b0) << 16);
                in[i + 1] = ref::fp32_to_bf16(a1) | ((uint32_t)ref::fp32_to_bf16(b1) << 16);
            }
        } else {
            float m = mu;
            if (l_max > 0.0f && m > l_max) m = l_max;
            uint32_t p = ref::fp32_to_bf16(m);
            for (uint32_t i = 0; i < ntx; i++) in[i] = p | (p << 16);
        }
        uint32_t st[4];
        ref::run_ldpc_worker(0, here, N, M, dmax, P, max_iter, mu, sigma, l_max, r_max, l_post_max,
                             start.s[0], start.s[1], start.s[2], start.s[3], h.data(), llr.data(),
                             rmsg.data(), st);
        // The worker started from the same generator state as the replay and draws the same numbers,
        // so `in` is the buffer it decoded and `rng` is where the next pair starts.
        fwrite(in.data(), 4, N, fo);
        fwrite(llr.data(), 4, N, fo);
        fwrite(st, 4, 4, fo);
        total[0] += st[0];
        total[1] += st[1];
        if (cw == 0) total[2] = st[2];
        total[3] = st[3];
    }
    fwrite(total, 4, 4, fo);
    fclose(fo);
    return 0;
}
