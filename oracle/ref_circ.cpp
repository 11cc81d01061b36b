// ORACLE — test infrastructure only.  Builds against the reference's circulant-engine golden stepper
// where it lies in the reference tree (-I <reference root>), untouched: its main() is renamed away and
// its tile functions are called directly.
//
// Decodes groups of 4 codewords of AR4JA rate 1/2, K = 1024 with the reference's
// step_tile_circulant_dma_scalar / step_tile_circulant_dma_sfpu (tests/test_circulant_dma_stepper.cpp:
// 332-482, 487-565): 40 tiles per iteration (32 degree-6 tiles of rows 512..1535, then 8 degree-3
// tiles of rows 0..511), driven the way its Monte Carlo loop drives them
// (tests/test_circulant_dma_stepper.cpp:760-822): after every iteration the full syndrome of each
// still-active codeword (bit = value < 0), a codeword meeting it is frozen with iterations =
// iteration + 1; a codeword still active after max_iter is a frame error whose bit errors are its
// first 1024 positions with value <= 0.
//
//   ref_circ <in.bin> <out.bin> <sfpu 0|1> <damping> <max_iter>
//
// in.bin: u32 n_groups, then per group 2560 x Packed4CW_BF16 (u16 cw[4] per variable node): the
// channel LLRs as bf16, punctured nodes 2048..2559 zero.
// out.bin, per group: the 2560 x u16[4] nodes after decoding, then u32 iters[4], u32 active[4]
// (1 = never met the syndrome), u32 bit_errors[4] (the loop's count, 0 for converged codewords).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#define main ref_circulant_stepper_main
#include "tests/test_circulant_dma_stepper.cpp"
#undef main

int main(int argc, char** argv) {
    if (argc != 6) {
        fprintf(stderr, "usage: ref_circ in.bin out.bin sfpu damping max_iter\n");
        return 2;
    }
    FILE* fi = fopen(argv[1], "rb");
    if (!fi) { perror("in"); return 2; }
    uint32_t n_groups = 0;
    if (fread(&n_groups, 4, 1, fi) != 1) { fprintf(stderr, "short input\n"); return 2; }
    const bool use_sfpu = atoi(argv[3]) != 0;
    const float damping = strtof(argv[4], nullptr);
    const uint32_t max_iter = (uint32_t)strtoul(argv[5], nullptr, 0);
    FILE* fo = fopen(argv[2], "wb");
    if (!fo) { perror("out"); return 2; }

    for (uint32_t g = 0; g < n_groups; ++g) {
        std::vector<Packed4CW_BF16> vnodes(2560);
        if (fread(vnodes.data(), sizeof(Packed4CW_BF16), 2560, fi) != 2560) {
            fprintf(stderr, "short input group %u\n", g);
            return 2;
        }
        std::vector<Packed4CW_BF16> r_msg_scalar(TOTAL_TILES * 192);
        std::vector<uint16_t> r_msg_sfpu(TOTAL_TILES * 1024, 0);
        TileScratchpad scratch;
        uint32_t active_mask = 0xF;
        uint32_t cw_iters[4] = {max_iter, max_iter, max_iter, max_iter};
        for (uint32_t iter = 0; iter < max_iter; ++iter) {
            const bool is_iter0 = (iter == 0);
            for (uint32_t t = 0; t < TOTAL_TILES; ++t) {
                if (use_sfpu)
                    step_tile_circulant_dma_sfpu(t, vnodes.data(), &r_msg_sfpu[t * 1024], is_iter0, scratch,
                                                 active_mask, false, damping);
                else
                    step_tile_circulant_dma_scalar(t, vnodes.data(), &r_msg_scalar[t * 192], is_iter0, scratch,
                                                   active_mask, false);
            }
            for (uint32_t cw = 0; cw < 4; ++cw) {
                if (!(active_mask & (1u << cw))) continue;
                bool satisfied = true;
                for (uint32_t m = 0; m < 1536 && satisfied; ++m) {
                    int syn = 0;
                    const uint32_t deg = (m < 512) ? 3 : 6;
                    for (uint32_t d = 0; d < deg; ++d)
                        if (bf16_to_fp32(vnodes[CHECK_TO_VAR[m][d]].cw[cw]) < 0.0f) syn ^= 1;
                    if (syn) satisfied = false;
                }
                if (satisfied) {
                    cw_iters[cw] = iter + 1;
                    active_mask &= ~(1u << cw);
                }
            }
            if (active_mask == 0) break;
        }
        uint32_t active[4], be[4];
        for (uint32_t cw = 0; cw < 4; ++cw) {
            active[cw] = (active_mask >> cw) & 1u;
            be[cw] = 0;
            if (active[cw])
                for (uint32_t k = 0; k < 1024; ++k)
                    if (bf16_to_fp32(vnodes[k].cw[cw]) <= 0.0f) be[cw]++;
        }
        fwrite(vnodes.data(), sizeof(Packed4CW_BF16), 2560, fo);
        fwrite(cw_iters, 4, 4, fo);
        fwrite(active, 4, 4, fo);
        fwrite(be, 4, 4, fo);
    }
    fclose(fi);
    fclose(fo);
    return 0;
}
