// ORACLE — test infrastructure only.  Builds against the reference's min* unit test
// (tests/unit_sfpu/test_piecewise_amin_star.cpp) where it lies in the reference tree, untouched: its
// main() is renamed away and its two-line min* (approx_min_star_2piece, :44-53, the circulant
// engine's form) is evaluated on caller pairs.
//
//   ref_gdelta <in.bin> <out.bin>
//
// in.bin: u32 n, then n pairs of f32 (a, b); out.bin: n f32 approx_min_star_2piece(a, b) and n f32
// with the bf16 rounding the test applies (use_bf16 = true).
#include <cstdint>
#include <cstdio>
#include <vector>

#define main ref_piecewise_amin_star_main
#include "tests/unit_sfpu/test_piecewise_amin_star.cpp"
#undef main

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: ref_gdelta in.bin out.bin\n");
        return 2;
    }
    FILE* fi = fopen(argv[1], "rb");
    if (!fi) { perror("in"); return 2; }
    uint32_t n = 0;
    if (fread(&n, 4, 1, fi) != 1) { fprintf(stderr, "short input\n"); return 2; }
    std::vector<float> ab(2 * (size_t)n);
    if (fread(ab.data(), 4, ab.size(), fi) != ab.size()) { fprintf(stderr, "short pairs\n"); return 2; }
    fclose(fi);
    std::vector<float> out(2 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) {
        out[i] = approx_min_star_2piece(ab[2 * i], ab[2 * i + 1], false);
        out[n + i] = approx_min_star_2piece(ab[2 * i], ab[2 * i + 1], true);
    }
    FILE* fo = fopen(argv[2], "wb");
    if (!fo) { perror("out"); return 2; }
    fwrite(out.data(), 4, out.size(), fo);
    fclose(fo);
    return 0;
}
