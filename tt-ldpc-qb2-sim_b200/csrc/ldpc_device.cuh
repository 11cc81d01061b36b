// Device-side building blocks of the AR4JA Monte Carlo path (sm_100a).
//
//   * Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
//     SC'11): a counter-based generator, so frame f's channel depends only on (seed, f) and any
//     chunk of frames can be regenerated independently (replaces the reference's per-core
//     xoshiro128+ streams, engines/scalar_5w/ldpc_decoder_core.h:26-65).
//   * Box-Muller AWGN and BPSK LLR formation: LLR = mu + sigma*n with mu = 4R Eb/N0,
//     sigma = sqrt(8R Eb/N0) (engines/scalar_5w/ldpc_sim_scalar.cpp:351-355).
//   * The Approximate-Min* step and storage rounding of the reference's scalar decoder
//     (engines/scalar_5w/ldpc_decoder_core.h:84-90, 154-201).  Every multiply and add of the decoder
//     is an explicit round-to-nearest intrinsic so the compiler never fuses them into an FMA: the
//     reference rounds after each operation and the results must match it bit for bit.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace ldpcb200 {

enum Storage : int { STORE_BF16 = 0, STORE_FP32 = 1, STORE_FP16 = 2 };
// ALGO_WROW is not a separate decoder: it is the weighted decoder (ALGO_WAMIN) for weight tables whose
// classes are uniform over each row's edges (one (alpha, beta) per protograph check row), which the
// kernels apply once per row instead of once per edge.  Callers request ALGO_WAMIN; the library
// picks the per-row kernel when the table allows it.
enum Algo : int { ALGO_AMIN = 0, ALGO_NMS = 1, ALGO_WAMIN = 2, ALGO_CIRC = 3, ALGO_WROW = 4 };
constexpr bool algo_weighted(int a) { return a == ALGO_WAMIN || a == ALGO_WROW; }

// ------------------------------------------------------------------ Philox-4x32-10
struct U32x4 { uint32_t x, y, z, w; };

// One round: each 32x32-bit product is one wide multiply (both halves at once).
__device__ __forceinline__ U32x4 philox_round(U32x4 c, uint32_t k0, uint32_t k1) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    return U32x4{(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0};
}

__device__ __forceinline__ U32x4 philox4x32_10(U32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        c = philox_round(c, k0, k1);
    }
    return c;
}

// Two uniforms -> two standard normals.  u1 = x0*2^-32 + 2^-33 lies in (0, 1]; the angle is
// 2*pi*(x1*2^-32) - pi in [-pi, pi), the range where the fast hardware sine/cosine are accurate.
__device__ __forceinline__ void box_muller(uint32_t x0, uint32_t x1, float& n0, float& n1) {
    const float u1 = __fmaf_rn(__uint2float_rn(x0), 2.3283064365386963e-10f, 1.1641532182693481e-10f);
    const float a = __fmaf_rn(__uint2float_rn(x1), 1.4629180792671596e-09f, -3.14159265358979f);
    const float rad = __fsqrt_rn(-2.0f * __logf(u1));
    float s, c;
    __sincosf(a, &s, &c);
    n0 = rad * c;
    n1 = rad * s;
}

// Per-frame Eb/N0 for mixed workloads: uniform in [lo, hi) dB, drawn from the frame's Philox stream
// with counter word 0 = 0xFFFFFFFF (the channel uses words 0 .. N/4), then the LLR mean and deviation
// of that Eb/N0 at code rate R (mu = 4 R Eb/N0, sigma = sqrt(8 R Eb/N0)) and its bin of [lo, hi).
constexpr int SNR_BINS = 32;

__device__ __forceinline__ void frame_snr(float lo, float hi, float rate, uint64_t frame, uint32_t stream,
                                          uint32_t k0, uint32_t k1, float& mu, float& sigma, int& bin) {
    const U32x4 x = philox4x32_10(U32x4{0xFFFFFFFFu, (uint32_t)frame, (uint32_t)(frame >> 32), stream}, k0, k1);
    const float u = __uint2float_rz(x.x >> 8) * (1.0f / 16777216.0f);
    const float g = exp10f(0.1f * __fmaf_rn(hi - lo, u, lo));
    mu = 4.0f * rate * g;
    sigma = sqrtf(8.0f * rate * g);
    bin = min((int)(u * (float)SNR_BINS), SNR_BINS - 1);
}

// ------------------------------------------------------------------ storage rounding
__device__ __forceinline__ float bf16_round(float x) {  // fp32_to_bf16, RNE (ldpc_decoder_core.h:84-90)
    return __bfloat162float(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float fp16_round_sat(float x) {  // IEEE fp16 RNE, saturated at 65504
    return __half2float(__float2half_rn(fminf(fmaxf(x, -65504.0f), 65504.0f)));
}

// ------------------------------------------------------------------ Approximate-Min*
// min*(m, a) = max(min(m, a) - g(|m - a|), 0), g piecewise linear (ldpc_decoder_core.h:186-190),
// stated as the reference writes it.  The kernels use amin_step_fma below, which returns the same
// bits for finite inputs in fewer instructions.
__device__ __forceinline__ float amin_step(float m, float a) {
    const float diff = fabsf(__fsub_rn(m, a));
    const float cur = fminf(m, a);
    const float c1 = __fsub_rn(0.69315f, __fmul_rn(0.40f, diff));
    const float c2 = __fsub_rn(0.49315f, __fmul_rn(0.328f, __fsub_rn(diff, 0.5f)));
    float corr = diff < 0.5f ? c1 : c2;
    corr = diff >= 2.0f ? 0.0f : corr;
    return fmaxf(__fsub_rn(cur, corr), 0.0f);
}

// The same step in 11 instructions.  The flag f2 = [diff < 2] comes from a saturated fused
// multiply-add: 2^30 (2 - diff) is >= 32 for every float diff below 2 and <= 0 otherwise, so
// saturation gives exactly 1 or 0.  With c the correction line of the region (c1 below 0.5, c2 from
// there on), u = cur - c * f2 subtracts c with one rounding or nothing (a product with a 0/1 flag is
// exact, and adding a signed zero leaves a value unchanged), so the result equals amin_step bit for
// bit.  Inputs must be finite (c * 0 would be NaN for diff = inf): the QC kernel never feeds inf.
// The product 0.328 (diff - 0.5) is one fused multiply-add, 0.328 diff - 0.164 with 0.164 exactly half
// of the float 0.328: it rounds the exact value 0.328 (diff - 0.5) once, as the reference's
// multiply does, because diff - 0.5 is exact for every diff in [0.25, 2) and c2 is used only on
// [0.5, 2).  (An earlier form selected both lines with two saturated flags, all on the FMA pipe: one
// more instruction per step and 6 % slower, although it kept the busier ALU pipe free.)
constexpr float AMIN_K2 = 0.328f;
__device__ __forceinline__ float amin_step_fma(float m, float a) {
    const float diff = fabsf(__fsub_rn(m, a));
    const float cur = fminf(m, a);
    const float c1 = __fsub_rn(0.69315f, __fmul_rn(0.40f, diff));
    const float c2 = __fsub_rn(0.49315f, __fmaf_rn(AMIN_K2, diff, -0.5f * AMIN_K2));
    const float f2 = __saturatef(__fmaf_rn(diff, -1073741824.0f, 2147483648.0f));
    const float c = diff < 0.5f ? c1 : c2;
    return fmaxf(__fmaf_rn(-c, f2, cur), 0.0f);
}

// The circulant engine's min* (tests/test_circulant_dma_stepper.cpp:39-54 and
// engines/tile_matrix_4cw/sfpi_host_emu.h:590-607): max(min(a, b) - max(c1 + k1 d, c2 + k2 d, 0), 0)
// with d = |a - b|, every product and sum rounded on its own (no fused multiply-add), so it equals the
// reference's fp32 expression bit for bit.  a, b >= +0; the result is never -0.
// |a - b| equals max - min exactly (rounding is symmetric), and the correction max(l1, l2, 0) is one
// three-input max (sm_100): 9 instructions per min*.
struct CircConsts { float c1, k1, c2, k2; };
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float circ_g(float a, float b, const CircConsts& k) {
    const float mn = fminf(a, b);
    const float d = fabsf(__fsub_rn(a, b));
    const float l1 = __fadd_rn(k.c1, __fmul_rn(k.k1, d));
    const float l2 = __fadd_rn(k.c2, __fmul_rn(k.k2, d));
    return fmaxf(__fsub_rn(mn, fmax3f(l1, l2, 0.0f)), 0.0f);
}

}  // namespace ldpcb200
