/*
 * ORACLE — test infrastructure only.  Nothing in the product links, loads or runs this file; only
 * tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU-baseline leg use it.
 *
 * CPU restatement of the reference's scalar AR4JA Monte Carlo path, one codeword at a time:
 *
 *   - channel:  xoshiro128+ (engines/scalar_5w/ldpc_decoder_core.h:13-65 and
 *               engines/scalar_5w/ldpc_sim_scalar.cpp:43-106 for the root seeding / long_jump),
 *               Marsaglia polar AWGN with the reference's fast_ln / fast_rsqrt
 *               (ldpc_decoder_core.h:92-152), LLR = mu + sigma*n, optional +-l_max clip,
 *               storage quantisation (ldpc_decoder_core.h:262-297),
 *   - decoder:  row-layered Approximate-Min* (ldpc_decoder_core.h:154-201, 413-520) or normalised
 *               min-sum (ldpc_decoder_core.h:320-411), rows in the order given, edges in row order,
 *               syndrome stop from iteration index 2 (ldpc_decoder_core.h:524-553),
 *   - tally:    bit errors = sign bits set over the first N-P positions, a frame error when that
 *               count is non-zero (ldpc_decoder_core.h:556-577).
 *
 * Storage modes: STORE_BF16 reproduces the reference numerics exactly (L and r rounded to bf16 with
 * round-to-nearest-even after every update, fp32_to_bf16 at ldpc_decoder_core.h:84-90);
 * STORE_FP32 keeps both in fp32; STORE_FP16 keeps L in fp32 and rounds r to IEEE fp16 (magnitudes
 * saturated at 65504).  All arithmetic is plain fp32 with one rounding per operation: build with
 * -ffp-contract=off so that no multiply-add is fused (the reference's expressions are separate
 * multiplies and adds).
 *
 * Parity pin: tests/golden holds outputs of the reference's own run_ldpc_worker, built from its
 * sources by oracle/Makefile; tests/test_oracle_golden.py checks this file against them bit for bit.
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <math.h>

#define STORE_BF16 0
#define STORE_FP32 1
#define STORE_FP16 2
#define ALGO_AMIN 0
#define ALGO_NMS 1
#define ORC_MAX_DEG 64

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* bf16 round-to-nearest-even of the fp32 bit pattern (ldpc_decoder_core.h:84-90). */
static inline uint16_t to_bf16_bits(float x) {
    uint32_t u = f2u(x);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
static inline float q_bf16(float x) { return u2f(((uint32_t)to_bf16_bits(x)) << 16); }

/* IEEE binary16 round-to-nearest-even, saturated at +-65504 (written out so the oracle does not
 * depend on compiler support for _Float16). */
static inline float q_fp16(float x) {
    if (x > 65504.0f) x = 65504.0f;
    if (x < -65504.0f) x = -65504.0f;
    uint32_t u = f2u(x);
    uint32_t sign = u & 0x80000000u;
    uint32_t a = u & 0x7FFFFFFFu;
    if (a < 0x33000000u) return u2f(sign);            /* |x| < 2^-25: rounds to zero */
    int e = (int)(a >> 23) - 127;
    uint32_t mant = (a & 0x7FFFFFu) | 0x800000u;       /* 24-bit significand */
    int keep;                                          /* significand bits kept */
    if (e >= -14) keep = 11;                           /* normal half */
    else keep = 11 - (-14 - e);                        /* subnormal half: fewer bits */
    int drop = 24 - keep;
    uint32_t q = mant >> drop;
    uint32_t rem = mant & ((1u << drop) - 1u);
    uint32_t half = 1u << (drop - 1);
    if (rem > half || (rem == half && (q & 1u))) q += 1u;
    /* value = q * 2^(e - keep + 1) */
    float v = ldexpf((float)q, e - keep + 1);
    return u2f(f2u(v) | sign);
}

static inline float store_L(int mode, float x) { return mode == STORE_BF16 ? q_bf16(x) : x; }
static inline float store_r(int mode, float x) {
    if (mode == STORE_BF16) return q_bf16(x);
    if (mode == STORE_FP16) return q_fp16(x);
    return x;
}

/* Approximate-Min* correction, ldpc_decoder_core.h:163,168,188,195. */
static inline float amin_corr(float diff) {
    if (diff >= 2.0f) return 0.0f;
    if (diff < 0.5f) return 0.69315f - 0.40f * diff;
    return 0.49315f - 0.328f * (diff - 0.5f);
}

/* One recursive min* step, ldpc_decoder_core.h:185-190 (and :193-197 for the final step). */
static inline float amin_step(float m, float a) {
    float diff = (m > a) ? (m - a) : (a - m);
    float cur = (m < a) ? m : a;
    float next = cur - amin_corr(diff);
    return (next > 0.0f) ? next : 0.0f;
}

static inline float fabs_bits(float x) { return u2f(f2u(x) & 0x7FFFFFFFu); }

/* Parity of the sign bits of L over every row; returns the number of rows that fail. */
static int syndrome_failures(int M, int dmax, const int32_t* rows, const int32_t* degs,
                             const float* L) {
    int fails = 0;
    for (int m = 0; m < M; m++) {
        uint32_t par = 0;
        for (int d = 0; d < degs[m]; d++) par ^= f2u(L[rows[(size_t)m * dmax + d]]) >> 31;
        fails += (int)par;
    }
    return fails;
}

/*
 * Decode one codeword from channel LLRs.
 *   rows      [M][dmax] variable indices (0-based, -1 padded), edges in row order
 *   degs      [M] row degrees
 *   llr_tx    [N-P] channel LLRs in fp32; positions N-P..N-1 are punctured (L = 0)
 *   l_max     channel clip (0 = off), applied before storage quantisation
 *   r_max, l_post_max: message and posterior clips (0 = off), ldpc_decoder_core.h:487,492-495
 * Outputs: post [N] final L (as stored), *iters, *synd_fail (failing rows after decoding),
 *          *bit_errors (sign bits over the first N-P positions).
 * Returns 0, or -1 on bad arguments.
 */
static int decode_impl(int N, int M, int P, int dmax, const int32_t* rows, const int32_t* degs,
                       int mode, int algo, int max_iter, float l_max, float r_max, float l_post_max,
                       const float* llr_tx, float* post, float* r_work, int32_t* iters,
                       int32_t* synd_fail, int32_t* bit_errors, int early_stop) {
    if (N <= 0 || M <= 0 || P < 0 || P > N || dmax <= 0 || dmax > ORC_MAX_DEG) return -1;
    const int ntx = N - P;
    float* L = post;
    for (int i = 0; i < ntx; i++) {
        float v = llr_tx[i];
        if (l_max > 0.0f) {
            if (v > l_max) v = l_max;
            else if (v < -l_max) v = -l_max;
        }
        L[i] = store_L(mode, v);
    }
    for (int i = ntx; i < N; i++) L[i] = 0.0f;
    float* r = r_work; /* [M][dmax] */
    for (size_t i = 0; i < (size_t)M * dmax; i++) r[i] = 0.0f;

    int done = 0;
    int it_used = max_iter;
    float q[ORC_MAX_DEG];
    for (int it = 0; it < max_iter; it++) {
        for (int m = 0; m < M; m++) {
            const int deg = degs[m];
            const int32_t* vn = rows + (size_t)m * dmax;
            float* rm = r + (size_t)m * dmax;
            uint32_t parity = 0;
            float mag_min, mag_all;   /* magnitude for the argmin edge / for every other edge */
            uint32_t min_idx = 0;
            if (algo == ALGO_NMS) {
                /* ldpc_decoder_core.h:322-366, 376-379 */
                float min1 = 999.0f, min2 = 999.0f;
                for (int d = 0; d < deg; d++) {
                    q[d] = L[vn[d]] - rm[d];
                    parity ^= f2u(q[d]) >> 31;
                    float a = fabs_bits(q[d]);
                    if (a < min1) { min2 = min1; min1 = a; min_idx = (uint32_t)d; }
                    else if (a < min2) { min2 = a; }
                }
                mag_min = 0.75f * min2;
                mag_all = 0.75f * min1;
            } else {
                /* ldpc_decoder_core.h:414-475 */
                float min_mag = 9999.0f;
                for (int d = 0; d < deg; d++) {
                    q[d] = L[vn[d]] - rm[d];
                    parity ^= f2u(q[d]) >> 31;
                    float a = fabs_bits(q[d]);
                    if (a < min_mag) { min_mag = a; min_idx = (uint32_t)d; }
                }
                /* compute_amin_star_general; compute_amin_star_deg3 gives the same values
                 * (both take the non-argmin edges in row order with identical arithmetic). */
                uint32_t first = (min_idx == 0) ? 1u : 0u;
                float m_oth = (deg > 1) ? fabs_bits(q[first]) : min_mag;
                for (int d = (int)first + 1; d < deg; d++) {
                    if ((uint32_t)d == min_idx) continue;
                    m_oth = amin_step(m_oth, fabs_bits(q[d]));
                }
                mag_min = m_oth;
                mag_all = amin_step(m_oth, min_mag);
            }
            for (int d = 0; d < deg; d++) {
                float mag = ((uint32_t)d == min_idx) ? mag_min : mag_all;
                if (r_max > 0.0f && mag > r_max) mag = r_max;
                uint32_t s = parity ^ (f2u(q[d]) >> 31);
                float rn = u2f(f2u(mag) | (s << 31));
                float ln = q[d] + rn;
                if (l_post_max > 0.0f) {
                    if (ln > l_post_max) ln = l_post_max;
                    else if (ln < -l_post_max) ln = -l_post_max;
                }
                L[vn[d]] = store_L(mode, ln);
                rm[d] = store_r(mode, rn);
            }
        }
        if (early_stop && it >= 2 && syndrome_failures(M, dmax, rows, degs, L) == 0) {
            done = 1;
            it_used = it + 1;
            break;
        }
    }
    (void)done;
    *iters = it_used;
    *synd_fail = syndrome_failures(M, dmax, rows, degs, L);
    int be = 0;
    for (int i = 0; i < ntx; i++) be += (int)(f2u(L[i]) >> 31);
    *bit_errors = be;
    return 0;
}

int oracle_decode(int N, int M, int P, int dmax, const int32_t* rows, const int32_t* degs,
                  int mode, int algo, int max_iter, float l_max, float r_max, float l_post_max,
                  const float* llr_tx, float* post, float* r_work, int32_t* iters,
                  int32_t* synd_fail, int32_t* bit_errors) {
    return decode_impl(N, M, P, dmax, rows, degs, mode, algo, max_iter, l_max, r_max, l_post_max, llr_tx,
                       post, r_work, iters, synd_fail, bit_errors, 1);
}

/* The same decoder run for exactly max_iter iterations with no syndrome stop: the unrolled decoder
 * the weighted (trainable) decoder reduces to at unit scale and zero offset.  The reference always
 * stops early (ldpc_decoder_core.h, the iteration loop's syndrome test); this variant exists to
 * check that reduction. */
int oracle_decode_nostop(int N, int M, int P, int dmax, const int32_t* rows, const int32_t* degs,
                         int mode, int algo, int max_iter, float l_max, float r_max, float l_post_max,
                         const float* llr_tx, float* post, float* r_work, int32_t* iters,
                         int32_t* synd_fail, int32_t* bit_errors) {
    return decode_impl(N, M, P, dmax, rows, degs, mode, algo, max_iter, l_max, r_max, l_post_max, llr_tx,
                       post, r_work, iters, synd_fail, bit_errors, 0);
}

/* ---------------- the circulant engine's decoder (rate 1/2 AR4JA, degrees 3 and 6) ---------------- */

/*
 * Restates the check-node arithmetic of the reference's circulant-engine golden stepper
 * (tests/test_circulant_dma_stepper.cpp) in its two forms:
 *
 *   CIRC_SCALAR  step_tile_circulant_dma_scalar (:332-482) with approx_min_star (:39-54): q = L - r
 *                in fp32, exact correction constants, r = +-mag, L = store(q + r) with r unrounded;
 *   CIRC_SFPU    step_tile_circulant_dma_sfpu (:487-565) with compute_tile_deg6_sfpi (:110-273) /
 *                compute_tile_deg3_sfpi (:278-327) and sfpi_amin_star_branchless
 *                (engines/tile_matrix_4cw/sfpi_host_emu.h:590-607), the device engine's math
 *                (engines/circulant_dma_4cw/compute_trisc.cpp:75-96, 299-658): Q = store(L - r), the
 *                correction constants truncated to bf16, mag scaled by the damping factor,
 *                r = store(+-mag), L = store(Q + r).
 *
 * Both use the min* g(a, b) = max(min(a, b) - max(c1 + k1 |a-b|, c2 + k2 |a-b|, 0), 0) with
 * (c1, k1, c2, k2) = (0.69315, -0.4, 0.65715, -0.328), and the pairwise tree of the degree-6 rows:
 * m03 = g(a0, a3), m14 = g(a1, a4), m25 = g(a2, a5); edge 0 gets g(g(m14, m25), a3), edge 3
 * g(g(m14, m25), a0), and likewise for the pairs (1, 4) and (2, 5); a degree-3 row gives each edge
 * g of the other two.  Edges are a row's columns in ascending order (the descriptor tables' edge
 * index, tools/generate_circulant_dma_tables.py:153-185).  Rows are visited in the order given
 * (the engine's tile schedule: rows 512..1535, then 0..511 for K = 1024).
 *
 * Stop and tally:
 *   CIRC_STOP_SYNDROME  the stepper's Monte Carlo loop (tests/test_circulant_dma_stepper.cpp:773-822):
 *                       full syndrome after every iteration (bit = value < 0); a frame that never
 *                       meets it is a frame error with bit errors = info positions with value <= 0;
 *   CIRC_STOP_GENIE     the device engine (engines/circulant_dma_4cw/reader_brisc.cpp:166-198,
 *                       writer_ncrisc.cpp:265-337): stop once no info position has its sign bit
 *                       set; a frame that never stops has bit errors = info positions with the sign
 *                       bit set, and is a frame error when that count is non-zero (always, unless
 *                       max_iter = 0).
 * A frame that stops reports zero bit errors, as both do.
 */
#define CIRC_SCALAR 0
#define CIRC_SFPU 1
#define CIRC_STOP_SYNDROME 0
#define CIRC_STOP_GENIE 1

static inline float trunc_bf16(float x) { return u2f(f2u(x) & 0xFFFF0000u); }

typedef struct { float c1, k1, c2, k2; } circ_consts;

static inline float circ_g(const circ_consts* k, float a, float b) {
    float mn = (b < a) ? b : a;
    float mx = (a < b) ? b : a;
    float diff = mx - mn;
    float line1 = k->c1 + k->k1 * diff;
    float line2 = k->c2 + k->k2 * diff;
    float corr = (line1 < line2) ? line2 : line1;
    if (corr < 0.0f) corr = 0.0f;
    float v = mn - corr;
    return (v < 0.0f) ? 0.0f : v;
}

/* The min* alone on n pairs ab[2i], ab[2i+1] (numerics as above), for pinning it to the
 * reference's min* unit test (tests/unit_sfpu/test_piecewise_amin_star.cpp:44-53). */
void oracle_circ_g_n(int numerics, const float* ab, int n, float* out) {
    circ_consts k = {0.69315f, -0.40f, 0.65715f, -0.328f};
    if (numerics == CIRC_SFPU) {
        k.c1 = trunc_bf16(k.c1); k.k1 = trunc_bf16(k.k1);
        k.c2 = trunc_bf16(k.c2); k.k2 = trunc_bf16(k.k2);
    }
    for (int i = 0; i < n; i++) out[i] = circ_g(&k, ab[2 * i], ab[2 * i + 1]);
}

static int syndrome_failures_lt0(int M, int dmax, const int32_t* rows, const int32_t* degs, const float* L) {
    int fails = 0;
    for (int m = 0; m < M; m++) {
        int par = 0;
        for (int d = 0; d < degs[m]; d++) par ^= (L[rows[(size_t)m * dmax + d]] < 0.0f);
        fails += par;
    }
    return fails;
}

/*
 * order [M]: the rows in update order.  n_info: the info positions 0..n_info-1 of the tally.
 * Outputs: post [N] final L, *iters, *synd_fail (rows failing, sign-bit parity), *bit_errors and
 * *frame_error as the engine tallies them.  Returns 0, or -1 on bad arguments (a row degree other
 * than 3 or 6, damping outside (0, 1]).
 */
int oracle_circ_decode(int N, int M, int P, int dmax, const int32_t* rows, const int32_t* degs,
                       const int32_t* order, int n_info, int mode, int numerics, float damping, int stop,
                       int max_iter, const float* llr_tx, float* post, float* r_work, int32_t* iters,
                       int32_t* synd_fail, int32_t* bit_errors, int32_t* frame_error) {
    if (N <= 0 || M <= 0 || P < 0 || P > N || dmax < 3 || dmax > ORC_MAX_DEG || n_info < 0 || n_info > N)
        return -1;
    if (!(damping > 0.0f && damping <= 1.0f)) return -1;
    for (int m = 0; m < M; m++)
        if (degs[m] != 3 && degs[m] != 6) return -1;
    circ_consts k = {0.69315f, -0.40f, 0.65715f, -0.328f};
    if (numerics == CIRC_SFPU) {
        k.c1 = trunc_bf16(k.c1); k.k1 = trunc_bf16(k.k1);
        k.c2 = trunc_bf16(k.c2); k.k2 = trunc_bf16(k.k2);
    }
    const int ntx = N - P;
    float* L = post;
    for (int i = 0; i < ntx; i++) L[i] = store_L(mode, llr_tx[i]);
    for (int i = ntx; i < N; i++) L[i] = 0.0f;
    float* r = r_work;
    for (size_t i = 0; i < (size_t)M * dmax; i++) r[i] = 0.0f;

    int stopped = 0, it_used = max_iter;
    for (int it = 0; it < max_iter && !stopped; it++) {
        for (int oi = 0; oi < M; oi++) {
            const int m = order[oi];
            const int deg = degs[m];
            const int32_t* vn = rows + (size_t)m * dmax;
            float* rm = r + (size_t)m * dmax;
            float q[6], a[6], mag[6];
            uint32_t par = 0, neg[6];
            for (int d = 0; d < deg; d++) {
                q[d] = L[vn[d]] - rm[d];
                if (numerics == CIRC_SFPU) {
                    q[d] = store_L(mode, q[d]);
                    neg[d] = f2u(q[d]) >> 31;          /* sign bit (sfpi::as<vInt> XOR) */
                } else {
                    neg[d] = q[d] < 0.0f;              /* (q < 0) ? -1 : 1 */
                }
                par ^= neg[d];
                a[d] = fabs_bits(q[d]);
            }
            if (deg == 6) {
                float m03 = circ_g(&k, a[0], a[3]), m14 = circ_g(&k, a[1], a[4]), m25 = circ_g(&k, a[2], a[5]);
                float o0 = circ_g(&k, m14, m25), o1 = circ_g(&k, m03, m25), o2 = circ_g(&k, m03, m14);
                mag[0] = circ_g(&k, o0, a[3]); mag[3] = circ_g(&k, o0, a[0]);
                mag[1] = circ_g(&k, o1, a[4]); mag[4] = circ_g(&k, o1, a[1]);
                mag[2] = circ_g(&k, o2, a[5]); mag[5] = circ_g(&k, o2, a[2]);
            } else {
                mag[0] = circ_g(&k, a[1], a[2]);
                mag[1] = circ_g(&k, a[0], a[2]);
                mag[2] = circ_g(&k, a[0], a[1]);
            }
            for (int d = 0; d < deg; d++) {
                float mg = mag[d];
                /* the degree-6 kernel always multiplies, the degree-3 one only below 1 (x 1 is exact) */
                if (numerics == CIRC_SFPU) mg = mg * damping;
                float rn = u2f(f2u(mg) | ((par ^ neg[d]) << 31));
                float rs = store_r(mode, rn);
                L[vn[d]] = store_L(mode, q[d] + (numerics == CIRC_SFPU ? rs : rn));
                rm[d] = rs;
            }
        }
        if (stop == CIRC_STOP_GENIE) {
            int errs = 0;
            for (int i = 0; i < n_info; i++) errs += (int)(f2u(L[i]) >> 31);
            if (errs == 0) { stopped = 1; it_used = it + 1; }
        } else if (syndrome_failures_lt0(M, dmax, rows, degs, L) == 0) {
            stopped = 1;
            it_used = it + 1;
        }
    }
    *iters = it_used;
    *synd_fail = syndrome_failures(M, dmax, rows, degs, L);
    int be = 0;
    if (!stopped)
        for (int i = 0; i < n_info; i++)
            be += stop == CIRC_STOP_GENIE ? (int)(f2u(L[i]) >> 31) : (L[i] <= 0.0f);
    *bit_errors = be;
    /* the device engine counts a frame error when an unstopped frame has an info error
     * (writer_ncrisc.cpp:333); the stepper when the frame never met the syndrome (:804-806) */
    *frame_error = stop == CIRC_STOP_GENIE ? be > 0 : !stopped;
    return 0;
}

/* ---------------- the reference's channel: xoshiro128+ and the polar method ---------------- */

typedef struct { uint32_t s[4]; } xo128;

static inline uint32_t xo_next(xo128* x) {
    uint32_t* s = x->s;
    const uint32_t result = s[0] + s[3];
    const uint32_t t = s[1] << 9;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 11) | (s[3] >> 21);
    return result;
}

/* Jump polynomials of xoshiro128+ (2^64 and 2^96 steps), ldpc_decoder_core.h:52-64 and
 * ldpc_sim_scalar.cpp:93-105: the published constants of the generator. */
static void xo_jump_poly(xo128* x, const uint32_t poly[4]) {
    uint32_t a = 0, b = 0, c = 0, d = 0;
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 32; k++) {
            if (poly[i] & (1u << k)) { a ^= x->s[0]; b ^= x->s[1]; c ^= x->s[2]; d ^= x->s[3]; }
            xo_next(x);
        }
    x->s[0] = a; x->s[1] = b; x->s[2] = c; x->s[3] = d;
}
static const uint32_t XO_JUMP[4] = {0x8764000b, 0xf542d2d3, 0x6fa035c3, 0x77f2db5b};
static const uint32_t XO_LONG_JUMP[4] = {0xb523952e, 0x0b6f099f, 0xccf5a0ef, 0x1c580662};

void oracle_xo_jump(uint32_t* s, int n_jumps, int n_long_jumps) {
    xo128 x; memcpy(x.s, s, 16);
    for (int i = 0; i < n_long_jumps; i++) xo_jump_poly(&x, XO_LONG_JUMP);
    for (int i = 0; i < n_jumps; i++) xo_jump_poly(&x, XO_JUMP);
    memcpy(s, x.s, 16);
}

/* Root state of the reference engine: splitmix32 seeding (ldpc_sim_scalar.cpp:46-63). */
void oracle_xo_seed(uint32_t seed, uint32_t* s) {
    uint32_t sm = seed;
    for (int i = 0; i < 4; i++) {
        uint32_t z = (sm += 0x9e3779b9u);
        z ^= z >> 16; z *= 0x21f0aaadu;
        z ^= z >> 15; z *= 0x735a2d97u;
        z ^= z >> 15;
        s[i] = z;
    }
    if ((s[0] | s[1] | s[2] | s[3]) == 0) s[0] = 1;
}

/* fast_ln / fast_rsqrt of the reference (ldpc_decoder_core.h:94-125): its own minimax polynomial
 * and two Newton steps. */
static inline float ref_fast_ln(float s) {
    uint32_t u = f2u(s);
    int32_t ex = (int32_t)((u >> 23) & 0xFF) - 127;
    u = (u & 0x007FFFFFu) | 0x3F800000u;
    float m = u2f(u) - 1.0f;
    float p = -0.02397957f;
    p = p * m + 0.10150005f;
    p = p * m - 0.21029369f;
    p = p * m + 0.32529514f;
    p = p * m - 0.49937260f;
    p = p * m + 0.99999183f;
    p = p * m;
    return (float)ex * 0.69314718056f + p;
}
static inline float ref_fast_rsqrt(float x) {
    uint32_t u = 0x5F3759DFu - (f2u(x) >> 1);
    float y = u2f(u);
    float xh = 0.5f * x;
    y = y * (1.5f - xh * y * y);
    y = y * (1.5f - xh * y * y);
    return y;
}

/* generate_awgn_llr_pair, ldpc_decoder_core.h:128-152. */
static inline void ref_awgn_pair(xo128* x, float mu, float sigma, float* l0, float* l1) {
    const float K = 4.656612875245797e-10f;
    float v1, v2, s;
    do {
        int32_t u1 = (int32_t)xo_next(x);
        int32_t u2 = (int32_t)xo_next(x);
        v1 = (float)u1 * K;
        v2 = (float)u2 * K;
        s = v1 * v1 + v2 * v2;
    } while (s >= 1.0f || s <= 1e-15f);
    float rs = ref_fast_rsqrt(s);
    float inv_s = rs * rs;
    float n2 = -2.0f * ref_fast_ln(s);
    float arg = n2 * inv_s;
    float factor = arg * ref_fast_rsqrt(arg);
    *l0 = mu + sigma * (v1 * factor);
    *l1 = mu + sigma * (v2 * factor);
}

/*
 * Channel LLRs of one codeword PAIR exactly as run_ldpc_worker draws them
 * (ldpc_decoder_core.h:262-292): per position pair, one polar pair for codeword 0, then one for
 * codeword 1.  Writes raw (unquantised, unclipped) fp32 LLRs: llr0/llr1 [ntx] (ntx even).
 * sigma <= 0 gives mu everywhere (:284-291; the clip to l_max is the caller's).
 * Updates the generator state in s.
 */
void oracle_ref_channel_pair(uint32_t* s, float mu, float sigma, int ntx, float* llr0, float* llr1) {
    xo128 x; memcpy(x.s, s, 16);
    if (sigma > 0.0f) {
        for (int i = 0; i < ntx; i += 2) {
            ref_awgn_pair(&x, mu, sigma, &llr0[i], &llr0[i + 1]);
            ref_awgn_pair(&x, mu, sigma, &llr1[i], &llr1[i + 1]);
        }
    } else {
        for (int i = 0; i < ntx; i++) { llr0[i] = mu; llr1[i] = mu; }
    }
    memcpy(s, x.s, 16);
}

/* ---------------- Philox-4x32-10 (Salmon et al., SC'11) and Box-Muller ---------------- */

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/*
 * Uniform pair -> Gaussian pair exactly as the GPU channel does it, in double precision (the GPU
 * uses fast fp32 hardware approximations of log, sqrt, sin and cos; tests compare with a
 * tolerance).  u1 = x0*2^-32 + 2^-33 in (0, 1], angle = 2*pi*(x1*2^-32) - pi.
 */
void oracle_box_muller(uint32_t x0, uint32_t x1, double* n0, double* n1) {
    double u1 = (double)x0 * 2.3283064365386963e-10 + 1.1641532182693481e-10;
    double a = (double)x1 * 2.3283064365386963e-10 * 6.283185307179586 - 3.141592653589793;
    double rad = sqrt(-2.0 * log(u1));
    *n0 = rad * cos(a);
    *n1 = rad * sin(a);
}

/* ---------------- whole-path Monte Carlo with the reference's channel (CPU baseline "port") ---- */

/*
 * Runs n_pairs codeword pairs exactly as one reference worker does (ldpc_decoder_core.h:258-578):
 * generator state s (advanced in place), BF16 storage, Approximate-Min*, no clips.
 * Accumulates frames, bit errors, frame errors, iteration sum (both codewords) into tally[4].
 */
void oracle_mc_pairs(int N, int M, int P, int dmax, const int32_t* rows, const int32_t* degs,
                     int max_iter, float mu, float sigma, uint32_t* s, int n_pairs,
                     float* scratch /* 2*ntx + N + M*dmax floats */, uint64_t* tally) {
    const int ntx = N - P;
    float* l0 = scratch;
    float* l1 = l0 + ntx;
    float* post = l1 + ntx;
    float* rw = post + N;
    for (int p = 0; p < n_pairs; p++) {
        oracle_ref_channel_pair(s, mu, sigma, ntx, l0, l1);
        for (int c = 0; c < 2; c++) {
            int32_t it, sf, be;
            oracle_decode(N, M, P, dmax, rows, degs, STORE_BF16, ALGO_AMIN, max_iter, 0.0f, 0.0f, 0.0f,
                          c ? l1 : l0, post, rw, &it, &sf, &be);
            tally[0] += 1;
            tally[1] += (uint64_t)be;
            tally[2] += be > 0;
            tally[3] += (uint64_t)it;
        }
    }
}
