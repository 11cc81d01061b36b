// Layered decoder for quasi-cyclic AR4JA codes on sm_100a: channel generation, row-layered
// Approximate-Min* (or normalised min-sum) decoding with syndrome stop, and error tallies, in one
// persistent kernel.
//
// Code structure (see ldpcb200/ar4ja.py): 12 layers of Z rows; layers 0-3 have degree 3, layers 4-11
// degree D; row j of layer l checks columns blk_off[l][e] + ((j + shift[l][e]) mod Z) for its edges e
// in ascending column order.  Rows inside a layer share no column, so the Z rows of a layer are
// updated at once and the result equals the reference's serial row loop
// (engines/scalar_5w/ldpc_decoder_core.h:311-522) bit for bit.
//
// Mapping.  One CTA of T = Z/R threads owns F frame slots.  Thread t updates rows t, t+T, ... of
// every layer (R rows), for all F slots in lockstep:
//   * L (posterior LLRs, N per slot) lives in shared memory: bf16 in the reference-numerics mode,
//     fp32 otherwise;
//   * the check-to-variable messages r of the thread's own rows never leave registers: 12 layers x R
//     rows x F slots x degree values, as packed 16-bit pairs (bf16 / fp16 storage) or fp32;
//   * the circulant shift is the address rotation (j + shift) & (Z-1) into the shared L array;
//   * after each iteration from the third on, hard decisions are packed with warp ballots and the
//     syndrome of each 32-row word is the XOR of the edge blocks' bit vectors rotated by their shifts
//     (funnel shifts), i.e. 12*Z/32 words per frame instead of one parity per row.
// A slot whose frame converges (or reaches max_iter) is tallied and refilled at once from a global
// frame counter: early-retire with slot refill, so fast and slow frames never wait for each other.
#pragma once
#include <cstdint>
#include <type_traits>
#include "ar4ja_fixed_tables.h"
#include "ldpc_device.cuh"

namespace ldpcb200 {

constexpr int QC_LAYERS = 12;
constexpr int QC_DEG_LOW = 3;  // degree of layers 0-3 (block row 0 of every AR4JA code)
constexpr int QC_DMAX = 18;
constexpr int QC_MAX_F = 4;

// Kernel arguments (one copy in the constant parameter bank; every descriptor read is a constant
// operand, not a memory instruction).
struct QcParams {
    int32_t blk_off[QC_LAYERS][QC_DMAX];  // column block * Z of edge e of layer l
    int32_t shift[QC_LAYERS][QC_DMAX];    // circulant shift of edge e of layer l
    int32_t n_vars;                       // N
    int32_t n_tx;                         // N - P: the transmitted prefix
    int32_t max_iter;
    float mu, sigma;                      // channel LLR mean and standard deviation
    float l_max, r_max, l_post_max;       // clips (0 = off)
    uint32_t seed_lo, seed_hi, stream;
    uint64_t first_frame;                 // global index of this launch's frame 0
    uint32_t n_frames;
    const float* llr_in;                  // external channel LLRs [n_frames][n_tx] (or null)
    float* post_out;                      // [n_frames][N] posteriors (optional)
    int32_t* iters_out;                   // [n_frames] (optional)
    int32_t* synd_out;                    // [n_frames] failing rows after decoding (optional)
    int32_t* be_out;                      // [n_frames] bit errors (optional)
    unsigned long long* tally;            // [TALLY_WORDS]
    unsigned long long* hist;             // [hist_bins] iterations histogram (optional)
    int32_t hist_bins;
    unsigned int* work;                   // frame claim counter, zero at launch
    void* r_base;                         // messages in global memory (RG kernels): [slot][edges]
    int32_t layer_off[QC_LAYERS];         // element offset of layer l's messages in a slot ([pair][row])
    int32_t slot_elems;                   // message elements per slot (edges, odd degrees padded)
    float ebn0_lo, ebn0_hi;               // per-frame Eb/N0 range in dB (used when hi > lo)
    float rate;                           // (N - M) / (N - P), for the per-frame mu and sigma
    unsigned long long* snr_bins;         // [4][SNR_BINS]: frames, frame errors, bit errors, iterations
    // weighted Approximate-Min* (ALGO_WAMIN): check output sign * max(alpha * m - beta, 0)
    // (alpha, beta) per iteration and edge slot: [w_iters][w_slots], edge e of layer l at slot
    // qc_edge_slot(l, e, D); iteration t uses row min(t, w_iters - 1).  ALGO_WROW: one pair per
    // iteration and layer, [w_iters][12].  Both test the syndrome from the first iteration on.
    const float2* wtab;
    int32_t w_iters, w_slots;
    // ALGO_CIRC stop rule and tally (the circulant engine's): QC_STOP_SYNDROME tests the syndrome
    // after every iteration; QC_STOP_GENIE stops a frame once none of its info positions
    // 0..n_info-1 has the sign bit set (the engine on silicon).  Other algorithms follow the
    // reference engine: syndrome from the third iteration on, bit errors over the first N-P positions.
    int32_t stop_rule;
    int32_t n_info;
    // ALGO_CIRC: the min* constants (c1, k1, c2, k2), the damping factor, and the arithmetic form
    // (circ_sfpu = 1: q and r rounded to storage before use, as the SFPU kernels do)
    float circ_c[4];
    float circ_damping;
    int32_t circ_sfpu;
};

enum QcStop : int { QC_STOP_SYNDROME = 0, QC_STOP_GENIE = 1 };

// Slot of edge e of layer l in a per-iteration row of the weight table: layers 0-3 (degree 3) first.
__host__ __device__ constexpr int qc_edge_slot(int l, int e, int D) {
    return l < 4 ? QC_DEG_LOW * l + e : QC_DEG_LOW * 4 + D * (l - 4) + e;
}

enum TallyWord : int {
    T_FRAMES = 0, T_BIT_ERR, T_FRAME_ERR, T_ITER_SUM, T_UNCONVERGED, T_MAX_ITER, T_BIT_ERR_SQ, TALLY_WORDS = 8
};

template <int MODE> struct LTraits;
template <> struct LTraits<STORE_BF16> {
    using T = uint16_t;
    static __device__ __forceinline__ float ld(const T* s, int i) { return __uint_as_float(uint32_t(s[i]) << 16); }
    static __device__ __forceinline__ void st(T* s, int i, float v) { s[i] = __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
    static __device__ __forceinline__ uint32_t sign(const T* s, int i) { return uint32_t(s[i]) >> 15; }
    static __device__ __forceinline__ float round_ch(float v) { return bf16_round(v); }
};
template <> struct LTraits<STORE_FP32> {
    using T = float;
    static __device__ __forceinline__ float ld(const T* s, int i) { return s[i]; }
    static __device__ __forceinline__ void st(T* s, int i, float v) { s[i] = v; }
    static __device__ __forceinline__ uint32_t sign(const T* s, int i) { return __float_as_uint(s[i]) >> 31; }
    static __device__ __forceinline__ float round_ch(float v) { return v; }
};
template <> struct LTraits<STORE_FP16> : LTraits<STORE_FP32> {};

// Check messages as stored in memory (one element per edge), for kernels that keep them there.
template <int MODE> struct RTraits;
template <> struct RTraits<STORE_BF16> {
    using T = uint16_t;
    static __device__ __forceinline__ float ld(const T* p) { return __uint_as_float(uint32_t(*p) << 16); }
    static __device__ __forceinline__ void st(T* p, float v) { *p = __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
};
template <> struct RTraits<STORE_FP32> {
    using T = float;
    static __device__ __forceinline__ float ld(const T* p) { return *p; }
    static __device__ __forceinline__ void st(T* p, float v) { *p = v; }
};
template <> struct RTraits<STORE_FP16> {
    using T = uint16_t;
    static __device__ __forceinline__ float ld(const T* p) { return __half2float(__ushort_as_half(*p)); }
    static __device__ __forceinline__ void st(T* p, float v) {
        *p = __half_as_ushort(__float2half_rn(fminf(fmaxf(v, -65504.0f), 65504.0f)));
    }
};

// Messages of one row in registers.
template <int d, int MODE> struct RowMsg {  // 16-bit storage: pairs packed in 32-bit words
    uint32_t w[(d + 1) / 2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < (d + 1) / 2; ++i) w[i] = 0u;
    }
    __device__ __forceinline__ float get(int e) const {
        const uint32_t x = w[e >> 1];
        if (MODE == STORE_BF16) return (e & 1) ? __uint_as_float(x & 0xFFFF0000u) : __uint_as_float(x << 16);
        const __half2 h = *reinterpret_cast<const __half2*>(&x);
        return (e & 1) ? __high2float(h) : __low2float(h);
    }
    __device__ __forceinline__ void set2(int e, float a, float b) {  // e even: edges e and e+1
        uint32_t x;
        if (MODE == STORE_BF16) {
            __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
            x = *reinterpret_cast<uint32_t*>(&v);
        } else {
            a = fminf(fmaxf(a, -65504.0f), 65504.0f);
            b = fminf(fmaxf(b, -65504.0f), 65504.0f);
            __half2 v = __floats2half2_rn(a, b);
            x = *reinterpret_cast<uint32_t*>(&v);
        }
        w[e >> 1] = x;
    }
};
template <int d> struct RowMsg<d, STORE_FP32> {
    float v[d];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < d; ++i) v[i] = 0.0f;
    }
    __device__ __forceinline__ float get(int e) const { return v[e]; }
    __device__ __forceinline__ void set2(int e, float a, float b) {
        v[e] = a;
        if (e + 1 < d) v[e + 1] = b;
    }
};

// Messages of one row kept in global memory (RG kernels).  Edges 2k and 2k+1 of a row share one
// 32-bit word (16-bit storage) or one float2 (fp32), pair k at w[k * stride]: a slot's messages are
// laid out [layer][pair][row], so the threads of a CTA (consecutive rows) touch consecutive words
// and a row's two edges cost one load and one store.  An odd degree's last pair holds a zero.
template <int d, int MODE> struct RowMsgGlobal {
    using W = typename std::conditional<MODE == STORE_FP32, float2, uint32_t>::type;
    W* w;
    int stride;
    __device__ __forceinline__ float get(int e) const {
        const W x = w[(e >> 1) * stride];
        if constexpr (MODE == STORE_FP32) {
            return (e & 1) ? x.y : x.x;
        } else if constexpr (MODE == STORE_BF16) {
            return (e & 1) ? __uint_as_float(x & 0xFFFF0000u) : __uint_as_float(x << 16);
        } else {
            const __half2 h = *reinterpret_cast<const __half2*>(&x);
            return (e & 1) ? __high2float(h) : __low2float(h);
        }
    }
    __device__ __forceinline__ void set2(int e, float a, float b) {  // e even: edges e and e+1
        W x;
        if constexpr (MODE == STORE_FP32) {
            x = make_float2(a, b);
        } else if constexpr (MODE == STORE_BF16) {
            __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
            x = *reinterpret_cast<uint32_t*>(&v);
        } else {
            a = fminf(fmaxf(a, -65504.0f), 65504.0f);
            b = fminf(fmaxf(b, -65504.0f), 65504.0f);
            __half2 v = __floats2half2_rn(a, b);
            x = *reinterpret_cast<uint32_t*>(&v);
        }
        w[(e >> 1) * stride] = x;
    }
};
// Row j of layer ly in message slot `slot` (Z rows per layer).
template <int d, int MODE, int Z>
__device__ __forceinline__ RowMsgGlobal<d, MODE> rg_row(const QcParams& p, size_t slot, int ly, int j) {
    using W = typename RowMsgGlobal<d, MODE>::W;
    auto* base = reinterpret_cast<typename RTraits<MODE>::T*>(p.r_base) + slot * p.slot_elems + p.layer_off[ly];
    return RowMsgGlobal<d, MODE>{reinterpret_cast<W*>(base) + j, Z};
}

// Update one row of degree d for the F slots (all slots in lockstep; slot f's L array at
// sL + f*lstride).  idx[e]: the row's column indices.
// ALGO_WAMIN: wt[f] points at the (alpha, beta) pairs of this layer's edges for slot f's current
// iteration (edge e at wt[f][e]: a constant offset, no class lookup).  ALGO_WROW: wt[f][0] is the
// layer's one pair, applied to the row's two magnitudes before they are spread over the edges (the
// same values as ALGO_WAMIN with that pair on every edge, at two multiplies per row instead of one
// per edge).
// BO: idx[e] holds byte offsets into the slot's L array instead of element indices (the column
// offset table of the OT layout), so no index scaling is needed.
// PAD: rows of a smaller degree padded to d with edges whose posterior is the largest finite value
// (the general step kernel): such an edge is never the minimum and a min* step with it returns the
// other operand unchanged, so only a row with fewer than two real edges needs care: its chain over
// the other edges then holds no real value (above 1e38), and the reference's m_others is the row's
// minimum (ldpc_decoder_core.h:180-181).
template <int d, int MODE, int ALGO, bool CLIP, int F, class MSG, bool BO = false, bool PAD = false>
__device__ __forceinline__ void row_update(const int (&idx)[d], typename LTraits<MODE>::T* sL, int lstride,
                                           MSG (&rm)[F], float r_cap, float lp_cap,
                                           const float2* const* wt = nullptr) {
    using LT = LTraits<MODE>;
    using LE = typename LT::T;
    auto lptr = [&](int f, int e) -> LE* {
        if constexpr (BO) return reinterpret_cast<LE*>(reinterpret_cast<char*>(sL + f * lstride) + idx[e]);
        else return sL + f * lstride + idx[e];
    };
    float q[F][d];
#pragma unroll
    for (int f = 0; f < F; ++f)
#pragma unroll
        for (int e = 0; e < d; ++e) q[f][e] = __fsub_rn(LT::ld(lptr(f, e), 0), rm[f].get(e));

#pragma unroll
    for (int f = 0; f < F; ++f) {
        uint32_t par = 0;
#pragma unroll
        for (int e = 0; e < d; ++e) par ^= __float_as_uint(q[f][e]);
        par &= 0x80000000u;
        float a[d];
#pragma unroll
        for (int e = 0; e < d; ++e) a[e] = fabsf(q[f][e]);
        // is_am[e]: edge e is the argmin of |q| with a strict < from the reference's initial values
        // (9999 for Approximate-Min*, 999 for min-sum), the first minimum winning.
        bool is_am[d];
        float mag_min, mag_all;
        if (ALGO == ALGO_AMIN || algo_weighted(ALGO)) {
            // Prefix minima pm_i = min(9999, |q_0|, .., |q_i|); mn = pm_{d-1}.  The argmin index am is
            // the first i with |q_i| = mn, so i < am exactly when pm_i > mn: up to degree 10 no index
            // is tracked.
            // The other edges in row order are o_i = |q_i| for i < am and |q_{i+1}| after it, and the
            // recursive min* (ldpc_decoder_core.h:176-201) over them takes d-2 steps, then one final
            // step with mn (d-1 steps in all).
            float mn;
            bool lt[d];  // lt[i] = (i < am)
            if constexpr (d > 10) {
                // Degree 18: the argmin as an integer (the first strict minimum), each flag one
                // integer compare where it is used.  Seventeen prefix-minimum flags do not fit the
                // predicate registers and were packed into and tested out of general registers:
                // +4-5 % on the rate-4/5 kernels, fewer spills at 64 registers; at degree 10 the
                // prefix form stays faster (r2/3 K=1024 26.0 against 25.2 M frames/s).
                float m1 = 9999.0f;
                int am = 0;
#pragma unroll
                for (int e = 0; e < d; ++e) {
                    am = a[e] < m1 ? e : am;
                    m1 = fminf(m1, a[e]);
                }
                mn = m1;
#pragma unroll
                for (int i = 0; i < d; ++i) lt[i] = (i + 1 < d) ? (i < am) : false;
            } else {
                float pm[d];
                pm[0] = fminf(a[0], 9999.0f);
#pragma unroll
                for (int e = 1; e < d; ++e) pm[e] = fminf(pm[e - 1], a[e]);
                mn = pm[d - 1];
#pragma unroll
                for (int i = 0; i < d; ++i) lt[i] = (i + 1 < d) ? (pm[i] > mn) : false;
            }
#pragma unroll
            for (int e = 0; e < d; ++e) is_am[e] = (e == 0 ? true : lt[e - 1]) && !lt[e];
            float m = fabsf(lt[0] ? q[f][0] : q[f][1]);
#pragma unroll
            for (int i = 1; i + 1 < d; ++i) m = amin_step_fma(m, fabsf(lt[i] ? q[f][i] : q[f][i + 1]));
            if (PAD) m = m > 1e38f ? mn : m;
            mag_min = m;
            mag_all = amin_step_fma(m, mn);
        } else {
            // normalised min-sum, alpha = 0.75 (ldpc_decoder_core.h:322-379)
            int am = 0;
            float m1 = 999.0f, m2 = 999.0f;
#pragma unroll
            for (int e = 0; e < d; ++e) {
                const bool l1 = a[e] < m1, l2 = a[e] < m2;
                m2 = l1 ? m1 : (l2 ? a[e] : m2);
                am = l1 ? e : am;
                m1 = l1 ? a[e] : m1;
            }
#pragma unroll
            for (int e = 0; e < d; ++e) is_am[e] = (e == am);
            mag_min = __fmul_rn(0.75f, m2);
            mag_all = __fmul_rn(0.75f, m1);
        }
        if (CLIP) {
            mag_min = fminf(mag_min, r_cap);
            mag_all = fminf(mag_all, r_cap);
        }
        if (ALGO == ALGO_WROW) {  // max(alpha * m - beta, 0) once per row
            const float2 w = wt[f][0];
            const float zmin = __fsub_rn(__fmul_rn(w.x, mag_min), w.y);
            const float zall = __fsub_rn(__fmul_rn(w.x, mag_all), w.y);
            mag_min = zmin > 0.0f ? zmin : 0.0f;
            mag_all = zall > 0.0f ? zall : 0.0f;
        }
        // r_e = +-mag with sign parity ^ sign(q_e): fold the parity into the magnitudes once.
        const uint32_t smin = __float_as_uint(mag_min) | par;
        const uint32_t sall = __float_as_uint(mag_all) | par;
        float rn[d];
#pragma unroll
        for (int e = 0; e < d; ++e) {
            uint32_t sel = is_am[e] ? smin : sall;
            if (ALGO == ALGO_WAMIN) {  // max(alpha * m - beta, 0): alpha = 1, beta = 0 leaves m unchanged
                const float2 w = wt[f][e];
                const float z = __fsub_rn(__fmul_rn(w.x, is_am[e] ? mag_min : mag_all), w.y);
                sel = __float_as_uint(z > 0.0f ? z : 0.0f) | par;
            }
            rn[e] = __uint_as_float(sel ^ (__float_as_uint(q[f][e]) & 0x80000000u));
            float ln = __fadd_rn(q[f][e], rn[e]);
            if (CLIP) ln = fminf(fmaxf(ln, -lp_cap), lp_cap);
            LT::st(lptr(f, e), 0, ln);
        }
#pragma unroll
        for (int e = 0; e < d; e += 2) rm[f].set2(e, rn[e], (e + 1 < d) ? rn[e + 1] : 0.0f);
    }
}

// Storage rounding of a check message (what RowMsg::set2 / RTraits::st keep).
template <int MODE> __device__ __forceinline__ float msg_round(float v) {
    if constexpr (MODE == STORE_BF16) return bf16_round(v);
    else if constexpr (MODE == STORE_FP16) return fp16_round_sat(v);
    else return v;
}

// ALGO_CIRC: one row of the circulant engine's decoder (degree 3 or 6; edges in ascending column
// order).  The degree-6 magnitudes come from the pairwise min* tree of
// tests/test_circulant_dma_stepper.cpp:404-425 and engines/circulant_dma_4cw/compute_trisc.cpp:
// 370-460: m03 = g(a0, a3), m14 = g(a1, a4), m25 = g(a2, a5); edge 0 gets g(g(m14, m25), a3), edge 3
// g(g(m14, m25), a0), and likewise for the pairs (1, 4) and (2, 5); a degree-3 row gives each edge g
// of the other two (:436-446).  Each magnitude is scaled by the damping factor, signed with the
// parity of the other edges, and r and L are stored with the storage rounding.  SFPU form
// (cs.sfpu): q is rounded to storage first and L = store(q + store(r)) (compute_trisc.cpp:351-360,
// 387-395); scalar form: L = store(q + r) with r unrounded (test_circulant_dma_stepper.cpp:452-456).
struct CircRt {
    CircConsts k;
    float damping;
    bool sfpu;
};
template <int d, int MODE, int F, class MSG, bool BO = false>
__device__ __forceinline__ void row_update_circ(const int (&idx)[d], typename LTraits<MODE>::T* sL, int lstride,
                                                MSG (&rm)[F], const CircRt& cr) {
    static_assert(d == 3 || d == 6, "the circulant engine's rows have degree 3 or 6");
    using LT = LTraits<MODE>;
    using LE = typename LT::T;
    auto lptr = [&](int f, int e) -> LE* {
        if constexpr (BO) return reinterpret_cast<LE*>(reinterpret_cast<char*>(sL + f * lstride) + idx[e]);
        else return sL + f * lstride + idx[e];
    };
#pragma unroll
    for (int f = 0; f < F; ++f) {
        float q[d], a[d], mag[d];
        uint32_t par = 0;
#pragma unroll
        for (int e = 0; e < d; ++e) {
            q[e] = __fsub_rn(LT::ld(lptr(f, e), 0), rm[f].get(e));
            if (cr.sfpu) q[e] = LT::round_ch(q[e]);
            par ^= __float_as_uint(q[e]);
            a[e] = fabsf(q[e]);
        }
        par &= 0x80000000u;
        if constexpr (d == 6) {
            const float m03 = circ_g(a[0], a[3], cr.k), m14 = circ_g(a[1], a[4], cr.k), m25 = circ_g(a[2], a[5], cr.k);
            const float o0 = circ_g(m14, m25, cr.k), o1 = circ_g(m03, m25, cr.k), o2 = circ_g(m03, m14, cr.k);
            mag[0] = circ_g(o0, a[3], cr.k);
            mag[3] = circ_g(o0, a[0], cr.k);
            mag[1] = circ_g(o1, a[4], cr.k);
            mag[4] = circ_g(o1, a[1], cr.k);
            mag[2] = circ_g(o2, a[5], cr.k);
            mag[5] = circ_g(o2, a[2], cr.k);
        } else {
            mag[0] = circ_g(a[1], a[2], cr.k);
            mag[1] = circ_g(a[0], a[2], cr.k);
            mag[2] = circ_g(a[0], a[1], cr.k);
        }
        float rn[d];
#pragma unroll
        for (int e = 0; e < d; ++e) {
            rn[e] = __uint_as_float(__float_as_uint(__fmul_rn(mag[e], cr.damping)) |
                                    (par ^ (__float_as_uint(q[e]) & 0x80000000u)));
            const float rs = msg_round<MODE>(rn[e]);
            LT::st(lptr(f, e), 0, __fadd_rn(q[e], cr.sfpu ? rs : rn[e]));
        }
#pragma unroll
        for (int e = 0; e < d; e += 2) rm[f].set2(e, rn[e], (e + 1 < d) ? rn[e + 1] : 0.0f);
    }
}

// ------------------------------------------------------------------------------------------------
// Paired mode: two frame slots per thread in lockstep, interleaved per variable in shared memory
// (element i of slot f at index 2i + f), so one address, one shared-memory access and one packed
// f32x2 instruction (FFMA2/FADD2/FMUL2) serve both frames.  Messages stay in registers, one 32-bit
// word per edge holding both frames' 16-bit values (bf16 or fp16).  Results equal the unpaired
// kernel bit for bit: every packed operation rounds each lane exactly like its scalar form.

template <int d, int MODE> struct RowMsgPair {  // w[e]: slot 0 in bits 15:0, slot 1 in bits 31:16
    uint32_t w[d];
    __device__ __forceinline__ void zero_slot(int f) {
#pragma unroll
        for (int e = 0; e < d; ++e) w[e] &= f ? 0x0000FFFFu : 0xFFFF0000u;
    }
    __device__ __forceinline__ float2 get2(int e) const {
        const uint32_t x = w[e];
        if (MODE == STORE_BF16) return make_float2(__uint_as_float(x << 16), __uint_as_float(x & 0xFFFF0000u));
        return __half22float2(*reinterpret_cast<const __half2*>(&x));
    }
    __device__ __forceinline__ void set2(int e, float2 v) {
        uint32_t x;
        if (MODE == STORE_BF16) {
            __nv_bfloat162 b = __floats2bfloat162_rn(v.x, v.y);
            x = *reinterpret_cast<uint32_t*>(&b);
        } else {  // IEEE fp16 with saturation at +-65504, both lanes in one conversion
            asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(x) : "f"(v.y), "f"(v.x));
        }
        w[e] = x;
    }
};

template <int MODE> __device__ __forceinline__ float2 ld_pair(const typename LTraits<MODE>::T* sL, int i) {
    if constexpr (MODE == STORE_BF16) {
        const uint32_t x = reinterpret_cast<const uint32_t*>(sL)[i];
        return make_float2(__uint_as_float(x << 16), __uint_as_float(x & 0xFFFF0000u));
    } else {
        return reinterpret_cast<const float2*>(sL)[i];
    }
}
template <int MODE> __device__ __forceinline__ void st_pair(typename LTraits<MODE>::T* sL, int i, float2 v) {
    if constexpr (MODE == STORE_BF16) {
        __nv_bfloat162 b = __floats2bfloat162_rn(v.x, v.y);
        reinterpret_cast<uint32_t*>(sL)[i] = *reinterpret_cast<uint32_t*>(&b);
    } else {
        reinterpret_cast<float2*>(sL)[i] = v;
    }
}

// amin_step_fma's result on two independent lanes, with the correction chosen by two saturated
// flags, f05 = [diff < 0.5] and f2 = [diff < 2], so that every operation but the flags is a packed
// f32x2 instruction: t = cur - c1 f05, u = t - c2 (f2 - f05), each subtracting c1, c2 or nothing
// exactly once.  m, a >= 0 and finite.  diff = max(m,a) - min(m,a) is |m - a| exactly; c1n = 0.4 diff - 0.69315 and
// c2n = 0.328 (diff - 0.5) - 0.49315 are the negated corrections (round-to-nearest is symmetric;
// the product as one fused multiply-add, as in amin_step_fma).
__device__ __forceinline__ float2 amin_step_pair(float2 m, float2 a) {
    const float2 one = make_float2(1.0f, 1.0f), neg1 = make_float2(-1.0f, -1.0f);
    const float2 cur = make_float2(fminf(m.x, a.x), fminf(m.y, a.y));
    const float2 mx = make_float2(fmaxf(m.x, a.x), fmaxf(m.y, a.y));
    const float2 diff = __ffma2_rn(cur, neg1, mx);
    const float2 c1n = __ffma2_rn(__fmul2_rn(diff, make_float2(0.40f, 0.40f)), one, make_float2(-0.69315f, -0.69315f));
    const float2 c2n = __ffma2_rn(__ffma2_rn(diff, make_float2(AMIN_K2, AMIN_K2),
                                             make_float2(-0.5f * AMIN_K2, -0.5f * AMIN_K2)),
                                  one, make_float2(-0.49315f, -0.49315f));
    const float2 f05 = make_float2(__saturatef(__fmaf_rn(diff.x, -1073741824.0f, 536870912.0f)),
                                   __saturatef(__fmaf_rn(diff.y, -1073741824.0f, 536870912.0f)));
    const float2 f2 = make_float2(__saturatef(__fmaf_rn(diff.x, -1073741824.0f, 2147483648.0f)),
                                  __saturatef(__fmaf_rn(diff.y, -1073741824.0f, 2147483648.0f)));
    const float2 g = __ffma2_rn(f05, neg1, f2);
    const float2 t = __ffma2_rn(c1n, f05, cur);
    const float2 u = __ffma2_rn(c2n, g, t);
    return make_float2(fmaxf(u.x, 0.0f), fmaxf(u.y, 0.0f));
}

// One row of degree d for both slots of a pair (Approximate-Min*, no clips).
template <int d, int MODE>
__device__ __forceinline__ void row_update_pair(const int (&idx)[d], typename LTraits<MODE>::T* sL,
                                                RowMsgPair<d, MODE>& rm) {
    float2 q[d];
#pragma unroll
    for (int e = 0; e < d; ++e) q[e] = __ffma2_rn(rm.get2(e), make_float2(-1.0f, -1.0f), ld_pair<MODE>(sL, idx[e]));
    uint32_t par0 = 0, par1 = 0;
#pragma unroll
    for (int e = 0; e < d; ++e) {
        par0 ^= __float_as_uint(q[e].x);
        par1 ^= __float_as_uint(q[e].y);
    }
    par0 &= 0x80000000u;
    par1 &= 0x80000000u;
    float pm0[d], pm1[d];
    pm0[0] = fminf(fabsf(q[0].x), 9999.0f);
    pm1[0] = fminf(fabsf(q[0].y), 9999.0f);
#pragma unroll
    for (int e = 1; e < d; ++e) {
        pm0[e] = fminf(pm0[e - 1], fabsf(q[e].x));
        pm1[e] = fminf(pm1[e - 1], fabsf(q[e].y));
    }
    const float2 mn = make_float2(pm0[d - 1], pm1[d - 1]);
    bool lt0[d], lt1[d];
#pragma unroll
    for (int i = 0; i < d; ++i) {
        lt0[i] = (i + 1 < d) ? (pm0[i] > mn.x) : false;
        lt1[i] = (i + 1 < d) ? (pm1[i] > mn.y) : false;
    }
    float2 m = make_float2(fabsf(lt0[0] ? q[0].x : q[1].x), fabsf(lt1[0] ? q[0].y : q[1].y));
#pragma unroll
    for (int i = 1; i + 1 < d; ++i)
        m = amin_step_pair(m, make_float2(fabsf(lt0[i] ? q[i].x : q[i + 1].x), fabsf(lt1[i] ? q[i].y : q[i + 1].y)));
    const float2 mall = amin_step_pair(m, mn);
    const uint32_t smin0 = __float_as_uint(m.x) | par0, sall0 = __float_as_uint(mall.x) | par0;
    const uint32_t smin1 = __float_as_uint(m.y) | par1, sall1 = __float_as_uint(mall.y) | par1;
#pragma unroll
    for (int e = 0; e < d; ++e) {
        const bool am0 = (e == 0 ? true : lt0[e - 1]) && !lt0[e];
        const bool am1 = (e == 0 ? true : lt1[e - 1]) && !lt1[e];
        const float2 rn = make_float2(__uint_as_float((am0 ? smin0 : sall0) ^ (__float_as_uint(q[e].x) & 0x80000000u)),
                                      __uint_as_float((am1 ? smin1 : sall1) ^ (__float_as_uint(q[e].y) & 0x80000000u)));
        st_pair<MODE>(sL, idx[e], __fadd2_rn(q[e], rn));
        rm.set2(e, rn);
    }
}

// Element i of frame slot f: slot-major (f * lstride + i) or interleaved in pairs (2i + f).
template <int MODE, bool PAIR> struct SlotView {
    typename LTraits<MODE>::T* p;
    __device__ __forceinline__ SlotView(typename LTraits<MODE>::T* base, int f, int lstride)
        : p(PAIR ? base + f : base + (size_t)f * lstride) {}
    __device__ __forceinline__ int at(int i) const { return PAIR ? 2 * i : i; }
    __device__ __forceinline__ float ld(int i) const { return LTraits<MODE>::ld(p, at(i)); }
    __device__ __forceinline__ void st(int i, float v) const { LTraits<MODE>::st(p, at(i), v); }
    __device__ __forceinline__ uint32_t sign(int i) const { return LTraits<MODE>::sign(p, at(i)); }
};

// Registers holding the messages of one CTA's rows: [layer][row][slot] rows, or one pair per row,
// or nothing when the messages live in global memory (RG).
template <int D, int R, int F, int MODE, bool PAIR, bool RG = false> struct MsgRegs {
    RowMsg<QC_DEG_LOW, MODE> r3[4][R][F];
    RowMsg<D, MODE> rD[8][R][F];
    __device__ __forceinline__ void zero_slot(int f) {
#pragma unroll
        for (int l = 0; l < 4; ++l)
#pragma unroll
            for (int rho = 0; rho < R; ++rho) r3[l][rho][f].zero();
#pragma unroll
        for (int l = 0; l < 8; ++l)
#pragma unroll
            for (int rho = 0; rho < R; ++rho) rD[l][rho][f].zero();
    }
};
template <int D, int R, int F, int MODE> struct MsgRegs<D, R, F, MODE, false, true> {
    __device__ __forceinline__ void zero_slot(int) {}
};
template <int D, int R, int F, int MODE> struct MsgRegs<D, R, F, MODE, true, false> {
    RowMsgPair<QC_DEG_LOW, MODE> r3[4];
    RowMsgPair<D, MODE> rD[8];
    __device__ __forceinline__ void zero_slot(int f) {
#pragma unroll
        for (int l = 0; l < 4; ++l) r3[l].zero_slot(f);
#pragma unroll
        for (int l = 0; l < 8; ++l) rD[l].zero_slot(f);
    }
};

// Column offset table (OT layout): for every layer, each thread's byte offsets of its row's columns in
// a slot's L array, stored as vectors of 4, then 2, then 1 offsets per thread ([chunk][thread]), so a
// row's offsets arrive in ceil(d/4) or so vector loads and a circulant read needs no index arithmetic.
__host__ __device__ constexpr int ot_layer_start(int l, int D) { return l < 4 ? QC_DEG_LOW * l : QC_DEG_LOW * 4 + D * (l - 4); }

// Position (in 32-bit words, relative to the layer's region of T * d words) of edge e of thread t.
__device__ __forceinline__ int ot_pos(int d, int e, int t, int T) {
    const int c4 = d & ~3, rem = d & 3;
    if (e < c4) return T * (e & ~3) + 4 * t + (e & 3);
    if (rem >= 2 && e < c4 + 2) return T * c4 + 2 * t + (e - c4);
    return T * (c4 + (rem >= 2 ? 2 : 0)) + t;
}

template <int d, int T>
__device__ __forceinline__ void ot_load(const uint32_t* tab, int t, int* idx) {
    constexpr int c4 = d & ~3, rem = d & 3;
#pragma unroll
    for (int c = 0; c < c4; c += 4) {
        const uint4 v = reinterpret_cast<const uint4*>(tab + T * c)[t];
        idx[c] = (int)v.x;
        idx[c + 1] = (int)v.y;
        idx[c + 2] = (int)v.z;
        idx[c + 3] = (int)v.w;
    }
    if constexpr (rem >= 2) {
        const uint2 v = reinterpret_cast<const uint2*>(tab + T * c4)[t];
        idx[c4] = (int)v.x;
        idx[c4 + 1] = (int)v.y;
    }
    if constexpr (rem & 1) idx[d - 1] = (int)tab[T * (c4 + (rem >= 2 ? 2 : 0)) + t];
}

// Edge e of layer l: column block offset (block * Z) and circulant shift, from the launch parameters
// or, for FIX >= 0, compiled in (the descriptors of code kQcFixedDev[FIX]; in the unrolled layer loop
// they become immediate operands).
template <int FIX>
__device__ __forceinline__ int qc_blk(const QcParams& p, int l, int e) {
    if constexpr (FIX >= 0) return kQcFixedDev[FIX].blk_off[l][e];
    else return p.blk_off[l][e];
}
template <int FIX>
__device__ __forceinline__ int qc_shift(const QcParams& p, int l, int e) {
    if constexpr (FIX >= 0) return kQcFixedDev[FIX].shift[l][e];
    else return p.shift[l][e];
}

// B: resident CTAs per SM the register allocation must allow (0 = the compiler's choice); a larger B
// caps registers per thread at 65536 / (B * Z/R) and trades registers for resident warps.
// PAIR: the paired mode above (F = 2, R = 1, 16-bit storage, Approximate-Min*, no clips).
// RG: messages in global memory (p.r_base, one region of p.slot_elems per slot) instead of
// registers, for codes whose rows per thread times degrees exceed the register file (K = 16384).
// OT: the column offset table above, built once per CTA in shared memory after the hard-decision
// words (T * (12 + 8 D) words); one row per thread.
// FIX: >= 0 for the descriptors of a known code compiled in (layouts 5 and 6; the host offers them
// only for a matrix whose descriptors are those).
// ROLL (layout 7, global messages only): the eight degree-D layers run as one loop that is not
// unrolled, each row's descriptors read from the kernel parameters by layer index.  The unrolled
// body of a degree-18 code is tens of KB of instructions; with one-warp CTAs whose warps are
// each at a different point of it, the instruction fetch stalls the SM.
template <int Z, int D, int R, int F, int MODE, int ALGO, bool CLIP, bool EXT, int B = 0, bool PAIR = false,
          bool RG = false, bool OT = false, int FIX = -1, bool ROLL = false>
__global__ void __launch_bounds__(Z / R, B) qc_decode_kernel(const __grid_constant__ QcParams p) {
    constexpr int T = Z / R;
    constexpr int W = Z / 32;  // 32-bit words per Z-bit block vector
    static_assert(Z % 32 == 0 && Z % R == 0 && T % 32 == 0, "Z must be a multiple of 32 and of 32*R");
    static_assert(F >= 1 && F <= QC_MAX_F, "frames per CTA");
    static_assert(!PAIR || (F == 2 && R == 1 && MODE != STORE_FP32 && ALGO == ALGO_AMIN && !CLIP && !RG),
                  "paired mode: two slots, one row per thread, 16-bit messages, Approximate-Min*, no clips");
    using RE = typename RTraits<MODE>::T;
    static_assert(!OT || (!PAIR && !RG && R == 1), "the offset table is built for one row per thread");
    static_assert(FIX < 0 || (!OT && !PAIR && FIX < QC_FIXED_COUNT), "compiled-in descriptors: no offset table");
    constexpr bool CIRC = ALGO == ALGO_CIRC;
    static_assert(!ROLL || (RG && FIX < 0 && !CIRC), "the rolled layer loop: global messages, parameter descriptors");
    static_assert(!CIRC || (D == 6 && !CLIP && !PAIR), "the circulant engine's decoder: degrees 3 and 6, no clips");
    using SV = SlotView<MODE, PAIR>;
    using LT = LTraits<MODE>;
    using LE = typename LT::T;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = p.n_vars;
    const int nblk = N / Z;
    const int lstride = (N + 7) & ~7;                      // elements per slot (16-byte multiple)
    LE* sL = reinterpret_cast<LE*>(smem_raw);
    uint32_t* sHB = reinterpret_cast<uint32_t*>(smem_raw + (size_t)F * lstride * sizeof(LE));  // [F][nblk*W]
    // OT: the column offset table after the hard-decision words, 16-byte aligned; ALGO_WAMIN: the
    // weight table after that
    uint32_t* sOT = reinterpret_cast<uint32_t*>(
        smem_raw + (((size_t)F * lstride * sizeof(LE) + (size_t)F * (N / 32) * 4 + 15) & ~(size_t)15));
    float2* sW = reinterpret_cast<float2*>(sOT + (OT ? T * (QC_DEG_LOW * 4 + D * 8) : 0));
    __shared__ uint32_t s_fid[QC_MAX_F];
    __shared__ uint32_t s_sfail[QC_MAX_F];
    __shared__ uint32_t s_be[QC_MAX_F];
    __shared__ uint32_t s_iz[QC_MAX_F];  // ALGO_CIRC: info positions with value <= 0

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const float r_cap = p.r_max > 0.0f ? p.r_max : __int_as_float(0x7f800000);
    const float lp_cap = p.l_post_max > 0.0f ? p.l_post_max : __int_as_float(0x7f800000);
    const CircRt cr{CircConsts{p.circ_c[0], p.circ_c[1], p.circ_c[2], p.circ_c[3]}, p.circ_damping, p.circ_sfpu != 0};

    MsgRegs<D, R, F, MODE, PAIR, RG> msg;
    if constexpr (OT) {  // each thread writes and later reads only its own entries: no barrier needed
        for (int l = 0; l < QC_LAYERS; ++l) {
            const int d = l < 4 ? QC_DEG_LOW : D;
            uint32_t* tab = sOT + T * ot_layer_start(l, D);
            for (int e = 0; e < d; ++e)
                tab[ot_pos(d, e, tid, T)] =
                    (uint32_t)((p.blk_off[l][e] + ((tid + p.shift[l][e]) & (Z - 1))) * (int)sizeof(LE));
        }
    }
    if constexpr (algo_weighted(ALGO)) {  // visible after the first refill's barrier
        for (int i = tid; i < p.w_iters * p.w_slots; i += T) sW[i] = p.wtab[i];
    }

    uint32_t act = 0;                // active slots (uniform)
    uint32_t need = (1u << F) - 1u;  // slots waiting for a frame (uniform)
    int it[F];
    uint32_t fid[F];
    int snr_bin[F];
#pragma unroll
    for (int f = 0; f < F; ++f) { it[f] = 0; fid[f] = 0xFFFFFFFFu; snr_bin[f] = 0; }
    const bool per_frame_snr = !EXT && p.ebn0_hi > p.ebn0_lo;

    // per-CTA tallies, kept by thread 0
    unsigned long long t_frames = 0, t_be = 0, t_fe = 0, t_it = 0, t_unc = 0, t_max = 0, t_be2 = 0;

    for (;;) {
        // ---------------------------------------------------------------- refill
        if (need) {
            if (tid == 0) {
#pragma unroll
                for (int f = 0; f < F; ++f)
                    if (need & (1u << f)) {
                        const uint32_t c = atomicAdd(p.work, 1u);
                        s_fid[f] = c < p.n_frames ? c : 0xFFFFFFFFu;
                    }
            }
            __syncthreads();
#pragma unroll
            for (int f = 0; f < F; ++f) {
                if (!(need & (1u << f))) continue;
                fid[f] = s_fid[f];
                it[f] = 0;
                if (fid[f] == 0xFFFFFFFFu) { act &= ~(1u << f); continue; }
                act |= 1u << f;
                if constexpr (RG) {  // the CTA clears the slot's messages; the barrier that ends the refill
                                     // makes the zeros visible to each row's owner
                    RE* rs = reinterpret_cast<RE*>(p.r_base) + ((size_t)blockIdx.x * F + f) * p.slot_elems;
                    for (int i = tid; i < p.slot_elems; i += T) rs[i] = RE(0);
                } else {
                    msg.zero_slot(f);
                }
                const SV L(sL, f, lstride);
                const int nq = p.n_tx >> 2;
                if (EXT) {
                    const float4* src = reinterpret_cast<const float4*>(p.llr_in + (size_t)fid[f] * p.n_tx);
                    for (int qd = tid; qd < nq; qd += T) {
                        const float4 v4 = src[qd];
                        float v[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            float x = v[k];
                            if (CLIP && p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                            L.st(4 * qd + k, x);
                        }
                    }
                } else {
                    const uint64_t gf = p.first_frame + fid[f];
                    float ch_mu = p.mu, ch_sigma = p.sigma;
                    if (per_frame_snr)
                        frame_snr(p.ebn0_lo, p.ebn0_hi, p.rate, gf, p.stream, p.seed_lo, p.seed_hi, ch_mu, ch_sigma,
                                  snr_bin[f]);
                    for (int qd = tid; qd < nq; qd += T) {
                        float n[4];
                        if (ch_sigma > 0.0f) {
                            const U32x4 x = philox4x32_10(U32x4{(uint32_t)qd, (uint32_t)gf, (uint32_t)(gf >> 32), p.stream},
                                                          p.seed_lo, p.seed_hi);
                            box_muller(x.x, x.y, n[0], n[1]);
                            box_muller(x.z, x.w, n[2], n[3]);
                        } else {
                            n[0] = n[1] = n[2] = n[3] = 0.0f;
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            float x = ch_sigma > 0.0f ? __fmaf_rn(ch_sigma, n[k], ch_mu) : ch_mu;
                            if (CLIP && p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                            L.st(4 * qd + k, x);
                        }
                    }
                }
                for (int i = p.n_tx + tid; i < N; i += T) L.st(i, 0.0f);
            }
            need = 0;
            __syncthreads();
        }
        if (!act) break;

        // ---------------------------------------------------------------- one layered iteration
        if (p.max_iter > 0) {
            const float2* wt[F];
#pragma unroll
            for (int f = 0; f < F; ++f)
                wt[f] = algo_weighted(ALGO) ? sW + min(it[f], p.w_iters - 1) * p.w_slots : nullptr;
            // OT: each layer's offsets are loaded one layer ahead, so their shared-memory latency
            // overlaps the previous row update; two register sets take the layers in turn (no copy
            // between them: +1.5 % on r1/2 K=1024 fp32 against copying the next set into the
            // current one).  ALGO_CIRC visits the degree-D layers first (the
            // circulant engine's tile schedule, rows 512..1535 before 0..511 for K = 1024:
            // engines/circulant_dma_4cw/ar4ja_circulant_descriptors_4cw.h:29-31).
            int offs[2][OT ? D : 1];
            if constexpr (OT) {
                if constexpr (CIRC) ot_load<D, T>(sOT + T * ot_layer_start(4, D), tid, offs[0]);
                else ot_load<QC_DEG_LOW, T>(sOT, tid, offs[0]);
            }
#pragma unroll
            for (int l = 0; l < (ROLL ? 4 : QC_LAYERS); ++l) {
                const int ly = CIRC ? (l + 4) % QC_LAYERS : l;        // the layer updated at step l
                const int ly_next = CIRC ? (l + 5) % QC_LAYERS : l + 1;
                const float2* wl[F];
#pragma unroll
                for (int f = 0; f < F; ++f)
                    wl[f] = ALGO == ALGO_WAMIN ? wt[f] + qc_edge_slot(ly, 0, D) : (ALGO == ALGO_WROW ? wt[f] + ly : nullptr);
                int (&cur)[OT ? D : 1] = offs[l & 1];  // this layer's offsets
                if constexpr (OT) {                     // start loading the next layer's
                    if (l + 1 < QC_LAYERS) {
                        const uint32_t* nt = sOT + T * ot_layer_start(ly_next, D);
                        if (ly_next < 4) ot_load<QC_DEG_LOW, T>(nt, tid, offs[(l + 1) & 1]);
                        else ot_load<D, T>(nt, tid, offs[(l + 1) & 1]);
                    }
                }
#pragma unroll
                for (int rho = 0; rho < R; ++rho) {
                    const int j = tid + rho * T;
                    if (ly < 4) {
                        int idx[QC_DEG_LOW];
                        if constexpr (OT) {
#pragma unroll
                            for (int e = 0; e < QC_DEG_LOW; ++e) idx[e] = cur[e];
                        } else
#pragma unroll
                            for (int e = 0; e < QC_DEG_LOW; ++e)
                                idx[e] = qc_blk<FIX>(p, ly, e) + ((j + qc_shift<FIX>(p, ly, e)) & (Z - 1));
                        if constexpr (RG) {
                            RowMsgGlobal<QC_DEG_LOW, MODE> rm[F];
#pragma unroll
                            for (int f = 0; f < F; ++f)
                                rm[f] = rg_row<QC_DEG_LOW, MODE, Z>(p, (size_t)blockIdx.x * F + f, ly, j);
                            if constexpr (CIRC) row_update_circ<QC_DEG_LOW, MODE, F>(idx, sL, lstride, rm, cr);
                            else row_update<QC_DEG_LOW, MODE, ALGO, CLIP, F>(idx, sL, lstride, rm, r_cap, lp_cap, wl);
                        } else if constexpr (PAIR)
                            row_update_pair<QC_DEG_LOW, MODE>(idx, sL, msg.r3[ly & 3]);
                        else if constexpr (CIRC)
                            row_update_circ<QC_DEG_LOW, MODE, F, RowMsg<QC_DEG_LOW, MODE>, OT>(
                                idx, sL, lstride, msg.r3[ly & 3][rho], cr);
                        else
                            row_update<QC_DEG_LOW, MODE, ALGO, CLIP, F, RowMsg<QC_DEG_LOW, MODE>, OT>(
                                idx, sL, lstride, msg.r3[ly & 3][rho], r_cap, lp_cap, wl);
                    } else {
                        int idx[D];
                        if constexpr (OT) {
#pragma unroll
                            for (int e = 0; e < D; ++e) idx[e] = cur[e];
                        } else
#pragma unroll
                            for (int e = 0; e < D; ++e)
                                idx[e] = qc_blk<FIX>(p, ly, e) + ((j + qc_shift<FIX>(p, ly, e)) & (Z - 1));
                        if constexpr (RG) {
                            RowMsgGlobal<D, MODE> rm[F];
#pragma unroll
                            for (int f = 0; f < F; ++f)
                                rm[f] = rg_row<D, MODE, Z>(p, (size_t)blockIdx.x * F + f, ly, j);
                            if constexpr (CIRC) row_update_circ<D, MODE, F>(idx, sL, lstride, rm, cr);
                            else row_update<D, MODE, ALGO, CLIP, F>(idx, sL, lstride, rm, r_cap, lp_cap, wl);
                        } else if constexpr (PAIR)
                            row_update_pair<D, MODE>(idx, sL, msg.rD[(ly - 4) & 7]);
                        else if constexpr (CIRC)
                            row_update_circ<D, MODE, F, RowMsg<D, MODE>, OT>(idx, sL, lstride,
                                                                            msg.rD[(ly - 4) & 7][rho], cr);
                        else
                            row_update<D, MODE, ALGO, CLIP, F, RowMsg<D, MODE>, OT>(
                                idx, sL, lstride, msg.rD[(ly - 4) & 7][rho], r_cap, lp_cap, wl);
                    }
                }
                __syncthreads();
            }
            if constexpr (ROLL) {
#pragma unroll 1
                for (int ly = 4; ly < QC_LAYERS; ++ly) {
                    const float2* wl[F];
#pragma unroll
                    for (int f = 0; f < F; ++f)
                        wl[f] = ALGO == ALGO_WAMIN ? wt[f] + qc_edge_slot(ly, 0, D)
                                                   : (ALGO == ALGO_WROW ? wt[f] + ly : nullptr);
#pragma unroll
                    for (int rho = 0; rho < R; ++rho) {
                        const int j = tid + rho * T;
                        int idx[D];
#pragma unroll
                        for (int e = 0; e < D; ++e) idx[e] = p.blk_off[ly][e] + ((j + p.shift[ly][e]) & (Z - 1));
                        RowMsgGlobal<D, MODE> rm[F];
#pragma unroll
                        for (int f = 0; f < F; ++f)
                            rm[f] = rg_row<D, MODE, Z>(p, (size_t)blockIdx.x * F + f, ly, j);
                        row_update<D, MODE, ALGO, CLIP, F>(idx, sL, lstride, rm, r_cap, lp_cap, wl);
                    }
                    __syncthreads();
                }
            }
#pragma unroll
            for (int f = 0; f < F; ++f) it[f] += (act >> f) & 1u;
        }

        // ---------------------------------------------------------------- syndrome / stop
        // The reference engine tests the syndrome from the third iteration on
        // (ldpc_decoder_core.h:524-526); the circulant engine and the weighted decoder (no
        // counterpart in the reference) from the first.
        constexpr int stop_from = (CIRC || algo_weighted(ALGO)) ? 1 : 3;
        uint32_t eval = 0;
#pragma unroll
        for (int f = 0; f < F; ++f)
            if ((act >> f) & 1u)
                if (it[f] >= stop_from || it[f] >= p.max_iter) eval |= 1u << f;
        if (!eval) continue;
        {
            // Pre-check: the sign parity of each thread's own rows in the two layers updated first in
            // the iteration (layers 0 and 2 of degree 3; layers 4 and 6 of degree D in the circulant
            // engine's order), or for the genie stop the sign bits of the info positions.  A frame
            // failing it has not stopped, so unless it has reached max_iter it needs no ballots,
            // syndrome words or counts this iteration.  Layers 0 and 2 show a failing row in about
            // 97 % of the checks of frames that have not yet converged (2.5 to 3 dB).  A frame that
            // passes goes through the full evaluation below, so the stop rule is unchanged.
            const bool genie = CIRC && p.stop_rule == QC_STOP_GENIE;
            constexpr int l0 = CIRC ? 4 : 0;
            constexpr int dl = CIRC ? D : QC_DEG_LOW;
            uint32_t cand = 0;
#pragma unroll
            for (int f = 0; f < F; ++f)
                if (((eval >> f) & 1u) && it[f] < p.max_iter) cand |= 1u << f;
#pragma unroll
            for (int f = 0; f < F; ++f) {
                if (!((cand >> f) & 1u)) continue;
                const SV L(sL, f, lstride);
                uint32_t bad = 0;
                if (genie) {
                    for (int i = tid; i < p.n_info; i += T) bad |= L.sign(i);
                } else {
#pragma unroll
                    for (int rho = 0; rho < R; ++rho) {
                        const int j = tid + rho * T;
#pragma unroll
                        for (int l = l0; l < l0 + 4; l += 2) {
                            uint32_t par = 0;
#pragma unroll
                            for (int e = 0; e < dl; ++e)
                                par ^= L.sign(qc_blk<FIX>(p, l, e) + ((j + qc_shift<FIX>(p, l, e)) & (Z - 1)));
                            bad |= par;
                        }
                    }
                }
                if (__syncthreads_or((int)bad)) eval &= ~(1u << f);
            }
            if (!eval) continue;
        }

        const int nwords = nblk * W;
#pragma unroll
        for (int f = 0; f < F; ++f) {
            if (!((eval >> f) & 1u)) continue;
            const SV L(sL, f, lstride);
            uint32_t* hb = sHB + f * nwords;
            for (int wd = warp; wd < nwords; wd += T / 32) {
                const uint32_t b = __ballot_sync(0xFFFFFFFFu, L.sign(wd * 32 + lane));
                if (lane == 0) hb[wd] = b;
            }
        }
        if (tid < F) { s_sfail[tid] = 0; s_be[tid] = 0; s_iz[tid] = 0; }
        __syncthreads();
        // syndrome words: (f, layer, word) -> XOR over the layer's edges of the rotated block vectors
        for (int t = tid; t < F * QC_LAYERS * W; t += T) {
            const int f = t / (QC_LAYERS * W);
            if (!((eval >> f) & 1u)) continue;
            const int l = (t / W) % QC_LAYERS, w = t % W;
            const uint32_t* hb = sHB + f * nwords;
            const int deg = l < 4 ? QC_DEG_LOW : D;
            uint32_t acc = 0;
            for (int e = 0; e < deg; ++e) {
                const int s = p.shift[l][e];
                const int base = p.blk_off[l][e] >> 5;
                const int ws = s >> 5;
                const uint32_t lo = hb[base + ((w + ws) & (W - 1))];
                const uint32_t hi = hb[base + ((w + ws + 1) & (W - 1))];
                acc ^= __funnelshift_r(lo, hi, s & 31);
            }
            if (acc) atomicAdd(&s_sfail[f], (uint32_t)__popc(acc));
        }
        // bit errors over the transmitted prefix (ALGO_CIRC: sign bits over the info positions)
        const int ntxw = CIRC ? p.n_info >> 5 : p.n_tx >> 5;
#pragma unroll
        for (int f = 0; f < F; ++f) {
            if (!((eval >> f) & 1u)) continue;
            const uint32_t* hb = sHB + f * nwords;
            uint32_t cnt = 0;
            for (int t = tid; t < ntxw; t += T) cnt += __popc(hb[t]);
            cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
            if (lane == 0 && cnt) atomicAdd(&s_be[f], cnt);
        }
        __syncthreads();
        uint32_t done = 0, stopped = 0;
#pragma unroll
        for (int f = 0; f < F; ++f) {
            if (!((eval >> f) & 1u)) continue;
            bool conv;
            if constexpr (CIRC)
                conv = it[f] >= 1 && (p.stop_rule == QC_STOP_GENIE ? s_be[f] == 0 : s_sfail[f] == 0);
            else
                conv = it[f] >= stop_from && s_sfail[f] == 0;
            if (conv) stopped |= 1u << f;
            if (conv || it[f] >= p.max_iter) done |= 1u << f;
        }
        if (!done) continue;
        if constexpr (CIRC) {
            // the circulant stepper's tally of a frame that never met the syndrome: info positions
            // with value <= 0 (tests/test_circulant_dma_stepper.cpp:807-816)
            const uint32_t zc = p.stop_rule == QC_STOP_GENIE ? 0u : (done & ~stopped);
            if (zc) {
#pragma unroll
                for (int f = 0; f < F; ++f) {
                    if (!((zc >> f) & 1u)) continue;
                    const SV L(sL, f, lstride);
                    uint32_t cnt = 0;
                    for (int i = tid; i < p.n_info; i += T) cnt += L.ld(i) <= 0.0f;
                    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
                    if (lane == 0 && cnt) atomicAdd(&s_iz[f], cnt);
                }
                __syncthreads();
            }
        }
#pragma unroll
        for (int f = 0; f < F; ++f) {
            if (!((done >> f) & 1u)) continue;
            uint32_t be = s_be[f];
            const uint32_t sf = s_sfail[f];
            bool fe = be > 0;
            if constexpr (CIRC) {  // a frame that stopped counts no errors; the stepper's frame error
                const bool st = (stopped >> f) & 1u;  // is "never met the syndrome"
                if (p.stop_rule == QC_STOP_GENIE) {
                    be = st ? 0u : be;
                    fe = be > 0;
                } else {
                    be = st ? 0u : s_iz[f];
                    fe = !st;
                }
            }
            if (tid == 0) {
                t_frames += 1;
                t_be += be;
                t_be2 += (unsigned long long)be * be;
                t_fe += fe;
                t_it += (unsigned)it[f];
                t_unc += sf != 0;
                t_max = max(t_max, (unsigned long long)it[f]);
                if (p.hist) atomicAdd(&p.hist[min(it[f], p.hist_bins - 1)], 1ull);
                if (per_frame_snr && p.snr_bins) {
                    atomicAdd(&p.snr_bins[snr_bin[f]], 1ull);
                    atomicAdd(&p.snr_bins[SNR_BINS + snr_bin[f]], (unsigned long long)fe);
                    atomicAdd(&p.snr_bins[2 * SNR_BINS + snr_bin[f]], (unsigned long long)be);
                    atomicAdd(&p.snr_bins[3 * SNR_BINS + snr_bin[f]], (unsigned long long)it[f]);
                }
                if (p.iters_out) p.iters_out[fid[f]] = it[f];
                if (p.synd_out) p.synd_out[fid[f]] = (int32_t)sf;
                if (p.be_out) p.be_out[fid[f]] = (int32_t)be;
            }
            if (p.post_out) {
                const SV L(sL, f, lstride);
                float* dst = p.post_out + (size_t)fid[f] * N;
                for (int i = tid; i < N; i += T) dst[i] = L.ld(i);
            }
        }
        need = done;
        act &= ~done;
        __syncthreads();  // s_be / s_sfail / sL of finished slots are reused below
    }
    if (tid == 0 && t_frames) {
        atomicAdd(&p.tally[T_FRAMES], t_frames);
        atomicAdd(&p.tally[T_BIT_ERR], t_be);
        atomicAdd(&p.tally[T_FRAME_ERR], t_fe);
        atomicAdd(&p.tally[T_ITER_SUM], t_it);
        atomicAdd(&p.tally[T_UNCONVERGED], t_unc);
        atomicMax(&p.tally[T_MAX_ITER], t_max);
        atomicAdd(&p.tally[T_BIT_ERR_SQ], t_be2);
    }
}

}  // namespace ldpcb200
