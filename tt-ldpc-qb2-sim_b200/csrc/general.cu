// General-matrix kernel (any parity-check matrix, the reference's file row order) and its host side.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "ldpc_general.cuh"
#include "ldpc_qc.cuh"  // TallyWord, LTraits

namespace ldpcb200 {

// Row-major tables of the general kernel, so that one lane reads a row's columns and messages with
// a few vector loads: columns [M][gen_dtc(DT)] int32 (-1 after the row's last edge), each row padded
// to a multiple of 4 (16 bytes); messages [M][gen_dtr<MODE>(DT)] elements per frame slot, rows
// unpadded (16-bit rows rounded to an even count), read and written with the widest vectors that
// tile a row (16, 8 or 4 bytes: 4 for 12-byte bf16 rows of degree 6, 8 for 24-byte fp32 ones).
// Padding the messages to 16 bytes as well was slower (bf16 9.93 vs 10.18, fp32 6.91 vs 8.25 M
// frames/s on the shipped r1/2 K=1024 file): the scratch of all resident slots outgrew L2.
__host__ __device__ constexpr int gen_dtc(int dt) { return (dt + 3) & ~3; }
template <int MODE>
__host__ __device__ constexpr int gen_dtr(int dt) {
    return MODE == STORE_FP32 ? dt : (dt + 1) & ~1;
}

// Message bytes of one frame slot.
static size_t gen_slot_bytes(int M, int dt, int storage) {
    return storage == STORE_FP32 ? (size_t)M * gen_dtr<STORE_FP32>(dt) * 4 : (size_t)M * gen_dtr<STORE_BF16>(dt) * 2;
}

template <int DT>
__device__ __forceinline__ void gen_load_cols(const int32_t* cols, int m, int (&col)[gen_dtc(DT)]) {
    const int4* cp = reinterpret_cast<const int4*>(cols + (size_t)m * gen_dtc(DT));
#pragma unroll
    for (int k = 0; k < gen_dtc(DT) / 4; ++k) {
        const int4 v = __ldg(cp + k);
        col[4 * k] = v.x;
        col[4 * k + 1] = v.y;
        col[4 * k + 2] = v.z;
        col[4 * k + 3] = v.w;
    }
}

// One row of degree deg <= DT, updated by one lane (ldpc_decoder_core.h:414-520).
template <int DT, int MODE, int ALGO>
__device__ __forceinline__ void gen_row(const GenParams& p, int m, typename LTraits<MODE>::T* L,
                                        typename RTraits<MODE>::T* r, float r_cap, float lp_cap) {
    using LT = LTraits<MODE>;
    using RT = RTraits<MODE>;
    using RE = typename RT::T;
    constexpr int DTR = gen_dtr<MODE>(DT);
    constexpr int RB = DTR * (int)sizeof(RE);
    constexpr int VW = RB % 16 == 0 ? 16 : RB % 8 == 0 ? 8 : 4;
    constexpr int NV = RB / VW;
    using VT = typename std::conditional<VW == 16, uint4,
                                         typename std::conditional<VW == 8, uint2, uint32_t>::type>::type;
    int deg = 0;
    int col[gen_dtc(DT)];
    float q[DT];
    gen_load_cols<DT>(p.cols, m, col);
#pragma unroll
    for (int e = 0; e < DT; ++e)
        if (col[e] >= 0) deg = e + 1;
    if (deg == 0) return;
    union {
        VT v[NV];
        RE e[DTR];
    } rm;
    VT* rp = reinterpret_cast<VT*>(r + (size_t)m * DTR);
#pragma unroll
    for (int k = 0; k < NV; ++k) rm.v[k] = rp[k];
    uint32_t par = 0;
#pragma unroll
    for (int e = 0; e < DT; ++e)
        if (e < deg) {
            q[e] = __fsub_rn(LT::ld(L, col[e]), RT::ld(&rm.e[e]));
            par ^= __float_as_uint(q[e]);
        }
    par &= 0x80000000u;
    int am = 0;
    float mag_min, mag_all;
    if (ALGO == ALGO_AMIN) {
        // As the QC kernel's row update: prefix minima pm_i = min(9999, |q_0|, .., |q_i|), the
        // argmin am = the first i with |q_i| = pm_{DT-1} (lt[i] = i < am), and the recursive min* over
        // the other edges in row order, o_i = |q_i| for i < am and |q_{i+1}| after it
        // (ldpc_decoder_core.h:414-475).  Edges past the row's degree are the largest float: never
        // the minimum, and a min* step with it leaves its value unchanged (diff >= 2, so nothing is
        // subtracted, and every intermediate stays finite), so the row runs DT - 1 steps whatever its
        // degree.
        float a[DT], pm[DT];
#pragma unroll
        for (int e = 0; e < DT; ++e) a[e] = e < deg ? fabsf(q[e]) : 3.40282347e38f;
        pm[0] = fminf(a[0], 9999.0f);
#pragma unroll
        for (int e = 1; e < DT; ++e) pm[e] = fminf(pm[e - 1], a[e]);
        const float mn = pm[DT - 1];
        bool lt[DT];
#pragma unroll
        for (int i = 0; i < DT; ++i) lt[i] = (i + 1 < DT) ? (pm[i] > mn) : false;
#pragma unroll
        for (int i = 0; i < DT; ++i) am += lt[i] ? 1 : 0;
        float mo = DT > 1 ? (lt[0] ? a[0] : a[1]) : mn;
#pragma unroll
        for (int i = 1; i + 1 < DT; ++i) mo = amin_step_fma(mo, lt[i] ? a[i] : a[i + 1]);
        if (deg == 1) mo = mn;  // m_others = min_mag when the row has one edge (:181)
        mag_min = mo;
        mag_all = amin_step_fma(mo, mn);
    } else {
        float m1 = 999.0f, m2 = 999.0f;
#pragma unroll
        for (int e = 0; e < DT; ++e)
            if (e < deg) {
                const float a = fabsf(q[e]);
                if (a < m1) { m2 = m1; m1 = a; am = e; }
                else if (a < m2) { m2 = a; }
            }
        mag_min = __fmul_rn(0.75f, m2);
        mag_all = __fmul_rn(0.75f, m1);
    }
    mag_min = fminf(mag_min, r_cap);
    mag_all = fminf(mag_all, r_cap);
    const uint32_t smin = __float_as_uint(mag_min) | par;
    const uint32_t sall = __float_as_uint(mag_all) | par;
#pragma unroll
    for (int e = 0; e < DT; ++e)
        if (e < deg) {
            const float rn = __uint_as_float(((e == am) ? smin : sall) ^ (__float_as_uint(q[e]) & 0x80000000u));
            float ln = __fadd_rn(q[e], rn);
            ln = fminf(fmaxf(ln, -lp_cap), lp_cap);
            LT::st(L, col[e], ln);
            RT::st(&rm.e[e], rn);
        }
#pragma unroll
    for (int k = 0; k < NV; ++k) rp[k] = rm.v[k];
}

// NW: frame slots (warps) per CTA; large codes use one so that a slot's L fits shared memory.
template <int DT, int MODE, int ALGO, bool EXT, int NW = GEN_WARPS>
__global__ void __launch_bounds__(32 * NW) general_kernel(const __grid_constant__ GenParams p) {
    using LT = LTraits<MODE>;
    using LE = typename LT::T;
    using RE = typename RTraits<MODE>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int N = p.N, M = p.M;
    const int lstride = (N + 7) & ~7;
    LE* L = reinterpret_cast<LE*>(smem_raw) + (size_t)warp * lstride;
    const size_t slot = (size_t)blockIdx.x * NW + warp;
    RE* r = reinterpret_cast<RE*>(p.r_base) + slot * (size_t)M * gen_dtr<MODE>(DT);
    const float r_cap = p.r_max > 0.0f ? p.r_max : __int_as_float(0x7f800000);
    const float lp_cap = p.l_post_max > 0.0f ? p.l_post_max : __int_as_float(0x7f800000);
    unsigned long long t_frames = 0, t_be = 0, t_fe = 0, t_it = 0, t_unc = 0, t_max = 0, t_be2 = 0;

    for (;;) {
        uint32_t fid = 0;
        if (lane == 0) fid = atomicAdd(p.work, 1u);
        fid = __shfl_sync(0xFFFFFFFFu, fid, 0);
        if (fid >= p.n_frames) break;
        const bool per_frame_snr = !EXT && p.ebn0_hi > p.ebn0_lo;
        int snr_bin = 0;
        // channel
        if (EXT) {
            const float* src = p.llr_in + (size_t)fid * p.n_tx;
            for (int i = lane; i < p.n_tx; i += 32) {
                float x = src[i];
                if (p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                LT::st(L, i, x);
            }
        } else {
            const uint64_t gf = p.first_frame + fid;
            float ch_mu = p.mu, ch_sigma = p.sigma;
            if (per_frame_snr)
                frame_snr(p.ebn0_lo, p.ebn0_hi, p.rate, gf, p.stream, p.seed_lo, p.seed_hi, ch_mu, ch_sigma, snr_bin);
            for (int qd = lane; qd * 4 < p.n_tx; qd += 32) {
                float n[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (ch_sigma > 0.0f) {
                    const U32x4 x = philox4x32_10(U32x4{(uint32_t)qd, (uint32_t)gf, (uint32_t)(gf >> 32), p.stream},
                                                  p.seed_lo, p.seed_hi);
                    box_muller(x.x, x.y, n[0], n[1]);
                    box_muller(x.z, x.w, n[2], n[3]);
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (4 * qd + k >= p.n_tx) break;
                    float x = ch_sigma > 0.0f ? __fmaf_rn(ch_sigma, n[k], ch_mu) : ch_mu;
                    if (p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                    LT::st(L, 4 * qd + k, x);
                }
            }
        }
        for (int i = p.n_tx + lane; i < N; i += 32) LT::st(L, i, 0.0f);
        {
            uint32_t* rz = reinterpret_cast<uint32_t*>(r);
            const size_t nw = (size_t)M * gen_dtr<MODE>(DT) * sizeof(RE) / 4;
            for (size_t i = lane; i < nw; i += 32) rz[i] = 0u;
        }
        __syncwarp();

        int it = 0;
        uint32_t sfail = 0;
        for (;;) {
            if (it >= p.max_iter) break;
            for (int k = 0; k < p.n_runs; ++k) {
                const int a = p.runs[k], b = p.runs[k + 1];
                for (int m = a + lane; m < b; m += 32) gen_row<DT, MODE, ALGO>(p, m, L, r, r_cap, lp_cap);
                __syncwarp();
            }
            ++it;
            if (it >= 3) {  // syndrome from iteration index 2 on (ldpc_decoder_core.h:526)
                // 32 rows at a time; the warp stops at the first group holding a failing row, so an
                // unconverged frame usually costs a few groups instead of all M rows
                bool bad = false;
                for (int m0 = 0; m0 < M && !bad; m0 += 32) {
                    const int m = m0 + lane;
                    uint32_t par = 0;
                    if (m < M) {
                        int col[gen_dtc(DT)];
                        gen_load_cols<DT>(p.cols, m, col);
#pragma unroll
                        for (int e = 0; e < DT; ++e)
                            if (col[e] >= 0) par ^= __float_as_uint(LT::ld(L, col[e])) >> 31;
                    }
                    bad = __any_sync(0xFFFFFFFFu, par) != 0;
                }
                if (!bad) break;
            }
        }
        // tally
        uint32_t be = 0;
        for (int i = lane; i < p.n_tx; i += 32) be += __float_as_uint(LT::ld(L, i)) >> 31;
        be = __reduce_add_sync(0xFFFFFFFFu, be);
        for (int m = lane; m < M; m += 32) {
            uint32_t par = 0;
            int col[gen_dtc(DT)];
            gen_load_cols<DT>(p.cols, m, col);
#pragma unroll
            for (int e = 0; e < DT; ++e)
                if (col[e] >= 0) par ^= __float_as_uint(LT::ld(L, col[e])) >> 31;
            sfail += par;
        }
        sfail = __reduce_add_sync(0xFFFFFFFFu, sfail);
        if (lane == 0) {
            t_frames += 1;
            t_be += be;
            t_be2 += (unsigned long long)be * be;
            t_fe += be > 0;
            t_it += (unsigned)it;
            t_unc += sfail != 0;
            t_max = max(t_max, (unsigned long long)it);
            if (p.hist) atomicAdd(&p.hist[min(it, p.hist_bins - 1)], 1ull);
            if (per_frame_snr && p.snr_bins) {
                atomicAdd(&p.snr_bins[snr_bin], 1ull);
                atomicAdd(&p.snr_bins[SNR_BINS + snr_bin], (unsigned long long)(be > 0));
                atomicAdd(&p.snr_bins[2 * SNR_BINS + snr_bin], (unsigned long long)be);
                atomicAdd(&p.snr_bins[3 * SNR_BINS + snr_bin], (unsigned long long)it);
            }
            if (p.iters_out) p.iters_out[fid] = it;
            if (p.synd_out) p.synd_out[fid] = (int32_t)sfail;
            if (p.be_out) p.be_out[fid] = (int32_t)be;
        }
        if (p.post_out) {
            float* dst = p.post_out + (size_t)fid * N;
            for (int i = lane; i < N; i += 32) dst[i] = LT::ld(L, i);
        }
        __syncwarp();
    }
    if (lane == 0 && t_frames) {
        atomicAdd(&p.tally[T_FRAMES], t_frames);
        atomicAdd(&p.tally[T_BIT_ERR], t_be);
        atomicAdd(&p.tally[T_FRAME_ERR], t_fe);
        atomicAdd(&p.tally[T_ITER_SUM], t_it);
        atomicAdd(&p.tally[T_UNCONVERGED], t_unc);
        atomicMax(&p.tally[T_MAX_ITER], t_max);
        atomicAdd(&p.tally[T_BIT_ERR_SQ], t_be2);
    }
}

// ----------------------------------------------------------------------------- host side

static int gfail(std::string& err, int code, const std::string& msg) {
    err = msg;
    return code;
}

// The row schedule of the general kernel.  Two rows that share no variable commute: updating them
// in either order, or at once, gives the same bits, because a row reads and writes only its own
// variables' posteriors and its own messages.  So any order that keeps every pair of rows sharing a
// variable in file order decodes exactly as the file order does.  Each row gets its earliest level,
// 1 + the highest level among the earlier rows it shares a variable with; the rows sorted by level
// (file order inside a level) are such an order, and the greedy cut of that order into steps of
// consecutive rows sharing no variable, at most 32 rows each (one warp pass), gives the steps the
// kernel runs with a warp barrier between them.  For the reference's shipped r1/2 K=1024 file (135
// runs of consecutive conflict-free rows in file order, 11.4 rows on average) this gives 51 steps of
// about 30 rows; for makeH order, Z/32 steps per layer as before.  `order` receives the file rows in
// schedule order, `starts` the first position of every step followed by M.
void general_schedule(const int32_t* rows, int N, int M, int dmax, std::vector<int32_t>& order,
                      std::vector<int32_t>& starts) {
    std::vector<int32_t> lev(M), last(N, 0);
    int maxl = 0;
    for (int m = 0; m < M; ++m) {
        int l = 0;
        for (int e = 0; e < dmax; ++e) {
            const int32_t c = rows[(size_t)m * dmax + e];
            if (c >= 0) l = std::max(l, last[c]);
        }
        lev[m] = ++l;
        maxl = std::max(maxl, l);
        for (int e = 0; e < dmax; ++e) {
            const int32_t c = rows[(size_t)m * dmax + e];
            if (c >= 0) last[c] = l;
        }
    }
    std::vector<int32_t> pos(maxl + 2, 0);
    for (int m = 0; m < M; ++m) ++pos[lev[m] + 1];
    for (int l = 1; l <= maxl + 1; ++l) pos[l] += pos[l - 1];
    order.assign(M, 0);
    for (int m = 0; m < M; ++m) order[pos[lev[m]]++] = m;
    starts.assign(1, 0);
    std::vector<char> used(N, 0);
    int start = 0;
    for (int k = 0; k < M; ++k) {
        const int32_t* rv = rows + (size_t)order[k] * dmax;
        bool cut = k - start == 32;
        for (int e = 0; e < dmax && !cut; ++e) cut = rv[e] >= 0 && used[rv[e]];
        if (cut) {
            starts.push_back(k);
            for (int j = start; j < k; ++j)
                for (int e = 0; e < dmax; ++e) {
                    const int32_t c = rows[(size_t)order[j] * dmax + e];
                    if (c >= 0) used[c] = 0;
                }
            start = k;
        }
        for (int e = 0; e < dmax; ++e)
            if (rv[e] >= 0) used[rv[e]] = 1;
    }
    starts.push_back(M);
}

int build_general(const int32_t* rows, int N, int M, int P, int dmax, GeneralCode* g, std::string& err) {
    g->N = N;
    g->M = M;
    g->P = P;
    g->dmax = dmax;
    int maxdeg = 0;
    for (int m = 0; m < M; ++m)
        for (int e = 0; e < dmax && rows[(size_t)m * dmax + e] >= 0; ++e) maxdeg = std::max(maxdeg, e + 1);
    g->dt = maxdeg <= 6 ? 6 : maxdeg <= 8 ? 8 : maxdeg <= 20 ? 20 : maxdeg <= 32 ? 32 : 0;
    if (!g->dt) return gfail(err, LDPC_ENOTSUP, "row degree above 32 is not supported");
    std::vector<int32_t> order, runs;
    general_schedule(rows, N, M, dmax, order, runs);
    g->n_runs = (int)runs.size() - 1;
    const int dtc = gen_dtc(g->dt);
    std::vector<int32_t> cols((size_t)dtc * M, -1);  // [M][dtc], rows in schedule order
    for (int k = 0; k < M; ++k)
        for (int e = 0; e < dmax; ++e) {
            const int32_t c = rows[(size_t)order[k] * dmax + e];
            if (c < 0) break;
            cols[(size_t)k * dtc + e] = c;
        }
    if (cudaMalloc(&g->d_cols, cols.size() * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&g->d_runs, runs.size() * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        return gfail(err, LDPC_ENOMEM, "device allocation failed");
    }
    if (cudaMemcpy(g->d_cols, cols.data(), cols.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g->d_runs, runs.data(), runs.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return gfail(err, LDPC_EIO, "copy of the matrix to the device failed");
    return build_general_steps(rows, dmax, g, err);
}

void free_general(GeneralCode* g) {
    cudaFree(g->d_cols);
    cudaFree(g->d_runs);
    cudaFree(g->d_r);
    cudaFree(g->d_scols[0]);
    cudaFree(g->d_scols[1]);
    cudaFree(g->d_slot[0]);
    cudaFree(g->d_slot[1]);
    cudaFree(g->d_slow);
    g->d_slow = nullptr;
    g->d_cols = g->d_runs = nullptr;
    g->d_scols[0] = g->d_scols[1] = nullptr;
    g->d_slot[0] = g->d_slot[1] = nullptr;
    g->d_r = nullptr;
    g->r_cap = 0;
    g->sdt = 0;
}

template <int DT, int MODE, int ALGO, bool EXT, int NW = GEN_WARPS>
static const void* gk() {
    return reinterpret_cast<const void*>(&general_kernel<DT, MODE, ALGO, EXT, NW>);
}

template <int DT, int MODE, int NW = GEN_WARPS>
static const void* pick_algo(int algo, bool ext) {
    if (algo == ALGO_AMIN) return ext ? gk<DT, MODE, ALGO_AMIN, true, NW>() : gk<DT, MODE, ALGO_AMIN, false, NW>();
    return ext ? gk<DT, MODE, ALGO_NMS, true, NW>() : gk<DT, MODE, ALGO_NMS, false, NW>();
}

template <int DT, int NW = GEN_WARPS>
static const void* pick_mode(int mode, int algo, bool ext) {
    if (mode == STORE_BF16) return pick_algo<DT, STORE_BF16, NW>(algo, ext);
    if (mode == STORE_FP32) return pick_algo<DT, STORE_FP32, NW>(algo, ext);
    return pick_algo<DT, STORE_FP16, NW>(algo, ext);
}

int launch_general(GeneralCode* g, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                   const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be,
                   unsigned long long* d_tally, unsigned long long* d_hist, int hist_bins, unsigned int* d_work,
                   int n_sm, cudaStream_t stream, std::string& err, unsigned long long* d_snr_bins) {
    const size_t esz = p->storage == STORE_BF16 ? 2 : 4;
    // four frame slots per CTA while their L arrays fit comfortably in shared memory, else one
    const int nw = (size_t)GEN_WARPS * ((g->N + 7) & ~7) * esz <= 160 * 1024 ? GEN_WARPS : 1;
    const void* fn = nw == GEN_WARPS ? (g->dt == 6    ? pick_mode<6>(p->storage, p->algo, ext)
                                        : g->dt == 8  ? pick_mode<8>(p->storage, p->algo, ext)
                                        : g->dt == 20 ? pick_mode<20>(p->storage, p->algo, ext)
                                                      : pick_mode<32>(p->storage, p->algo, ext))
                                     : (g->dt == 6    ? pick_mode<6, 1>(p->storage, p->algo, ext)
                                        : g->dt == 8  ? pick_mode<8, 1>(p->storage, p->algo, ext)
                                        : g->dt == 20 ? pick_mode<20, 1>(p->storage, p->algo, ext)
                                                      : pick_mode<32, 1>(p->storage, p->algo, ext));
    const size_t smem = (size_t)nw * ((g->N + 7) & ~7) * esz;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return gfail(err, LDPC_ENOTSUP, "general kernel: frame too large for shared memory");
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * nw, smem) != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        return gfail(err, LDPC_ENOTSUP, "general kernel does not fit on an SM");
    }
    const uint64_t want = (n + nw - 1) / nw;
    const uint64_t grid = std::min<uint64_t>(want, (uint64_t)per_sm * n_sm);
    if (!grid) return 0;
    const size_t need = grid * nw * gen_slot_bytes(g->M, g->dt, p->storage);
    if (g->r_cap < need) {
        cudaFree(g->d_r);
        g->d_r = nullptr;
        g->r_cap = 0;
        if (cudaMalloc(&g->d_r, need) != cudaSuccess) {
            cudaGetLastError();
            return gfail(err, LDPC_ENOMEM, "message scratch allocation failed");
        }
        g->r_cap = need;
    }
    GenParams gp;
    memset(&gp, 0, sizeof gp);
    gp.cols = g->d_cols;
    gp.runs = g->d_runs;
    gp.n_runs = g->n_runs;
    gp.N = g->N;
    gp.M = g->M;
    gp.n_tx = g->N - g->P;
    gp.dmax = g->dmax;
    gp.max_iter = p->max_iter;
    gp.mu = p->mu;
    gp.sigma = p->sigma;
    gp.l_max = p->l_max;
    gp.r_max = p->r_max;
    gp.l_post_max = p->l_post_max;
    gp.seed_lo = (uint32_t)p->seed;
    gp.seed_hi = (uint32_t)(p->seed >> 32);
    gp.stream = p->stream;
    gp.first_frame = first;
    gp.n_frames = n;
    gp.r_base = g->d_r;
    gp.llr_in = d_llr;
    gp.post_out = d_post;
    gp.iters_out = d_it;
    gp.synd_out = d_sf;
    gp.be_out = d_be;
    gp.tally = d_tally;
    gp.hist = d_hist;
    gp.hist_bins = hist_bins;
    gp.work = d_work;
    gp.ebn0_lo = p->ebn0_lo_db;
    gp.ebn0_hi = p->ebn0_hi_db;
    gp.rate = (float)((double)(g->N - g->M) / (double)(g->N - g->P));
    gp.snr_bins = d_snr_bins;
    void* args[] = {&gp};
    cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(32 * nw), args, smem, stream);
    if (e != cudaSuccess) return gfail(err, LDPC_EIO, std::string("general kernel launch: ") + cudaGetErrorString(e));
    return 0;
}

}  // namespace ldpcb200

// ----------------------------------------------------------------------------- no-allocation decode
//
// ldpc_decode_llr_static: the general kernel with every byte of its scratch in one file-scope
// device array, for callers that must not have a library allocate device memory on their GPU (a host
// application that reserves the whole GPU up front through its own pool, or one that must keep its
// device footprint fixed and known before it starts).  The caller passes device pointers for the
// channel LLRs and the outputs; this code calls no cudaMalloc/cudaFree and allocates no host memory.
//
// Scratch layout (LDPC_STATIC_SCRATCH_BYTES, 256-byte aligned regions):
//   [0, 256)           frame-claim counter (u32) and tallies (TALLY_WORDS x u64)
//   rows               the caller's [M][dmax] row table, copied in
//   cols               the same table in schedule order, [M][dtc] (the general kernel's layout)
//   runs               step starts (M + 1 entries) and their count
//   bitmap             N bits, used while the steps are cut
//   lev, last, order, cnt   work space of the schedule: M, N, M and M + 2 ints
//   messages           [slots][dmax][M] check messages, one region per frame slot
// Every call rewrites the tables and zeroes the counter and tallies; the messages are zeroed by the
// kernel when it starts a frame.  All calls share the one array, so calls whose work overlaps on the
// GPU (different streams, or different host threads) race on it: serialise them.

static __device__ __align__(256) unsigned char g_static_scratch[LDPC_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
unsigned char* g_static_addr[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// The schedule of general_schedule on the device (the same levels, order and steps), one warp, no
// waits on other threads: the caller's [M][dmax] row table in, the [M][dtc] table in schedule order
// and the step starts out.  lev [M], last [N], order [M] and cnt [M + 2] are work space.
__global__ void static_setup_kernel(const int32_t* rows, int M, int dmax, int N, int dtc, int32_t* cols,
                                    int32_t* runs, int32_t* n_runs, uint32_t* bitmap, int32_t* lev,
                                    int32_t* last, int32_t* order, int32_t* cnt) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x;
    for (int c = lane; c < N; c += 32) last[c] = 0;
    for (int w = lane; w < (N + 31) / 32; w += 32) bitmap[w] = 0u;
    __syncwarp();
    // earliest levels, rows in file order (a row's columns on its lanes)
    int maxl = 0;
    for (int m = 0; m < M; ++m) {
        const int c = lane < dmax ? rows[(size_t)m * dmax + lane] : -1;
        const int l = __reduce_max_sync(full, c >= 0 ? last[c] : 0) + 1;
        __syncwarp();
        if (c >= 0) last[c] = l;
        if (lane == 0) lev[m] = l;
        maxl = max(maxl, l);
        __syncwarp();
    }
    // stable counting sort by level: cnt[l] = first position of level l
    for (int l = lane; l < maxl + 2; l += 32) cnt[l] = 0;
    __syncwarp();
    for (int m = lane; m < M; m += 32) atomicAdd(&cnt[lev[m]], 1);
    __syncwarp();
    if (lane == 0) {
        int s = 0;
        for (int l = 1; l <= maxl; ++l) {
            const int t = cnt[l];
            cnt[l] = s;
            s += t;
        }
    }
    __syncwarp();
    for (int m0 = 0; m0 < M; m0 += 32) {
        const int m = m0 + lane;
        const int l = m < M ? lev[m] : -1;
        const unsigned peers = __match_any_sync(full, l);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        const int base = m < M ? cnt[l] : 0;
        __syncwarp();
        if (m < M) {
            order[base + rank] = m;
            if (lane == 31 - __clz(peers)) cnt[l] = base + __popc(peers);
        }
        __syncwarp();
    }
    // the table in schedule order, [M][dtc]
    for (int i = lane; i < M * dtc; i += 32) {
        const int k = i / dtc, e = i % dtc;
        cols[i] = e < dmax ? rows[(size_t)order[k] * dmax + e] : -1;
    }
    __syncwarp();
    // greedy steps of at most 32 rows sharing no variable
    int nr = 0, start = 0;
    if (lane == 0) runs[0] = 0;
    for (int k = 0; k < M; ++k) {
        const int c = lane < dmax ? rows[(size_t)order[k] * dmax + lane] : -1;
        const bool clash = c >= 0 && ((bitmap[c >> 5] >> (c & 31)) & 1u);
        if (__any_sync(full, clash) || k - start == 32) {
            ++nr;
            if (lane == 0) runs[nr] = k;
            for (int j = start; j < k; ++j) {
                const int c2 = lane < dmax ? rows[(size_t)order[j] * dmax + lane] : -1;
                if (c2 >= 0) atomicAnd(&bitmap[c2 >> 5], ~(1u << (c2 & 31)));
            }
            start = k;
            __syncwarp();
        }
        if (c >= 0) atomicOr(&bitmap[c >> 5], 1u << (c & 31));
        __syncwarp();
    }
    ++nr;
    if (lane == 0) {
        runs[nr] = M;
        *n_runs = nr;
    }
}

int sfail(int code, std::string& err, const char* msg) {
    err = msg;
    return code;
}

}  // namespace

namespace ldpcb200 {

int decode_llr_static(const ldpc_matrix* h, const ldpc_run_params* p, const float* d_llr, int64_t n,
                      float* d_post, int32_t* d_iters, int32_t* d_synd, int32_t* d_be, ldpc_tally* out,
                      cudaStream_t stream, std::string& err) {
    char msg[256];
    if (!h || !h->rows || !p) return sfail(LDPC_EINVAL, err, "matrix or params are NULL");
    if (n < 0) return sfail(LDPC_EINVAL, err, "n_frames out of range");
    if (n > 0 && !d_llr) return sfail(LDPC_EINVAL, err, "d_llr is NULL");
    const int N = h->n_vars, M = h->n_checks, P = h->n_punct, dmax = h->max_check_deg;
    if (N <= 0 || M <= 0 || dmax <= 0 || dmax > 32 || P < 0 || P >= N)
        return sfail(LDPC_EINVAL, err, "bad matrix dimensions (need N > P >= 0, M > 0, 1 <= max_check_deg <= 32)");
    if (p->max_iter < 0 || p->storage < 0 || p->storage > 2 || p->algo < 0 || p->algo > 1)
        return sfail(LDPC_EINVAL, err, "bad run parameters");
    int maxdeg = 0;
    for (int64_t i = 0; i < (int64_t)M * dmax; ++i) {
        const int32_t c = h->rows[i];
        if (c < -1 || c >= N) return sfail(LDPC_EINVAL, err, "edge index out of bounds");
        if (c >= 0 && i % dmax > 0 && h->rows[i - 1] < 0)
            return sfail(LDPC_EINVAL, err, "edge after the -1 that ends its row");
        if (c >= 0) maxdeg = std::max(maxdeg, (int)(i % dmax) + 1);
    }
    const int dt = maxdeg <= 6 ? 6 : maxdeg <= 8 ? 8 : maxdeg <= 20 ? 20 : 32;
    const int dtc = gen_dtc(dt);
    const size_t esz = p->storage == STORE_BF16 ? 2 : 4;
    // frame slots per CTA as ldpc_decode_llr's warp kernel takes them: four while their posteriors fit
    // comfortably in shared memory, else one
    const int nw = (size_t)GEN_WARPS * ((N + 7) & ~7) * esz <= 160 * 1024 ? GEN_WARPS : 1;
    const size_t off_rows = 256;
    const size_t off_cols = off_rows + align256((size_t)M * dmax * 4);
    const size_t off_runs = off_cols + align256((size_t)M * dtc * 4);
    const size_t off_bits = off_runs + align256((size_t)(M + 2) * 4);
    const size_t off_lev = off_bits + align256((size_t)(N + 31) / 32 * 4);
    const size_t off_last = off_lev + align256((size_t)M * 4);
    const size_t off_order = off_last + align256((size_t)N * 4);
    const size_t off_cnt = off_order + align256((size_t)M * 4);
    const size_t off_msgs = off_cnt + align256((size_t)(M + 2) * 4);
    const size_t per_slot = gen_slot_bytes(M, dt, p->storage);
    if (off_msgs + nw * per_slot > LDPC_STATIC_SCRATCH_BYTES) {
        snprintf(msg, sizeof msg,
                 "matrix needs %zu bytes of static scratch for one CTA of %d frame slots; the maximum is %zu",
                 off_msgs + nw * per_slot, nw, (size_t)LDPC_STATIC_SCRATCH_BYTES);
        return sfail(LDPC_ENOMEM, err, msg);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return sfail(LDPC_ENODEV, err, "no current CUDA device");
    }
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_addr[dev]) {  // once per device, with that device current
            void* a = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&a, g_static_scratch);
            if (e != cudaSuccess || !a) {
                snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
                cudaGetLastError();
                return sfail(LDPC_EIO, err, msg);
            }
            g_static_addr[dev] = static_cast<unsigned char*>(a);
        }
        base = g_static_addr[dev];
    }
    const void* fn = nw == GEN_WARPS ? (dt == 6    ? pick_mode<6>(p->storage, p->algo, true)
                                        : dt == 8  ? pick_mode<8>(p->storage, p->algo, true)
                                        : dt == 20 ? pick_mode<20>(p->storage, p->algo, true)
                                                   : pick_mode<32>(p->storage, p->algo, true))
                                     : (dt == 6    ? pick_mode<6, 1>(p->storage, p->algo, true)
                                        : dt == 8  ? pick_mode<8, 1>(p->storage, p->algo, true)
                                        : dt == 20 ? pick_mode<20, 1>(p->storage, p->algo, true)
                                                   : pick_mode<32, 1>(p->storage, p->algo, true));
    const size_t smem = (size_t)nw * ((N + 7) & ~7) * esz;
    if (smem > 48 * 1024 && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return sfail(LDPC_ENOTSUP, err, "frame too large for shared memory");
    }
    int per_sm = 0, n_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * nw, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        return sfail(LDPC_ENOTSUP, err, "general kernel does not fit on an SM");
    }
    // The kernel claims frames with a 32-bit counter (and every warp makes one claim past the last
    // frame), so a call decodes its frames in launches of at most 2^31, the counter re-zeroed between
    // them and the tallies summed across them.
    constexpr uint64_t kLaunchFrames = 1ull << 31;
    const uint64_t fit = (LDPC_STATIC_SCRATCH_BYTES - off_msgs) / (nw * per_slot);
    const uint64_t grid = std::min<uint64_t>({(std::min<uint64_t>((uint64_t)n, kLaunchFrames) + nw - 1) / nw,
                                              (uint64_t)per_sm * n_sm, fit});
    unsigned int* d_work = reinterpret_cast<unsigned int*>(base);
    unsigned long long* d_tally = reinterpret_cast<unsigned long long*>(base + 64);
    int32_t* d_rows = reinterpret_cast<int32_t*>(base + off_rows);
    int32_t* d_cols = reinterpret_cast<int32_t*>(base + off_cols);
    int32_t* d_runs = reinterpret_cast<int32_t*>(base + off_runs);
    int32_t* d_nruns = d_runs + (M + 1);
    uint32_t* d_bits = reinterpret_cast<uint32_t*>(base + off_bits);
    cudaError_t e = cudaMemsetAsync(base, 0, 256, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_rows, h->rows, (size_t)M * dmax * 4, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        static_setup_kernel<<<1, 32, 0, stream>>>(d_rows, M, dmax, N, dtc, d_cols, d_runs, d_nruns, d_bits,
                                                  reinterpret_cast<int32_t*>(base + off_lev),
                                                  reinterpret_cast<int32_t*>(base + off_last),
                                                  reinterpret_cast<int32_t*>(base + off_order),
                                                  reinterpret_cast<int32_t*>(base + off_cnt));
        e = cudaGetLastError();
    }
    int32_t n_runs = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n_runs, d_nruns, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "static decode setup: %s", cudaGetErrorString(e));
        return sfail(LDPC_EIO, err, msg);
    }
    for (uint64_t off = 0; e == cudaSuccess && grid > 0 && off < (uint64_t)n; off += kLaunchFrames) {
        const uint64_t cnt = std::min<uint64_t>(kLaunchFrames, (uint64_t)n - off);
        if (off) e = cudaMemsetAsync(d_work, 0, sizeof(unsigned int), stream);
        if (e != cudaSuccess) break;
        GenParams gp;
        memset(&gp, 0, sizeof gp);
        gp.cols = d_cols;
        gp.runs = d_runs;
        gp.n_runs = n_runs;
        gp.N = N;
        gp.M = M;
        gp.n_tx = N - P;
        gp.dmax = dmax;
        gp.max_iter = p->max_iter;
        gp.l_max = p->l_max;
        gp.r_max = p->r_max;
        gp.l_post_max = p->l_post_max;
        gp.n_frames = (uint32_t)cnt;
        gp.r_base = base + off_msgs;
        gp.llr_in = d_llr + off * (uint64_t)(N - P);
        gp.post_out = d_post ? d_post + off * (uint64_t)N : nullptr;
        gp.iters_out = d_iters ? d_iters + off : nullptr;
        gp.synd_out = d_synd ? d_synd + off : nullptr;
        gp.be_out = d_be ? d_be + off : nullptr;
        gp.tally = d_tally;
        gp.hist = nullptr;
        gp.hist_bins = 1;
        gp.work = d_work;
        void* args[] = {&gp};
        e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(32 * nw), args, smem, stream);
    }
    unsigned long long t[TALLY_WORDS] = {};
    if (e == cudaSuccess) e = cudaMemcpyAsync(t, d_tally, sizeof t, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "static decode: %s", cudaGetErrorString(e));
        return sfail(LDPC_EIO, err, msg);
    }
    if (out) {
        out->frames = t[T_FRAMES];
        out->bit_errors = t[T_BIT_ERR];
        out->frame_errors = t[T_FRAME_ERR];
        out->iter_sum = t[T_ITER_SUM];
        out->unconverged = t[T_UNCONVERGED];
        out->max_iters = t[T_MAX_ITER];
        out->kernel_ms = 0.0f;
        out->reserved1 = 0.0f;
        out->bit_errors_sq = t[T_BIT_ERR_SQ];
    }
    return 0;
}

}  // namespace ldpcb200
