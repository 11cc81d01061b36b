// General-matrix kernel (any parity-check matrix, the reference's file row order) and its host side.
#include <algorithm>
#include <cstring>
#include <unordered_set>
#include <vector>

#include "ldpc_general.cuh"
#include "ldpc_qc.cuh"  // TallyWord, LTraits

namespace ldpcb200 {

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

// One row of degree deg <= DT, updated by one lane (ldpc_decoder_core.h:414-520).
template <int DT, int MODE, int ALGO>
__device__ __forceinline__ void gen_row(const GenParams& p, int m, typename LTraits<MODE>::T* L,
                                        typename RTraits<MODE>::T* r, float r_cap, float lp_cap) {
    using LT = LTraits<MODE>;
    using RT = RTraits<MODE>;
    const int M = p.M;
    int deg = 0;
    int col[DT];
    float q[DT];
#pragma unroll
    for (int e = 0; e < DT; ++e) {
        col[e] = e < p.dmax ? p.cols[e * M + m] : -1;
        if (col[e] >= 0) deg = e + 1;
    }
    if (deg == 0) return;
    uint32_t par = 0;
#pragma unroll
    for (int e = 0; e < DT; ++e)
        if (e < deg) {
            q[e] = __fsub_rn(LT::ld(L, col[e]), RT::ld(r + (size_t)e * M + m));
            par ^= __float_as_uint(q[e]);
        }
    par &= 0x80000000u;
    int am = 0;
    float mag_min, mag_all;
    if (ALGO == ALGO_AMIN) {
        float mn = 9999.0f;
#pragma unroll
        for (int e = 0; e < DT; ++e)
            if (e < deg) {
                const float a = fabsf(q[e]);
                if (a < mn) { mn = a; am = e; }
            }
        float mo = __int_as_float(0x7f800000);
#pragma unroll
        for (int e = 0; e < DT; ++e)
            if (e < deg && e != am) mo = amin_step(mo, fabsf(q[e]));
        if (deg == 1) mo = mn;  // m_others = min_mag when the row has one edge (:181)
        mag_min = mo;
        mag_all = amin_step(mo, mn);
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
            RT::st(r + (size_t)e * M + m, rn);
        }
}

template <int DT, int MODE, int ALGO, bool EXT>
__global__ void __launch_bounds__(32 * GEN_WARPS) general_kernel(const __grid_constant__ GenParams p) {
    using LT = LTraits<MODE>;
    using LE = typename LT::T;
    using RE = typename RTraits<MODE>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int N = p.N, M = p.M;
    const int lstride = (N + 7) & ~7;
    LE* L = reinterpret_cast<LE*>(smem_raw) + (size_t)warp * lstride;
    const size_t slot = (size_t)blockIdx.x * GEN_WARPS + warp;
    RE* r = reinterpret_cast<RE*>(p.r_base) + slot * (size_t)p.dmax * M;
    const float r_cap = p.r_max > 0.0f ? p.r_max : __int_as_float(0x7f800000);
    const float lp_cap = p.l_post_max > 0.0f ? p.l_post_max : __int_as_float(0x7f800000);
    unsigned long long t_frames = 0, t_be = 0, t_fe = 0, t_it = 0, t_unc = 0, t_max = 0;

    for (;;) {
        uint32_t fid = 0;
        if (lane == 0) fid = atomicAdd(p.work, 1u);
        fid = __shfl_sync(0xFFFFFFFFu, fid, 0);
        if (fid >= p.n_frames) break;
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
            for (int qd = lane; qd * 4 < p.n_tx; qd += 32) {
                float n[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (p.sigma > 0.0f) {
                    const U32x4 x = philox4x32_10(U32x4{(uint32_t)qd, (uint32_t)gf, (uint32_t)(gf >> 32), p.stream},
                                                  p.seed_lo, p.seed_hi);
                    box_muller(x.x, x.y, n[0], n[1]);
                    box_muller(x.z, x.w, n[2], n[3]);
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (4 * qd + k >= p.n_tx) break;
                    float x = p.sigma > 0.0f ? __fmaf_rn(p.sigma, n[k], p.mu) : p.mu;
                    if (p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                    LT::st(L, 4 * qd + k, x);
                }
            }
        }
        for (int i = p.n_tx + lane; i < N; i += 32) LT::st(L, i, 0.0f);
        for (size_t i = lane; i < (size_t)p.dmax * M; i += 32) r[i] = RE(0);
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
                uint32_t bad = 0;
                for (int m = lane; m < M && !bad; m += 32) {
                    uint32_t par = 0;
                    for (int e = 0; e < p.dmax; ++e) {
                        const int c = p.cols[e * M + m];
                        if (c < 0) break;
                        par ^= __float_as_uint(LT::ld(L, c)) >> 31;
                    }
                    bad |= par;
                }
                if (!__any_sync(0xFFFFFFFFu, bad)) break;
            }
        }
        // tally
        uint32_t be = 0;
        for (int i = lane; i < p.n_tx; i += 32) be += __float_as_uint(LT::ld(L, i)) >> 31;
        be = __reduce_add_sync(0xFFFFFFFFu, be);
        for (int m = lane; m < M; m += 32) {
            uint32_t par = 0;
            for (int e = 0; e < p.dmax; ++e) {
                const int c = p.cols[e * M + m];
                if (c < 0) break;
                par ^= __float_as_uint(LT::ld(L, c)) >> 31;
            }
            sfail += par;
        }
        sfail = __reduce_add_sync(0xFFFFFFFFu, sfail);
        if (lane == 0) {
            t_frames += 1;
            t_be += be;
            t_fe += be > 0;
            t_it += (unsigned)it;
            t_unc += sfail != 0;
            t_max = max(t_max, (unsigned long long)it);
            if (p.hist) atomicAdd(&p.hist[min(it, p.hist_bins - 1)], 1ull);
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
    }
}

// ----------------------------------------------------------------------------- host side

static int gfail(std::string& err, int code, const std::string& msg) {
    err = msg;
    return code;
}

int build_general(const int32_t* rows, int N, int M, int P, int dmax, GeneralCode* g, std::string& err) {
    g->N = N;
    g->M = M;
    g->P = P;
    g->dmax = dmax;
    int maxdeg = 0;
    std::vector<int32_t> cols((size_t)dmax * M, -1);
    std::vector<int32_t> runs{0};
    std::unordered_set<int32_t> used;
    for (int m = 0; m < M; ++m) {
        int d = 0;
        std::vector<int32_t> rv;
        for (int e = 0; e < dmax; ++e) {
            const int32_t c = rows[(size_t)m * dmax + e];
            if (c < 0) break;
            cols[(size_t)e * M + m] = c;
            rv.push_back(c);
            d = e + 1;
        }
        maxdeg = std::max(maxdeg, d);
        bool clash = false;
        for (int32_t c : rv) clash |= used.count(c) > 0;
        if (clash) {
            runs.push_back(m);
            used.clear();
        }
        for (int32_t c : rv) used.insert(c);
    }
    runs.push_back(M);
    g->n_runs = (int)runs.size() - 1;
    g->dt = maxdeg <= 8 ? 8 : maxdeg <= 20 ? 20 : maxdeg <= 32 ? 32 : 0;
    if (!g->dt) return gfail(err, LDPC_ENOTSUP, "row degree above 32 is not supported");
    if (cudaMalloc(&g->d_cols, cols.size() * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&g->d_runs, runs.size() * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        return gfail(err, LDPC_ENOMEM, "device allocation failed");
    }
    if (cudaMemcpy(g->d_cols, cols.data(), cols.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g->d_runs, runs.data(), runs.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return gfail(err, LDPC_EIO, "copy of the matrix to the device failed");
    return 0;
}

void free_general(GeneralCode* g) {
    cudaFree(g->d_cols);
    cudaFree(g->d_runs);
    cudaFree(g->d_r);
    g->d_cols = g->d_runs = nullptr;
    g->d_r = nullptr;
    g->r_cap = 0;
}

template <int DT, int MODE, int ALGO, bool EXT>
static const void* gk() {
    return reinterpret_cast<const void*>(&general_kernel<DT, MODE, ALGO, EXT>);
}

template <int DT, int MODE>
static const void* pick_algo(int algo, bool ext) {
    if (algo == ALGO_AMIN) return ext ? gk<DT, MODE, ALGO_AMIN, true>() : gk<DT, MODE, ALGO_AMIN, false>();
    return ext ? gk<DT, MODE, ALGO_NMS, true>() : gk<DT, MODE, ALGO_NMS, false>();
}

template <int DT>
static const void* pick_mode(int mode, int algo, bool ext) {
    if (mode == STORE_BF16) return pick_algo<DT, STORE_BF16>(algo, ext);
    if (mode == STORE_FP32) return pick_algo<DT, STORE_FP32>(algo, ext);
    return pick_algo<DT, STORE_FP16>(algo, ext);
}

int launch_general(GeneralCode* g, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                   const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be,
                   unsigned long long* d_tally, unsigned long long* d_hist, int hist_bins, unsigned int* d_work,
                   int n_sm, cudaStream_t stream, std::string& err) {
    const void* fn = g->dt == 8    ? pick_mode<8>(p->storage, p->algo, ext)
                     : g->dt == 20 ? pick_mode<20>(p->storage, p->algo, ext)
                                   : pick_mode<32>(p->storage, p->algo, ext);
    const size_t esz = p->storage == STORE_BF16 ? 2 : 4;
    const size_t smem = (size_t)GEN_WARPS * ((g->N + 7) & ~7) * esz;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return gfail(err, LDPC_ENOTSUP, "general kernel: frame too large for shared memory");
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * GEN_WARPS, smem) != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        return gfail(err, LDPC_ENOTSUP, "general kernel does not fit on an SM");
    }
    const uint64_t want = (n + GEN_WARPS - 1) / GEN_WARPS;
    const uint64_t grid = std::min<uint64_t>(want, (uint64_t)per_sm * n_sm);
    if (!grid) return 0;
    const size_t rsz = p->storage == STORE_FP32 ? 4 : 2;
    const size_t need = grid * GEN_WARPS * (size_t)g->dmax * g->M * rsz;
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
    void* args[] = {&gp};
    cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(32 * GEN_WARPS), args, smem, stream);
    if (e != cudaSuccess) return gfail(err, LDPC_EIO, std::string("general kernel launch: ") + cudaGetErrorString(e));
    return 0;
}

}  // namespace ldpcb200
