// Weighted Approximate-Min* decoder: forward and adjoint kernels (see ldpc_weighted.cuh).
//
// Both kernels are templates over the real type.  float is the training and simulation type; its
// arithmetic is the plain decoder's (the same correctly rounded operations in the same order, the
// same min* step), so alpha = 1, beta = 0 gives the plain fp32 decoder's values bit for bit.  double
// exists to check the adjoint against central finite differences, which need more precision than
// float has.
#include <cstdio>
#include <string>

#include "../../include/ldpcb200.h"
#include "ldpc_weighted.cuh"

namespace ldpcb200 {

template <typename Real>
struct WOps;

template <>
struct WOps<float> {
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float abs(float a) { return fabsf(a); }
    static __device__ __forceinline__ float min(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ uint32_t neg(float a) { return __float_as_uint(a) >> 31; }
    static __device__ __forceinline__ float with_sign(float mag, uint32_t neg) {
        return __uint_as_float((__float_as_uint(mag) & 0x7FFFFFFFu) | (neg << 31));
    }
    static __device__ __forceinline__ float step(float m, float a) { return amin_step_fma(m, a); }
};

template <>
struct WOps<double> {
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double abs(double a) { return fabs(a); }
    static __device__ __forceinline__ double min(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ uint32_t neg(double a) {
        return (uint32_t)((unsigned long long)__double_as_longlong(a) >> 63);
    }
    static __device__ __forceinline__ double with_sign(double mag, uint32_t neg) {
        const unsigned long long u = ((unsigned long long)__double_as_longlong(mag) & 0x7FFFFFFFFFFFFFFFull) |
                                     ((unsigned long long)neg << 63);
        return __longlong_as_double((long long)u);
    }
    // max(min(m, a) - g(|m - a|), 0), g = 0.69315 - 0.4 d (d < 0.5), 0.49315 - 0.328 (d - 0.5) (d < 2), 0
    static __device__ __forceinline__ double step(double m, double a) {
        const double diff = fabs(__dsub_rn(m, a));
        const double cur = fmin(m, a);
        const double g = diff < 0.5 ? __dsub_rn(0.69315, __dmul_rn(0.40, diff))
                                    : (diff < 2.0 ? __dsub_rn(0.49315, __dmul_rn(0.328, __dsub_rn(diff, 0.5))) : 0.0);
        const double v = __dsub_rn(cur, g);
        return v > 0.0 ? v : 0.0;
    }
};

// One min* step with its partial derivatives.  Where the result is clamped to 0 both derivatives are
// 0; at m == a the minimum's derivative goes to a (a subgradient).
template <typename Real>
__device__ __forceinline__ Real wstep_grad(Real m, Real a, Real& dm, Real& da) {
    const Real v = WOps<Real>::step(m, a);
    if (!(v > Real(0))) {
        dm = Real(0);
        da = Real(0);
        return v;
    }
    const Real diff = WOps<Real>::abs(WOps<Real>::sub(m, a));
    const Real gp = diff < Real(0.5) ? Real(-0.40) : (diff < Real(2.0) ? Real(-0.328) : Real(0));
    const Real sg = m > a ? Real(1) : (m < a ? Real(-1) : Real(0));
    const Real cm = m < a ? Real(1) : Real(0);
    dm = cm - gp * sg;
    da = (Real(1) - cm) + gp * sg;
    return v;
}

// Row structure shared by forward and backward: sign parity, argmin flags and the prefix-min test
// lt[i] ("the argmin lies after edge i"), as the plain decoder's row update.
template <typename Real, int d>
__device__ __forceinline__ Real wrow_prep(const Real (&q)[d], uint32_t& par, bool (&lt)[d], bool (&is_am)[d]) {
    using O = WOps<Real>;
    par = 0;
#pragma unroll
    for (int e = 0; e < d; ++e) par ^= O::neg(q[e]);
    Real pm[d];
    pm[0] = O::min(O::abs(q[0]), Real(9999));
#pragma unroll
    for (int e = 1; e < d; ++e) pm[e] = O::min(pm[e - 1], O::abs(q[e]));
    const Real mn = pm[d - 1];
#pragma unroll
    for (int i = 0; i < d; ++i) lt[i] = (i + 1 < d) ? (pm[i] > mn) : false;
#pragma unroll
    for (int e = 0; e < d; ++e) is_am[e] = (e == 0 ? true : lt[e - 1]) && !lt[e];
    return mn;
}

// One weighted row, forward: q in, new messages out.
template <typename Real, int d>
__device__ __forceinline__ void wrow_forward(const Real (&q)[d], const Real (&al)[d], const Real (&be)[d],
                                             Real (&rn)[d]) {
    using O = WOps<Real>;
    uint32_t par;
    bool lt[d], is_am[d];
    const Real mn = wrow_prep<Real, d>(q, par, lt, is_am);
    Real m = O::abs(lt[0] ? q[0] : q[1]);
#pragma unroll
    for (int i = 1; i + 1 < d; ++i) m = O::step(m, O::abs(lt[i] ? q[i] : q[i + 1]));
    const Real mall = O::step(m, mn);
#pragma unroll
    for (int e = 0; e < d; ++e) {
        Real z = O::sub(O::mul(al[e], is_am[e] ? m : mall), be[e]);
        z = z > Real(0) ? z : Real(0);
        rn[e] = O::with_sign(z, par ^ O::neg(q[e]));
    }
}

// One weighted row, backward.  A[e]: adjoint of the new message r_e (its own later uses plus the new
// L_v = q_e + r_e); gLv[e]: adjoint of the new L_v.  Out: gq[e] (adjoint of q_e) and the per-edge
// parameter gradients.
template <typename Real, int d>
__device__ __forceinline__ void wrow_backward(const Real (&q)[d], const Real (&al)[d], const Real (&be)[d],
                                              const Real (&A)[d], const Real (&gLv)[d], Real (&gq)[d],
                                              Real (&ga)[d], Real (&gb)[d]) {
    using O = WOps<Real>;
    uint32_t par;
    bool lt[d], is_am[d];
    const Real mn = wrow_prep<Real, d>(q, par, lt, is_am);
    // chain with derivatives: m_1 = |o_0|, m_{i+1} = step(m_i, |o_i|), o_i the i-th non-argmin edge
    Real dmi[d > 2 ? d - 2 : 1], doi[d > 2 ? d - 2 : 1];
    Real m = O::abs(lt[0] ? q[0] : q[1]);
#pragma unroll
    for (int i = 1; i + 1 < d; ++i) m = wstep_grad<Real>(m, O::abs(lt[i] ? q[i] : q[i + 1]), dmi[i - 1], doi[i - 1]);
    Real dm_all, dmn_all;
    const Real mall = wstep_grad<Real>(m, mn, dm_all, dmn_all);
    Real g_min = Real(0), g_all = Real(0);
#pragma unroll
    for (int e = 0; e < d; ++e) {
        const Real mag = is_am[e] ? m : mall;
        const Real z = O::sub(O::mul(al[e], mag), be[e]);
        const Real sgn = ((par ^ O::neg(q[e])) & 1u) ? Real(-1) : Real(1);
        const Real w = z > Real(0) ? A[e] * sgn : Real(0);
        ga[e] = w * mag;
        gb[e] = -w;
        const Real gmag = w * al[e];
        if (is_am[e]) g_min += gmag; else g_all += gmag;
    }
    Real gm = g_min + g_all * dm_all;
    const Real gmn = g_all * dmn_all;
    Real go[d > 1 ? d - 1 : 1];
#pragma unroll
    for (int i = d - 2; i >= 1; --i) {
        go[i] = gm * doi[i - 1];
        gm = gm * dmi[i - 1];
    }
    go[0] = gm;
#pragma unroll
    for (int e = 0; e < d; ++e) {
        const Real gabs = is_am[e] ? gmn : (lt[e] ? go[e] : go[e > 0 ? e - 1 : 0]);
        gq[e] = gLv[e] + (O::neg(q[e]) ? -gabs : gabs);
    }
}

template <typename Real>
__device__ __forceinline__ Real warp_sum(Real v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// The parameters of iteration t for the edges of layer l.
template <typename Real, int d>
__device__ __forceinline__ void wparams(const WParams& p, const Real* sa, const Real* sb, int t, int l, Real (&al)[d],
                                        Real (&be)[d]) {
#pragma unroll
    for (int e = 0; e < d; ++e) {
        const int c = p.edge_class[l][e];
        al[e] = sa[t * p.n_classes + c];
        be[e] = sb[t * p.n_classes + c];
    }
}

// Forward update of row j of layer l (degree d): q from L and the old messages, new messages and L.
// With a stash, q is also written there (the backward pass's recomputation).
template <typename Real, int Z, int d>
__device__ __forceinline__ void wlayer_row_fwd(const WParams& p, Real* L, Real* r, Real* stash, const Real* sa,
                                               const Real* sb, int t, int l, int j) {
    Real q[d], al[d], be[d], rn[d];
    int idx[d];
#pragma unroll
    for (int e = 0; e < d; ++e) {
        idx[e] = p.blk_off[l][e] + ((j + p.shift[l][e]) & (Z - 1));
        const int k = p.layer_off[l] + e * Z + j;
        q[e] = WOps<Real>::sub(L[idx[e]], r[k]);
        if (stash) stash[k] = q[e];
    }
    wparams<Real, d>(p, sa, sb, t, l, al, be);
    wrow_forward<Real, d>(q, al, be, rn);
#pragma unroll
    for (int e = 0; e < d; ++e) {
        L[idx[e]] = WOps<Real>::add(q[e], rn[e]);
        r[p.layer_off[l] + e * Z + j] = rn[e];
    }
}

// Backward of row j of layer l: adjoints of L (shared) and of the messages (global) in place, the
// parameter gradients summed over the warp into the block's accumulators.
template <typename Real, int Z, int d>
__device__ __forceinline__ void wlayer_row_bwd(const WParams& p, Real* gL, Real* gr, const Real* stash, const Real* sa,
                                               const Real* sb, Real* ga_acc, Real* gb_acc, int t, int l, int j,
                                               int lane) {
    Real q[d], al[d], be[d], A[d], gLv[d], gq[d], gal[d], gbe[d];
    int idx[d];
#pragma unroll
    for (int e = 0; e < d; ++e) {
        idx[e] = p.blk_off[l][e] + ((j + p.shift[l][e]) & (Z - 1));
        const int k = p.layer_off[l] + e * Z + j;
        q[e] = stash[k];
        gLv[e] = gL[idx[e]];
        A[e] = gLv[e] + gr[k];
    }
    wparams<Real, d>(p, sa, sb, t, l, al, be);
    wrow_backward<Real, d>(q, al, be, A, gLv, gq, gal, gbe);
#pragma unroll
    for (int e = 0; e < d; ++e) {
        gL[idx[e]] = gq[e];
        gr[p.layer_off[l] + e * Z + j] = -gq[e];
        const Real sa_ = warp_sum<Real>(gal[e]), sb_ = warp_sum<Real>(gbe[e]);
        if (lane == 0) {
            atomicAdd(&ga_acc[t * p.n_classes + p.edge_class[l][e]], sa_);
            atomicAdd(&gb_acc[t * p.n_classes + p.edge_class[l][e]], sb_);
        }
    }
}

// Shared-memory arrays are padded to 16 bytes.
template <typename Real>
__host__ __device__ constexpr int wpad(int n) {
    return (n + (int)(16 / sizeof(Real)) - 1) & ~((int)(16 / sizeof(Real)) - 1);
}

// One CTA per frame, Z/R threads; thread tid updates rows tid + rho*T of every layer and is the only
// thread that touches those rows' messages (element layer_off + e*Z + row), so the message array
// needs no synchronisation; L lives in shared memory, a barrier after every layer.
template <typename Real, int Z, int D, int R>
__global__ void __launch_bounds__(Z / R) wfwd_kernel(const __grid_constant__ WParams p) {
    constexpr int T = Z / R;
    extern __shared__ __align__(16) unsigned char smw_raw[];
    Real* smw = reinterpret_cast<Real*>(smw_raw);
    const int N = p.n_vars, E = p.n_edges, TC = p.n_iter * p.n_classes;
    Real* L = smw;
    Real* sa = L + wpad<Real>(N);
    Real* sb = sa + wpad<Real>(TC);
    const int b = blockIdx.x, tid = threadIdx.x;
    const Real* alpha = static_cast<const Real*>(p.alpha);
    const Real* beta = static_cast<const Real*>(p.beta);
    for (int i = tid; i < TC; i += T) {
        sa[i] = alpha[i];
        sb[i] = beta[i];
    }
    const Real* llr = static_cast<const Real*>(p.llr) + (size_t)b * p.n_tx;
    for (int i = tid; i < N; i += T) L[i] = i < p.n_tx ? llr[i] : Real(0);
    Real* r = static_cast<Real*>(p.rwork) + (size_t)b * E;
    for (int i = tid; i < E; i += T) r[i] = Real(0);
    Real* ckpt = static_cast<Real*>(p.ckpt);
    Real* post = static_cast<Real*>(p.post);
    __syncthreads();
    for (int t = 0; t < p.n_iter; ++t) {
        if (t % p.ckpt_every == 0) {
            Real* ck = ckpt + ((size_t)(t / p.ckpt_every) * p.n_frames + b) * (size_t)(N + E);
            for (int i = tid; i < N; i += T) ck[i] = L[i];
            for (int i = tid; i < E; i += T) ck[N + i] = r[i];
            __syncthreads();
        }
#pragma unroll
        for (int l = 0; l < QC_LAYERS; ++l) {
#pragma unroll
            for (int rho = 0; rho < R; ++rho) {
                if (l < 4)
                    wlayer_row_fwd<Real, Z, QC_DEG_LOW>(p, L, r, nullptr, sa, sb, t, l, tid + rho * T);
                else
                    wlayer_row_fwd<Real, Z, D>(p, L, r, nullptr, sa, sb, t, l, tid + rho * T);
            }
            __syncthreads();
        }
        if (p.post_all || t == p.n_iter - 1) {
            Real* dst = post + ((size_t)(p.post_all ? t : 0) * p.n_frames + b) * N;
            for (int i = tid; i < N; i += T) dst[i] = L[i];
        }
    }
}

// Adjoint: segments of ckpt_every iterations in reverse; each is recomputed from its checkpoint
// (stashing every layer's q), then walked back layer by layer.
template <typename Real, int Z, int D, int R>
__global__ void __launch_bounds__(Z / R) wbwd_kernel(const __grid_constant__ WParams p) {
    constexpr int T = Z / R;
    extern __shared__ __align__(16) unsigned char smw_raw[];
    Real* smw = reinterpret_cast<Real*>(smw_raw);
    const int N = p.n_vars, E = p.n_edges, TC = p.n_iter * p.n_classes;
    Real* L = smw;
    Real* gL = L + wpad<Real>(N);
    Real* sa = gL + wpad<Real>(N);
    Real* sb = sa + wpad<Real>(TC);
    Real* ga_acc = sb + wpad<Real>(TC);
    Real* gb_acc = ga_acc + wpad<Real>(TC);
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
    const Real* alpha = static_cast<const Real*>(p.alpha);
    const Real* beta = static_cast<const Real*>(p.beta);
    for (int i = tid; i < TC; i += T) {
        sa[i] = alpha[i];
        sb[i] = beta[i];
        ga_acc[i] = Real(0);
        gb_acc[i] = Real(0);
    }
    for (int i = tid; i < N; i += T) gL[i] = Real(0);
    Real* r = static_cast<Real*>(p.rwork) + (size_t)b * E;
    Real* gr = static_cast<Real*>(p.gr) + (size_t)b * E;
    Real* st = static_cast<Real*>(p.stash) + (size_t)b * p.ckpt_every * E;
    const Real* ckpt = static_cast<const Real*>(p.ckpt);
    const Real* gpost = static_cast<const Real*>(p.gpost);
    for (int i = tid; i < E; i += T) gr[i] = Real(0);
    __syncthreads();
    const int n_seg = (p.n_iter + p.ckpt_every - 1) / p.ckpt_every;
    for (int seg = n_seg - 1; seg >= 0; --seg) {
        const int t0 = seg * p.ckpt_every, t1 = min(p.n_iter, t0 + p.ckpt_every);
        const Real* ck = ckpt + ((size_t)seg * p.n_frames + b) * (size_t)(N + E);
        for (int i = tid; i < N; i += T) L[i] = ck[i];
        for (int i = tid; i < E; i += T) r[i] = ck[N + i];
        __syncthreads();
        for (int t = t0; t < t1; ++t) {
            Real* sq = st + (size_t)(t - t0) * E;
#pragma unroll
            for (int l = 0; l < QC_LAYERS; ++l) {
#pragma unroll
                for (int rho = 0; rho < R; ++rho) {
                    if (l < 4)
                        wlayer_row_fwd<Real, Z, QC_DEG_LOW>(p, L, r, sq, sa, sb, t, l, tid + rho * T);
                    else
                        wlayer_row_fwd<Real, Z, D>(p, L, r, sq, sa, sb, t, l, tid + rho * T);
                }
                __syncthreads();
            }
        }
        for (int t = t1 - 1; t >= t0; --t) {
            if (gpost && (p.post_all || t == p.n_iter - 1)) {
                const Real* gp = gpost + ((size_t)(p.post_all ? t : 0) * p.n_frames + b) * N;
                for (int i = tid; i < N; i += T) gL[i] += gp[i];
                __syncthreads();
            }
            const Real* sq = st + (size_t)(t - t0) * E;
#pragma unroll
            for (int l = QC_LAYERS - 1; l >= 0; --l) {
#pragma unroll
                for (int rho = 0; rho < R; ++rho) {
                    if (l < 4)
                        wlayer_row_bwd<Real, Z, QC_DEG_LOW>(p, gL, gr, sq, sa, sb, ga_acc, gb_acc, t, l,
                                                            tid + rho * T, lane);
                    else
                        wlayer_row_bwd<Real, Z, D>(p, gL, gr, sq, sa, sb, ga_acc, gb_acc, t, l, tid + rho * T,
                                                   lane);
                }
                __syncthreads();
            }
        }
    }
    if (p.gllr) {
        Real* g = static_cast<Real*>(p.gllr) + (size_t)b * p.n_tx;
        for (int i = tid; i < p.n_tx; i += T) g[i] = gL[i];
    }
    Real* galpha = static_cast<Real*>(p.galpha);
    Real* gbeta = static_cast<Real*>(p.gbeta);
    for (int i = tid; i < TC; i += T) {
        if (ga_acc[i] != Real(0)) atomicAdd(&galpha[i], ga_acc[i]);
        if (gb_acc[i] != Real(0)) atomicAdd(&gbeta[i], gb_acc[i]);
    }
}

// ----------------------------------------------------------------------------- host side

size_t weighted_smem_bytes(const WParams& p, bool fwd, int real_bytes) {
    const int TC = p.n_iter * p.n_classes;
    if (real_bytes == 8)
        return fwd ? (size_t)(wpad<double>(p.n_vars) + 2 * wpad<double>(TC)) * 8
                   : (size_t)(2 * wpad<double>(p.n_vars) + 4 * wpad<double>(TC)) * 8;
    return fwd ? (size_t)(wpad<float>(p.n_vars) + 2 * wpad<float>(TC)) * 4
               : (size_t)(2 * wpad<float>(p.n_vars) + 4 * wpad<float>(TC)) * 4;
}

template <typename Real, int Z, int D, int R>
static int wlaunch(const WParams& p, bool fwd, cudaStream_t s, std::string& err) {
    constexpr int T = Z / R;
    static_assert(T % 32 == 0, "the parameter-gradient reduction needs whole warps");
    const void* fn = fwd ? reinterpret_cast<const void*>(&wfwd_kernel<Real, Z, D, R>)
                         : reinterpret_cast<const void*>(&wbwd_kernel<Real, Z, D, R>);
    const size_t smem = weighted_smem_bytes(p, fwd, (int)sizeof(Real));
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        err = "weighted decoder: frame too large for shared memory";
        return LDPC_ENOTSUP;
    }
    void* args[] = {const_cast<WParams*>(&p)};
    const cudaError_t e = cudaLaunchKernel(fn, dim3(p.n_frames), dim3(T), args, smem, s);
    if (e != cudaSuccess) {
        err = std::string("weighted decoder launch: ") + cudaGetErrorString(e);
        return LDPC_EIO;
    }
    return 0;
}

// Code shapes (Z, D, rows per thread) of the float kernels: rate 1/2 and 4/5 at K = 1024 and 4096,
// rate 2/3 at K = 1024.  The double kernels (adjoint checks) cover rate 1/2 and 4/5 at K = 1024.
#define W_SHAPES_F32(X) X(128, 6, 1) X(512, 6, 1) X(64, 10, 1) X(32, 18, 1) X(128, 18, 1)
#define W_SHAPES_F64(X) X(128, 6, 1) X(32, 18, 1)

bool weighted_supported(int Z, int D, int real_bytes) {
#define W_SUP(z, d, r) if (Z == z && D == d) return true;
    if (real_bytes == 4) { W_SHAPES_F32(W_SUP) }
    if (real_bytes == 8) { W_SHAPES_F64(W_SUP) }
#undef W_SUP
    return false;
}

static int wdispatch(const WParams& p, int Z, int D, int real_bytes, bool fwd, cudaStream_t s, std::string& err) {
#define W_CALL_F32(z, d, r) if (Z == z && D == d) return wlaunch<float, z, d, r>(p, fwd, s, err);
#define W_CALL_F64(z, d, r) if (Z == z && D == d) return wlaunch<double, z, d, r>(p, fwd, s, err);
    if (real_bytes == 4) { W_SHAPES_F32(W_CALL_F32) }
    if (real_bytes == 8) { W_SHAPES_F64(W_CALL_F64) }
#undef W_CALL_F32
#undef W_CALL_F64
    err = "weighted decoder is not built for this code shape";
    return LDPC_ENOTSUP;
}

int weighted_forward(const WParams& p, int Z, int D, int real_bytes, cudaStream_t s, std::string& err) {
    return p.n_frames ? wdispatch(p, Z, D, real_bytes, true, s, err) : 0;
}

int weighted_backward(const WParams& p, int Z, int D, int real_bytes, cudaStream_t s, std::string& err) {
    return p.n_frames ? wdispatch(p, Z, D, real_bytes, false, s, err) : 0;
}

}  // namespace ldpcb200
