// Step kernel for a general parity-check matrix (any .chinn / .chinn.out file, the reference's serial
// row order kept where rows share a variable) and its host side.
//
// Steps of at most 32 rows that share no variable, every pair of rows sharing one in file order (as
// in the warp kernel's general_schedule), each padded to 32 rows so that lane j always takes row j of
// the step, and every row is padded to the kernel's degree bound DT: a lane without a row and an edge past its row's degree point at a dummy posterior slot
// (index N) holding the largest finite value.  Such an edge is never a row's minimum, a min* step with
// it returns the other operand, its sign is +, and the value it writes back rounds to itself, so the
// padded rows update exactly like the real ones (row_update's PAD case) with no per-edge predicate
// and no branch on the row's degree.
//
// One CTA = one warp = one frame slot, so the frame's posteriors start at shared-memory offset 0 and
// the column table holds byte offsets that are the shared-memory addresses themselves.  Variables
// sit in slots chosen against bank conflicts (relabel_slots), which only the channel writes and the
// posterior output look up.  Per step a lane reads its row's byte offsets (DT 32-bit words, laid out
// [step][word group][lane] so that every load of the warp is contiguous) and its row's check
// messages from a global scratch laid out [slot][step][word][lane] (coalesced 4-byte words); both for
// the next step are loaded while the current step's row is updated.  The messages of all resident
// slots stay mostly in L2.
//
// The schedule is the step kernel's own (step_schedule below): steps of one degree class, so that a
// step of rows of degree <= DT/2 runs the row body of DT/2 edges.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ldpc_general.cuh"
#include "ldpc_qc.cuh"  // row_update, RowMsg, LTraits, TallyWord

namespace ldpcb200 {

// 32-bit message words of one row: packed 16-bit pairs, or one fp32 value per edge.
template <int MODE>
__host__ __device__ constexpr int step_words(int dt) {
    return MODE == STORE_FP32 ? dt : (dt + 1) / 2;
}

// Word index of (lane, edge e) inside a step of the column table: DT/4 groups of 4 words per lane
// ([group][lane][4], one 16-byte load each), then for DT % 4 == 2 one group of 2 ([lane][2]).
__host__ __device__ constexpr int step_tab_word(int dt, int lane, int e) {
    return e / 4 < dt / 4 ? (e / 4) * 128 + lane * 4 + (e % 4) : (dt / 4) * 128 + lane * 2 + (e - (dt / 4) * 4);
}

template <int DT>
__device__ __forceinline__ void step_cols(const int32_t* __restrict__ tab, int s, int lane, int (&c)[DT]) {
    static_assert(DT % 2 == 0, "even degree bound");
    const int32_t* b = tab + (size_t)s * (DT * 32);
#pragma unroll
    for (int k = 0; k < DT / 4; ++k) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(b + k * 128) + lane);
        c[4 * k] = v.x;
        c[4 * k + 1] = v.y;
        c[4 * k + 2] = v.z;
        c[4 * k + 3] = v.w;
    }
    if constexpr (DT % 4 == 2) {
        const int2 v = __ldg(reinterpret_cast<const int2*>(b + (DT / 4) * 128) + lane);
        c[DT - 2] = v.x;
        c[DT - 1] = v.y;
    }
}

template <int DT, int MODE>
__device__ __forceinline__ void msg_load(const uint32_t* rs, int s, RowMsg<DT, MODE>& m) {
    constexpr int W = step_words<MODE>(DT);
    const uint32_t* b = rs + (size_t)s * (W * 32);
#pragma unroll
    for (int w = 0; w < W; ++w) {
        if constexpr (MODE == STORE_FP32) m.v[w] = __uint_as_float(__ldcg(b + w * 32));
        else m.w[w] = __ldcg(b + w * 32);
    }
}

// Stores the first WS message words of a row (all of them by default; a low step's rows change only
// the words of their first DT/2 edges).
template <int DT, int MODE, int WS = step_words<MODE>(DT)>
__device__ __forceinline__ void msg_store(uint32_t* rs, int s, const RowMsg<DT, MODE>& m) {
    constexpr int W = step_words<MODE>(DT);
    uint32_t* b = rs + (size_t)s * (W * 32);
#pragma unroll
    for (int w = 0; w < WS; ++w) {
        if constexpr (MODE == STORE_FP32) __stcg(b + w * 32, __float_as_uint(m.v[w]));
        else __stcg(b + w * 32, m.w[w]);
    }
}

// Raw storage bits of the posterior at a byte offset; its sign bit is bit SB.
template <int MODE>
__device__ __forceinline__ uint32_t l_bits(const unsigned char* s, int off) {
    if constexpr (MODE == STORE_BF16) return *reinterpret_cast<const uint16_t*>(s + off);
    else return *reinterpret_cast<const uint32_t*>(s + off);
}
template <int MODE> constexpr int l_sign_bit() { return MODE == STORE_BF16 ? 15 : 31; }

// Resident step-kernel CTAs (one warp each) an SM is compiled for: 32 is the per-SM block limit, and
// 65536 registers / 1024 threads leaves 64 registers a thread.
constexpr int STEP_MIN_CTAS = 32;

template <int DT, int MODE, int ALGO, bool CLIP, bool EXT>
__global__ void __launch_bounds__(32, STEP_MIN_CTAS) general_step_kernel(const __grid_constant__ GenParams p) {
    using LT = LTraits<MODE>;
    using LE = typename LT::T;
    using MSG = RowMsg<DT, MODE>;
    constexpr int W = step_words<MODE>(DT);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LE* L = reinterpret_cast<LE*>(smem_raw);
    const int lane = threadIdx.x;
    const int N = p.N, S = p.n_steps;
    const int32_t* __restrict__ tab = p.scols;
    const int32_t* __restrict__ slot = p.slot;  // shared-memory slot of each variable
    uint32_t* rs = reinterpret_cast<uint32_t*>(p.r_base) + (size_t)blockIdx.x * ((size_t)S * W * 32) + lane;
    const float inf = __int_as_float(0x7f800000);
    const float r_cap = CLIP && p.r_max > 0.0f ? p.r_max : inf;
    unsigned long long t_frames = 0, t_be = 0, t_fe = 0, t_it = 0, t_unc = 0, t_max = 0, t_be2 = 0;

    for (;;) {
        uint32_t fid = 0;
        if (lane == 0) fid = atomicAdd(p.work, 1u);
        fid = __shfl_sync(0xFFFFFFFFu, fid, 0);
        if (fid >= p.n_frames) break;
        const bool per_frame_snr = !EXT && p.ebn0_hi > p.ebn0_lo;
        int snr_bin = 0;
        // channel (as the warp kernel), variable i into its slot
        if (EXT) {
            const float* src = p.llr_in + (size_t)fid * p.n_tx;
            for (int i = lane; i < p.n_tx; i += 32) {
                float x = src[i];
                if (p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                LT::st(L, __ldg(slot + i), x);
            }
        } else {
            const uint64_t gf = p.first_frame + fid;
            float ch_mu = p.mu, ch_sigma = p.sigma;
            if (per_frame_snr)
                frame_snr(p.ebn0_lo, p.ebn0_hi, p.rate, gf, p.stream, p.seed_lo, p.seed_hi, ch_mu, ch_sigma, snr_bin);
            for (int qd = lane; qd * 4 < p.n_tx; qd += 32) {
                float nz[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (ch_sigma > 0.0f) {
                    const U32x4 x = philox4x32_10(U32x4{(uint32_t)qd, (uint32_t)gf, (uint32_t)(gf >> 32), p.stream},
                                                  p.seed_lo, p.seed_hi);
                    box_muller(x.x, x.y, nz[0], nz[1]);
                    box_muller(x.z, x.w, nz[2], nz[3]);
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (4 * qd + k >= p.n_tx) break;
                    float x = ch_sigma > 0.0f ? __fmaf_rn(ch_sigma, nz[k], ch_mu) : ch_mu;
                    if (p.l_max > 0.0f) x = fminf(fmaxf(x, -p.l_max), p.l_max);
                    LT::st(L, __ldg(slot + 4 * qd + k), x);
                }
            }
        }
        for (int i = p.n_tx + lane; i < N; i += 32) LT::st(L, i, 0.0f);
        if (lane == 0) {  // the dummy slot: bf16 0x7F7F, or FLT_MAX
            if constexpr (MODE == STORE_BF16) L[N] = (uint16_t)0x7F7Fu;
            else L[N] = __int_as_float(0x7F7FFFFF);
        }
        __syncwarp();

        int it = 0;
        bool conv = false;
        // Two register sets, A and B, take the steps in turn: while one step's row is updated from
        // one set, the next step's columns and messages (step 0 of the next iteration after the last;
        // in the first iteration a step's messages start at zero) load into the other.
        // A low step (every row of degree <= DT/2) runs the row body of DT/2 edges on the first half
        // of the step's columns and messages: its padded edges past DT/2 are never touched.
        constexpr int DL = DT / 2;
        int cA[DT], cB[DT];
        MSG mA[1], mB[1];
        int lowA = __ldg(p.slow), lowB = 0;
        mA[0].zero();
        step_cols<DT>(tab, 0, lane, cA);
        auto one_step = [&](int s, int (&c)[DT], MSG (&m)[1], int low, int (&cn)[DT], MSG (&mn)[1], int& lown) {
            const int sn = s + 1 < S ? s + 1 : 0;
            step_cols<DT>(tab, sn, lane, cn);
            lown = __ldg(p.slow + sn);
            if (it > 0 || sn == 0) msg_load<DT, MODE>(rs, sn, mn[0]);
            else mn[0].zero();
            if (low) {
                row_update<DL, MODE, ALGO, CLIP, 1, MSG, true, true>(reinterpret_cast<const int(&)[DL]>(c), L, 0, m,
                                                                     r_cap, inf);
                msg_store<DT, MODE, step_words<MODE>(DL)>(rs, s, m[0]);
            } else {
                row_update<DT, MODE, ALGO, CLIP, 1, MSG, true, true>(c, L, 0, m, r_cap, inf);
                msg_store<DT, MODE>(rs, s, m[0]);
            }
            __syncwarp();
        };
        for (;;) {
            if (it >= p.max_iter) break;
            int s = 0;
            for (; s + 1 < S; s += 2) {
                one_step(s, cA, mA, lowA, cB, mB, lowB);
                one_step(s + 1, cB, mB, lowB, cA, mA, lowA);
            }
            if (s < S) {  // an odd step count: the last step leaves step 0 in B
                one_step(s, cA, mA, lowA, cB, mB, lowB);
#pragma unroll
                for (int e = 0; e < DT; ++e) cA[e] = cB[e];
                mA[0] = mB[0];
                lowA = lowB;
            }
            ++it;
            if (it >= 3) {  // syndrome from iteration index 2 on (ldpc_decoder_core.h:526), one step at a time
                bool bad = false;
                for (int s = 0; s < S && !bad; ++s) {
                    int c[DT];
                    step_cols<DT>(tab, s, lane, c);
                    uint32_t x = 0;
#pragma unroll
                    for (int e = 0; e < DT; ++e) x ^= l_bits<MODE>(smem_raw, c[e]);
                    bad = __any_sync(0xFFFFFFFFu, (x >> l_sign_bit<MODE>()) & 1u) != 0;
                }
                if (!bad) {
                    conv = true;
                    break;
                }
            }
        }
        // tally
        uint32_t be = 0;
        for (int i = lane; i < p.n_tx; i += 32) be += LT::sign(L, i);
        be = __reduce_add_sync(0xFFFFFFFFu, be);
        uint32_t sfail = 0;
        if (!conv) {
            for (int s = 0; s < S; ++s) {
                int c[DT];
                step_cols<DT>(tab, s, lane, c);
                uint32_t x = 0;
#pragma unroll
                for (int e = 0; e < DT; ++e) x ^= l_bits<MODE>(smem_raw, c[e]);
                sfail += (x >> l_sign_bit<MODE>()) & 1u;
            }
            sfail = __reduce_add_sync(0xFFFFFFFFu, sfail);
        }
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
        if (EXT && p.post_out) {
            float* dst = p.post_out + (size_t)fid * N;
            for (int i = lane; i < N; i += 32) dst[i] = LT::ld(L, __ldg(slot + i));
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

static int sfail_(std::string& err, int code, const std::string& msg) {
    err = msg;
    return code;
}

// Degree bounds the step kernel is built for.
int step_dt(int maxdeg) { return maxdeg <= 6 ? 6 : maxdeg <= 8 ? 8 : maxdeg <= 10 ? 10 : 0; }

// Shared-memory slots of the posteriors, chosen against bank conflicts.  Every load or store of the
// step kernel's row update is one edge position e of one step across the warp's 32 lanes: the
// variables of that access group should sit in distinct banks (4-byte words w, bank w mod 32).
// Greedy: variables in decreasing order of the groups they belong to, each placed in a free slot of
// the bank holding fewest variables of its groups so far (ties: the bank with most free slots).
// Transmitted variables keep slots in [0, N-P) and punctured ones in [N-P, N), so the kernel's channel
// writes, zeroing and bit-error count cover the same slot ranges.  On the shipped r1/2 K=1024 file's
// schedule this takes the busiest bank of an access from 2.90 words on average to 1.67.
static std::vector<int32_t> relabel_slots(const std::vector<std::vector<int32_t>>& groups, int N, int n_tx,
                                          int esz) {
    std::vector<std::vector<int32_t>> vg(N);
    for (int g = 0; g < (int)groups.size(); ++g)
        for (int32_t v : groups[g]) vg[v].push_back(g);
    std::vector<int32_t> load(groups.size() * 32, 0), slot(N, -1);
    const int per_word = 4 / esz;
    for (int cls = 0; cls < 2; ++cls) {
        const int lo = cls == 0 ? 0 : n_tx, hi = cls == 0 ? n_tx : N;
        std::vector<std::vector<int32_t>> free_(32);
        for (int sl = lo; sl < hi; ++sl) free_[(sl / per_word) % 32].push_back(sl);
        std::vector<size_t> head(32, 0);
        std::vector<int32_t> vs;
        for (int v = lo; v < hi; ++v) vs.push_back(v);
        std::stable_sort(vs.begin(), vs.end(), [&](int32_t a, int32_t b) { return vg[a].size() > vg[b].size(); });
        for (int32_t v : vs) {
            int best = -1;
            long best_c = 0;
            size_t best_free = 0;
            for (int b = 0; b < 32; ++b) {
                const size_t nf = free_[b].size() - head[b];
                if (!nf) continue;
                long c = 0;
                for (int32_t g : vg[v]) c += load[(size_t)g * 32 + b];
                if (best < 0 || c < best_c || (c == best_c && nf > best_free)) {
                    best = b;
                    best_c = c;
                    best_free = nf;
                }
            }
            slot[v] = free_[best][head[best]++];
            for (int32_t g : vg[v]) ++load[(size_t)g * 32 + best];
        }
    }
    return slot;
}

// The step kernel's schedule.  Rows that share no variable commute bit for bit, so any order that
// keeps every pair of rows sharing a variable in file order decodes as the file order does: a row
// depends on the last earlier row on each of its variables.  List scheduling over that dependency
// graph: each step takes up to 32 rows whose predecessors are all in earlier steps (such rows share
// no variable with one another) and of one degree class, low (degree <= dl) or high, so a low step
// runs the kernel's low-degree row body (dl edges) instead of the full one.  The class of a step is
// high when 32 high rows are ready, else low when 32 low rows are, else the class with more ready rows
// (high on a tie); inside a class the rows with the longest chain of dependants go first, then file
// order.  On the shipped r1/2 K=1024 file (512 rows of degree 3, 1024 of degree 6) this gives 36 steps
// of degree 6 and 18 of degree 3 in place of 51 mixed steps.
void step_schedule(const int32_t* rows, int N, int M, int dmax, int dl, std::vector<int32_t>& order,
                   std::vector<int32_t>& starts, std::vector<uint8_t>& low) {
    std::vector<int32_t> deg(M, 0), npred(M, 0), height(M, 1), last(N, -1);
    std::vector<std::vector<int32_t>> succ(M);
    for (int m = 0; m < M; ++m) {
        const int32_t* rv = rows + (size_t)m * dmax;
        for (int e = 0; e < dmax && rv[e] >= 0; ++e) {
            const int32_t p = last[rv[e]];
            if (p >= 0 && (succ[p].empty() || succ[p].back() != m)) {
                succ[p].push_back(m);
                ++npred[m];
            }
            last[rv[e]] = m;
            deg[m] = e + 1;
        }
    }
    for (int m = M - 1; m >= 0; --m)
        for (int32_t s : succ[m]) height[m] = std::max(height[m], height[s] + 1);
    auto before = [&](int32_t a, int32_t b) { return height[a] != height[b] ? height[a] < height[b] : a > b; };
    std::vector<int32_t> ready[2];  // heaps (std::push_heap with `before`): [0] high, [1] low
    auto push = [&](int32_t m) {
        std::vector<int32_t>& q = ready[deg[m] <= dl ? 1 : 0];
        q.push_back(m);
        std::push_heap(q.begin(), q.end(), before);
    };
    for (int m = 0; m < M; ++m)
        if (!npred[m]) push(m);
    order.clear();
    starts.clear();
    low.clear();
    std::vector<int32_t> step;
    while ((int)order.size() < M) {
        const size_t nh = ready[0].size(), nl = ready[1].size();
        int c = nh >= 32 ? 0 : nl >= 32 ? 1 : (nl > nh ? 1 : 0);
        if (ready[c].empty()) c = 1 - c;
        starts.push_back((int32_t)order.size());
        low.push_back((uint8_t)c);
        step.clear();
        while (!ready[c].empty() && step.size() < 32) {
            std::pop_heap(ready[c].begin(), ready[c].end(), before);
            step.push_back(ready[c].back());
            ready[c].pop_back();
        }
        order.insert(order.end(), step.begin(), step.end());
        for (int32_t m : step)
            for (int32_t s : succ[m])
                if (--npred[s] == 0) push(s);
    }
    starts.push_back(M);
}

int build_general_steps(const int32_t* rows, int dmax, GeneralCode* g, std::string& err) {
    int maxdeg = 0;
    for (int m = 0; m < g->M; ++m)
        for (int e = 0; e < dmax && rows[(size_t)m * dmax + e] >= 0; ++e) maxdeg = std::max(maxdeg, e + 1);
    const int dt = step_dt(maxdeg);
    g->sdt = 0;
    if (!dt) return 0;  // the warp kernel decodes this matrix
    std::vector<int32_t> order, starts;
    std::vector<uint8_t> low;
    step_schedule(rows, g->N, g->M, dmax, dt / 2, order, starts, low);
    const int S = (int)starts.size() - 1;
    // the access groups of the row update: edge position e of step s across its lanes
    std::vector<std::vector<int32_t>> groups((size_t)S * dt);
    for (int s = 0; s < S; ++s)
        for (int j = 0; j < starts[s + 1] - starts[s]; ++j) {
            const int32_t* rv = rows + (size_t)order[starts[s] + j] * dmax;
            for (int e = 0; e < dmax && rv[e] >= 0; ++e) groups[(size_t)s * dt + e].push_back(rv[e]);
        }
    for (int k = 0; k < 2; ++k) {
        const int esz = k == 0 ? 2 : 4;
        const std::vector<int32_t> slot = relabel_slots(groups, g->N, g->N - g->P, esz);
        std::vector<int32_t> tab((size_t)S * dt * 32, g->N * esz);
        for (int s = 0; s < S; ++s)
            for (int j = 0; j < starts[s + 1] - starts[s]; ++j) {
                const int32_t* rv = rows + (size_t)order[starts[s] + j] * dmax;
                for (int e = 0; e < dmax && rv[e] >= 0; ++e)
                    tab[(size_t)s * dt * 32 + step_tab_word(dt, j, e)] = slot[rv[e]] * esz;
            }
        if (cudaMalloc(&g->d_scols[k], tab.size() * sizeof(int32_t)) != cudaSuccess ||
            cudaMalloc(&g->d_slot[k], slot.size() * sizeof(int32_t)) != cudaSuccess) {
            cudaGetLastError();
            return sfail_(err, LDPC_ENOMEM, "device allocation failed");
        }
        if (cudaMemcpy(g->d_scols[k], tab.data(), tab.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(g->d_slot[k], slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
            return sfail_(err, LDPC_EIO, "copy of the step table to the device failed");
    }
    const std::vector<int32_t> low32(low.begin(), low.end());
    if (cudaMalloc(&g->d_slow, low32.size() * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        return sfail_(err, LDPC_ENOMEM, "device allocation failed");
    }
    if (cudaMemcpy(g->d_slow, low32.data(), low32.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return sfail_(err, LDPC_EIO, "copy of the step classes to the device failed");
    g->s_steps = S;
    g->sdt = dt;
    return 0;
}

template <int DT, int MODE, int ALGO, bool CLIP>
static const void* sk(bool ext) {
    return ext ? reinterpret_cast<const void*>(&general_step_kernel<DT, MODE, ALGO, CLIP, true>)
               : reinterpret_cast<const void*>(&general_step_kernel<DT, MODE, ALGO, CLIP, false>);
}

template <int DT, int MODE>
static const void* sk_algo(int algo, bool clip, bool ext) {
    if (algo == ALGO_AMIN) return clip ? sk<DT, MODE, ALGO_AMIN, true>(ext) : sk<DT, MODE, ALGO_AMIN, false>(ext);
    return clip ? sk<DT, MODE, ALGO_NMS, true>(ext) : sk<DT, MODE, ALGO_NMS, false>(ext);
}

template <int DT>
static const void* sk_mode(int mode, int algo, bool clip, bool ext) {
    if (mode == STORE_BF16) return sk_algo<DT, STORE_BF16>(algo, clip, ext);
    if (mode == STORE_FP32) return sk_algo<DT, STORE_FP32>(algo, clip, ext);
    return sk_algo<DT, STORE_FP16>(algo, clip, ext);
}

int launch_general_step(GeneralCode* g, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                        const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be,
                        unsigned long long* d_tally, unsigned long long* d_hist, int hist_bins, unsigned int* d_work,
                        int n_sm, cudaStream_t stream, std::string& err, unsigned long long* d_snr_bins) {
    // The posterior clip would clamp the dummy slot; the warp kernel runs it.
    if (!g->sdt || (p->algo != ALGO_AMIN && p->algo != ALGO_NMS) || p->l_post_max > 0.0f) return LDPC_ENOTSUP;
    const bool clip = p->r_max > 0.0f;
    const size_t esz = p->storage == STORE_BF16 ? 2 : 4;
    const size_t smem = (size_t)((g->N + 1 + 7) & ~7) * esz;
    const void* fn = g->sdt == 6   ? sk_mode<6>(p->storage, p->algo, clip, ext)
                     : g->sdt == 8 ? sk_mode<8>(p->storage, p->algo, clip, ext)
                                   : sk_mode<10>(p->storage, p->algo, clip, ext);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return LDPC_ENOTSUP;  // frame too large for one CTA's shared memory: the warp kernel's one-slot CTAs
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32, smem) != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        return LDPC_ENOTSUP;
    }
    if (g->step_ctas > 0) per_sm = std::min(per_sm, g->step_ctas);
    const uint64_t grid = std::min<uint64_t>(n, (uint64_t)per_sm * n_sm);
    if (!grid) return 0;
    const int S = g->s_steps;
    const size_t words = (size_t)S * (p->storage == STORE_FP32 ? g->sdt : g->sdt / 2) * 32;
    const size_t need = grid * words * 4;
    if (g->r_cap < need) {
        cudaFree(g->d_r);
        g->d_r = nullptr;
        g->r_cap = 0;
        if (cudaMalloc(&g->d_r, need) != cudaSuccess) {
            cudaGetLastError();
            return sfail_(err, LDPC_ENOMEM, "message scratch allocation failed");
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
    gp.l_post_max = 0.0f;
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
    gp.scols = g->d_scols[esz == 2 ? 0 : 1];
    gp.slot = g->d_slot[esz == 2 ? 0 : 1];
    gp.slow = g->d_slow;
    gp.n_steps = S;
    void* args[] = {&gp};
    cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(32), args, smem, stream);
    if (e != cudaSuccess) return sfail_(err, LDPC_EIO, std::string("general step kernel launch: ") + cudaGetErrorString(e));
    return 0;
}

}  // namespace ldpcb200
