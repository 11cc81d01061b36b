// Host side of libldpcb200: handles, structure detection, launch configuration, and the C ABI of
// include/ldpcb200.h.  No CPU decoding path exists: every decode runs in a CUDA kernel, and a shape
// that was not compiled is an error (LDPC_ENOTSUP).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ldpcb200.h"
#include "ldpc_general.cuh"
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"
#include "ldpc_weighted.cuh"

using namespace ldpcb200;

// ----------------------------------------------------------------------------- errors
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(LDPC_EIO, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ----------------------------------------------------------------------------- registry
namespace ldpcb200 {
static const QcTable* g_tables = nullptr;
void register_qc_table(QcTable* t) {
    t->next = g_tables;
    g_tables = t;
}
const QcTable* qc_tables() { return g_tables; }
}  // namespace ldpcb200

static const void* find_qc(const QcKey& k) {
    for (const QcTable* t = qc_tables(); t; t = t->next)
        for (int i = 0; i < t->count; ++i)
            if (t->entries[i].key == k) return t->entries[i].fn;
    return nullptr;
}

// ----------------------------------------------------------------------------- handle
struct ldpc_handle {
    int device = 0;
    int kind = LDPC_KERNEL_GENERAL;
    int n_sm = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // code
    int N = 0, M = 0, P = 0, dmax = 0;
    std::vector<int32_t> rows;  // [M][dmax]
    // QC structure
    int Z = 0, D = 0;
    int32_t blk_off[QC_LAYERS][QC_DMAX] = {};
    int32_t shift[QC_LAYERS][QC_DMAX] = {};
    int fix = -1;  // index of kQcFixedHost holding exactly these descriptors (layout 5 kernels), or -1
    // per storage mode: rows per thread, frames per CTA, min CTAs/SM, messages in global memory;
    // all zero = the default shape
    int shape[3][4] = {};
    void* d_rmsg = nullptr;  // message scratch of RG kernels
    size_t rmsg_cap = 0;
    bool gen_built = false;
    // general structure (device)
    GeneralCode gen{};
    // device scratch
    unsigned long long* d_tally = nullptr;  // [TALLY_WORDS]
    unsigned int* d_work = nullptr;
    unsigned long long* d_hist = nullptr;
    int hist_bins = 0;
    unsigned long long* d_snr = nullptr;  // [4][SNR_BINS]
    float* d_llr = nullptr;
    size_t llr_cap = 0;
    float* d_post = nullptr;
    size_t post_cap = 0;
    int32_t* d_frame_out = nullptr;  // 3 * cap
    size_t frame_cap = 0;
    // weights of LDPC_ALGO_WAMIN runs
    float2* d_wtab = nullptr;  // [w_iters][w_slots] (alpha, beta) per iteration and edge slot
    int w_iters = 0, w_slots = 0;
    // when every row's edges share one class: [w_iters][12] (alpha, beta) per iteration and layer,
    // for the per-row weighted kernels (ALGO_WROW)
    float2* d_wtab_row = nullptr;
    bool w_row = false;
    // settings of LDPC_ALGO_CIRC runs (default: the circulant engine on silicon)
    ldpc_circ_config circ{LDPC_CIRC_SFPU, LDPC_CIRC_STOP_GENIE, 0.9375f, 0};
    unsigned long long* h_tally = nullptr;  // pinned
    int64_t launches = 0;
    // ldpc_decode_llr: a copy stream and an event that let the decoding of one chunk of frames
    // overlap the host->device copy of the next (created on first use)
    cudaStream_t cstream = nullptr;
    cudaEvent_t cev = nullptr;
    // ldpc_decode_llr_bf16: the caller's bf16 LLRs on the device before they are widened
    uint16_t* d_llr16 = nullptr;
    size_t llr16_cap = 0;
    // pageable caller arrays: a ring of pinned buffers the host fills while earlier pieces copy to the
    // device (created on first use)
    static constexpr int kStageSlots = 3;
    static constexpr size_t kStageBytes = 32u << 20;
    void* stage[kStageSlots] = {};
    cudaEvent_t stage_ev[kStageSlots] = {};
    bool stage_busy[kStageSlots] = {};
    int stage_next = 0;
};

static int detect_qc(ldpc_handle* h) {
    // 12 layers of Z rows; layers 0-3 of degree 3, layers 4-11 of one degree D; each edge of a layer
    // is a circulant: column(j) = blk*Z + ((j + s) mod Z) for every row j of the layer, and the
    // edges of a layer sit in distinct blocks (then the layer's rows share no column).
    if (h->M % QC_LAYERS) return 0;
    const int Z = h->M / QC_LAYERS;
    if (Z < 32 || (Z & (Z - 1)) || h->N % Z || h->P % Z) return 0;
    int D = -1;
    for (int l = 0; l < QC_LAYERS; ++l) {
        const int32_t* r0 = &h->rows[(size_t)(l * Z) * h->dmax];
        int d = 0;
        while (d < h->dmax && r0[d] >= 0) ++d;
        if (l < 4 && d != QC_DEG_LOW) return 0;
        if (l >= 4) {
            if (D < 0) D = d;
            if (d != D) return 0;
        }
        if (d > QC_DMAX) return 0;
        std::vector<int> blks;
        for (int e = 0; e < d; ++e) {
            const int c0 = r0[e];
            const int blk = c0 / Z, s = c0 % Z;
            blks.push_back(blk);
            for (int j = 0; j < Z; ++j) {
                const int32_t* rj = &h->rows[(size_t)(l * Z + j) * h->dmax];
                if (rj[e] != blk * Z + ((j + s) & (Z - 1))) return 0;
            }
            h->blk_off[l][e] = blk * Z;
            h->shift[l][e] = s;
        }
        for (int j = 0; j < Z; ++j) {
            const int32_t* rj = &h->rows[(size_t)(l * Z + j) * h->dmax];
            if (d < h->dmax && rj[d] >= 0) return 0;
        }
        std::sort(blks.begin(), blks.end());
        if (std::adjacent_find(blks.begin(), blks.end()) != blks.end()) return 0;
    }
    h->Z = Z;
    h->D = D;
    // a code whose descriptors some kernels have compiled in (layout 5)
    h->fix = -1;
    for (int i = 0; i < QC_FIXED_COUNT && h->fix < 0; ++i) {
        const QcFixedTable& t = kQcFixedHost[i];
        bool same = t.Z == Z && t.D == D;
        for (int l = 0; l < QC_LAYERS && same; ++l)
            for (int e = 0; e < (l < 4 ? QC_DEG_LOW : D) && same; ++e)
                same = t.blk_off[l][e] == h->blk_off[l][e] && t.shift[l][e] == h->shift[l][e];
        if (same) h->fix = i;
    }
    return 1;
}

static int ensure_cap(void** p, size_t* cap, size_t need) {
    if (*cap >= need) return 0;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(LDPC_ENOMEM, "cudaMalloc of %zu bytes failed", need);
    }
    *cap = need;
    return 0;
}

extern "C" int ldpc_abi_version(void) { return LDPCB200_ABI_VERSION; }

extern "C" int ldpc_last_error(char* buf, size_t len) {
    if (buf && len) {
        strncpy(buf, g_err.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return (int)g_err.size();
}

extern "C" void ldpc_destroy(ldpc_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_tally);
    cudaFree(h->d_work);
    cudaFree(h->d_hist);
    cudaFree(h->d_snr);
    cudaFree(h->d_llr);
    cudaFree(h->d_post);
    cudaFree(h->d_frame_out);
    cudaFree(h->d_rmsg);
    cudaFree(h->d_wtab);
    cudaFree(h->d_wtab_row);
    free_general(&h->gen);
    if (h->h_tally) cudaFreeHost(h->h_tally);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    if (h->cev) cudaEventDestroy(h->cev);
    if (h->cstream) cudaStreamDestroy(h->cstream);
    cudaFree(h->d_llr16);
    for (int i = 0; i < ldpc_handle::kStageSlots; ++i) {
        if (h->stage[i]) cudaFreeHost(h->stage[i]);
        if (h->stage_ev[i]) cudaEventDestroy(h->stage_ev[i]);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" int ldpc_create(const ldpc_matrix* m, int device, ldpc_handle** out) {
    if (!out) return fail(LDPC_EINVAL, "out is NULL");
    *out = nullptr;
    if (!m || !m->rows) return fail(LDPC_EINVAL, "matrix is NULL");
    if (m->n_vars <= 0 || m->n_checks <= 0 || m->max_check_deg <= 0 || m->max_check_deg > 64)
        return fail(LDPC_EINVAL, "bad matrix dimensions N=%d M=%d max_check_deg=%d", m->n_vars,
                    m->n_checks, m->max_check_deg);
    if (m->n_punct < 0 || m->n_punct >= m->n_vars)
        return fail(LDPC_EINVAL, "punctured count %d outside [0, N)", m->n_punct);
    for (int64_t i = 0; i < (int64_t)m->n_checks * m->max_check_deg; ++i) {
        if (m->rows[i] >= m->n_vars || m->rows[i] < -1)
            return fail(LDPC_EINVAL, "edge index out of bounds: row=%lld, col=%d",
                        (long long)(i / m->max_check_deg) + 1, m->rows[i] + 1);
        if (m->rows[i] >= 0 && i % m->max_check_deg > 0 && m->rows[i - 1] < 0)
            return fail(LDPC_EINVAL, "row %lld: edge after the -1 that ends the row",
                        (long long)(i / m->max_check_deg) + 1);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LDPC_ENODEV, "no CUDA device");
    }
    ldpc_handle* h = new (std::nothrow) ldpc_handle();
    if (!h) return fail(LDPC_ENOMEM, "host allocation failed");
    if (device < 0) cudaGetDevice(&device);
    h->device = device;
    h->N = m->n_vars;
    h->M = m->n_checks;
    h->P = m->n_punct;
    h->dmax = m->max_check_deg;
    h->rows.assign(m->rows, m->rows + (size_t)h->M * h->dmax);
    int rc = 0;
    auto bail = [&](int code) { ldpc_destroy(h); return code; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(LDPC_ENODEV, "cudaSetDevice(%d) failed", device));
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail(fail(LDPC_ENODEV, "no device properties"));
    if (prop.major < 10) return bail(fail(LDPC_ENODEV, "device %s (sm_%d%d) is not sm_100", prop.name, prop.major, prop.minor));
    h->n_sm = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)
        return bail(fail(LDPC_EIO, "stream/event creation failed"));
    if (cudaMalloc(&h->d_tally, TALLY_WORDS * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&h->d_work, 64) != cudaSuccess ||
        cudaMallocHost(&h->h_tally, TALLY_WORDS * sizeof(unsigned long long)) != cudaSuccess)
        return bail(fail(LDPC_ENOMEM, "device allocation failed"));
    h->hist_bins = 1024;
    if (cudaMalloc(&h->d_hist, h->hist_bins * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&h->d_snr, 4 * SNR_BINS * sizeof(unsigned long long)) != cudaSuccess)
        return bail(fail(LDPC_ENOMEM, "device allocation failed"));
    if (detect_qc(h) && h->N - h->P > 0 && ((h->N - h->P) % 32) == 0) {
        h->kind = LDPC_KERNEL_QC;
    } else {
        h->kind = LDPC_KERNEL_GENERAL;
        if ((rc = build_general(h->rows.data(), h->N, h->M, h->P, h->dmax, &h->gen, g_err)) != 0)
            return bail(rc);
        h->gen_built = true;
    }
    *out = h;
    return 0;
}

extern "C" int ldpc_row_schedule(const ldpc_matrix* m, int32_t* order, int32_t* starts) {
    if (!m || !m->rows || !order || !starts) return fail(LDPC_EINVAL, "matrix or output is NULL");
    if (m->n_vars <= 0 || m->n_checks <= 0 || m->max_check_deg <= 0 || m->max_check_deg > 64)
        return fail(LDPC_EINVAL, "bad matrix dimensions N=%d M=%d max_check_deg=%d", m->n_vars, m->n_checks,
                    m->max_check_deg);
    for (int64_t i = 0; i < (int64_t)m->n_checks * m->max_check_deg; ++i) {
        if (m->rows[i] >= m->n_vars || m->rows[i] < -1)
            return fail(LDPC_EINVAL, "edge index out of bounds: row=%lld, col=%d",
                        (long long)(i / m->max_check_deg) + 1, m->rows[i] + 1);
        if (m->rows[i] >= 0 && i % m->max_check_deg > 0 && m->rows[i - 1] < 0)
            return fail(LDPC_EINVAL, "row %lld: edge after the -1 that ends the row",
                        (long long)(i / m->max_check_deg) + 1);
    }
    std::vector<int32_t> o, st;
    general_schedule(m->rows, m->n_vars, m->n_checks, m->max_check_deg, o, st);
    std::copy(o.begin(), o.end(), order);
    std::copy(st.begin(), st.end(), starts);
    return (int)st.size() - 1;
}

extern "C" int ldpc_step_schedule(const ldpc_matrix* m, int32_t* order, int32_t* starts, int32_t* low) {
    if (!low) return fail(LDPC_EINVAL, "matrix or output is NULL");
    int rc = ldpc_row_schedule(m, order, starts);  // argument checks (and a scratch use of the outputs)
    if (rc < 0) return rc;
    int maxdeg = 0;
    for (int i = 0; i < m->n_checks; ++i)
        for (int e = 0; e < m->max_check_deg && m->rows[(size_t)i * m->max_check_deg + e] >= 0; ++e)
            maxdeg = std::max(maxdeg, e + 1);
    const int dt = step_dt(maxdeg);
    if (!dt) return fail(LDPC_ENOTSUP, "rows of degree %d: the step kernel takes degrees up to 10", maxdeg);
    std::vector<int32_t> o, st;
    std::vector<uint8_t> lo;
    step_schedule(m->rows, m->n_vars, m->n_checks, m->max_check_deg, dt / 2, o, st, lo);
    std::copy(o.begin(), o.end(), order);
    std::copy(st.begin(), st.end(), starts);
    std::copy(lo.begin(), lo.end(), low);
    return (int)st.size() - 1;
}

extern "C" int ldpc_kernel_kind(const ldpc_handle* h) {
    if (!h) return fail(LDPC_EINVAL, "handle is NULL");
    return h->kind;
}

extern "C" int64_t ldpc_launch_count(const ldpc_handle* h) { return h ? h->launches : -1; }

extern "C" int64_t ldpc_launch_param_bytes(const ldpc_handle* h) {
    if (!h) return fail(LDPC_EINVAL, "handle is NULL");
    return h->kind == LDPC_KERNEL_QC ? (int64_t)sizeof(QcParams) : (int64_t)sizeof(GenParams);
}

static const void* find_shape(const ldpc_handle* h, int storage, int algo, int clip, int ext, int R, int F, int B, int G) {
    if ((G == 5 || G == 6) && h->fix < 0) return nullptr;  // compiled-in descriptors of another code
    return find_qc(QcKey{h->Z, h->D, R, F, storage, algo, clip, ext, B, G});
}

// The default shape of a numerics variant: one row per thread and one frame per CTA with messages in
// registers when that is built, else the first shape built for it (e.g. the global-message kernel of
// a K = 16384 code).
static bool default_shape(const ldpc_handle* h, int storage, int algo, int clip, int ext, int s[4]) {
    if (find_shape(h, storage, algo, clip, ext, 1, 1, 0, 0)) {
        s[0] = 1; s[1] = 1; s[2] = 0; s[3] = 0;
        return true;
    }
    for (const QcTable* t = qc_tables(); t; t = t->next)
        for (int i = 0; i < t->count; ++i) {
            const QcKey& k = t->entries[i].key;
            if (k.Z == h->Z && k.D == h->D && k.mode == storage && k.algo == algo && k.clip == clip && k.ext == ext &&
                ((k.G != 5 && k.G != 6) || h->fix >= 0)) {
                s[0] = k.R; s[1] = k.F; s[2] = k.B; s[3] = k.G;
                return true;
            }
        }
    return false;
}

static bool default_shape_exists(const ldpc_handle* h, int storage, int algo) {
    int s[4];
    return default_shape(h, storage, algo, 0, 0, s);
}

extern "C" int ldpc_set_weights(ldpc_handle* h, const float* alpha, const float* beta, int n_iter, int n_classes,
                                const int32_t* edge_class) {
    if (!h) return fail(LDPC_EINVAL, "handle is NULL");
    if (n_iter == 0) {
        h->w_iters = 0;
        h->w_row = false;
        return 0;
    }
    if (h->kind != LDPC_KERNEL_QC) return fail(LDPC_ENOTSUP, "the weighted decoder needs a QC code");
    if (!alpha || !beta || !edge_class || n_iter < 0 || n_iter > 1000 || n_classes < 1 || n_classes > 127)
        return fail(LDPC_EINVAL, "bad weights (n_iter %d, n_classes %d)", n_iter, n_classes);
    // expand the class table to one (alpha, beta) pair per edge slot and iteration, so the kernel
    // addresses a layer's weights at constant offsets
    const int slots = QC_DEG_LOW * 4 + h->D * 8;
    for (int l = 0; l < QC_LAYERS; ++l)
        for (int e = 0; e < (l < 4 ? QC_DEG_LOW : h->D); ++e) {
            const int32_t c = edge_class[l * QC_DMAX + e];
            if (c < 0 || c >= n_classes) return fail(LDPC_EINVAL, "edge class of layer %d edge %d out of range", l, e);
        }
    const size_t cnt = (size_t)n_iter * slots;
    if (cnt * sizeof(float2) > 64 * 1024)
        return fail(LDPC_EINVAL, "weight table of %d iterations x %d edge slots is above 64 KB", n_iter, slots);
    std::vector<float2> tab(cnt);
    for (int t = 0; t < n_iter; ++t)
        for (int l = 0; l < QC_LAYERS; ++l)
            for (int e = 0; e < (l < 4 ? QC_DEG_LOW : h->D); ++e) {
                const size_t k = (size_t)t * n_classes + edge_class[l * QC_DMAX + e];
                if (!(alpha[k] == alpha[k]) || !(beta[k] == beta[k])) return fail(LDPC_EINVAL, "NaN weight");
                tab[(size_t)t * slots + qc_edge_slot(l, e, h->D)] = make_float2(alpha[k], beta[k]);
            }
    CU(cudaSetDevice(h->device));
    // one class per row (every edge of a layer in the same class): also the per-layer table of the
    // per-row kernels
    bool row_uniform = true;
    for (int l = 0; l < QC_LAYERS; ++l)
        for (int e = 1; e < (l < 4 ? QC_DEG_LOW : h->D); ++e)
            row_uniform = row_uniform && edge_class[l * QC_DMAX + e] == edge_class[l * QC_DMAX];
    std::vector<float2> tab_row;
    if (row_uniform) {
        tab_row.resize((size_t)n_iter * QC_LAYERS);
        for (int t = 0; t < n_iter; ++t)
            for (int l = 0; l < QC_LAYERS; ++l) {
                const size_t k = (size_t)t * n_classes + edge_class[l * QC_DMAX];
                tab_row[(size_t)t * QC_LAYERS + l] = make_float2(alpha[k], beta[k]);
            }
    }
    cudaFree(h->d_wtab);
    cudaFree(h->d_wtab_row);
    h->d_wtab = nullptr;
    h->d_wtab_row = nullptr;
    h->w_iters = 0;
    h->w_row = false;
    CU(cudaMalloc(&h->d_wtab, cnt * sizeof(float2)));
    CU(cudaMemcpy(h->d_wtab, tab.data(), cnt * sizeof(float2), cudaMemcpyHostToDevice));
    if (row_uniform) {
        CU(cudaMalloc(&h->d_wtab_row, tab_row.size() * sizeof(float2)));
        CU(cudaMemcpy(h->d_wtab_row, tab_row.data(), tab_row.size() * sizeof(float2), cudaMemcpyHostToDevice));
    }
    h->w_iters = n_iter;
    h->w_slots = slots;
    h->w_row = row_uniform;
    return 0;
}

extern "C" int ldpc_set_circulant(ldpc_handle* h, const ldpc_circ_config* c) {
    if (!h) return fail(LDPC_EINVAL, "handle is NULL");
    if (!c) return fail(LDPC_EINVAL, "config is NULL");
    if (c->numerics != LDPC_CIRC_SCALAR && c->numerics != LDPC_CIRC_SFPU)
        return fail(LDPC_EINVAL, "unknown circulant numerics %d", c->numerics);
    if (c->stop != LDPC_CIRC_STOP_SYNDROME && c->stop != LDPC_CIRC_STOP_GENIE)
        return fail(LDPC_EINVAL, "unknown circulant stop rule %d", c->stop);
    if (!(c->damping > 0.0f && c->damping <= 1.0f)) return fail(LDPC_EINVAL, "damping must lie in (0, 1]");
    if (c->numerics == LDPC_CIRC_SCALAR && c->damping != 1.0f)
        return fail(LDPC_EINVAL, "the scalar stepper has no damping (damping must be 1)");
    if (c->reserved0 != 0) return fail(LDPC_EINVAL, "reserved0 must be 0");
    h->circ = *c;
    return 0;
}

// Shapes of the general kernels (layouts 3 and 4 of ldpc_set_launch_shape).
static bool general_shape_ok(const ldpc_handle* h, int R, int F, int B, int G) {
    if (G == GEN_LAYOUT_STEP) return R == 1 && F == 1 && B >= 0 && B <= 32 && h->gen.sdt > 0;
    return G == GEN_LAYOUT_WARP && R == 1 && F == GEN_WARPS && B == 0;
}

extern "C" int ldpc_set_launch_shape(ldpc_handle* h, int storage, int R, int F, int B, int G) {
    if (!h) return fail(LDPC_EINVAL, "handle is NULL");
    if (storage < -1 || storage > 2 || R < 0 || F < 0 || B < 0 || G < 0 || G > 7)
        return fail(LDPC_EINVAL, "bad shape storage=%d R=%d F=%d B=%d G=%d", storage, R, F, B, G);
    const int lo = storage < 0 ? 0 : storage, hi = storage < 0 ? 2 : storage;
    const bool reset = R == 0 && F == 0 && B == 0 && G == 0;
    if (h->kind != LDPC_KERNEL_QC) {
        if (!reset && !general_shape_ok(h, R, F, B, G))
            return fail(LDPC_ENOTSUP, "shape R=%d F=%d B=%d G=%d not built for this general matrix", R, F, B, G);
        for (int s = lo; s <= hi; ++s) {
            h->shape[s][0] = R;
            h->shape[s][1] = F;
            h->shape[s][2] = B;
            h->shape[s][3] = G;
        }
        return 0;
    }
    if (G == 3 || G == 4) return fail(LDPC_ENOTSUP, "layouts 3 and 4 are the general kernels'");
    bool any = reset;
    auto built = [&](int s) {
        return find_shape(h, s, LDPC_ALGO_AMIN, 0, 0, R, F, B, G) || find_shape(h, s, LDPC_ALGO_WAMIN, 0, 0, R, F, B, G) ||
               find_shape(h, s, ALGO_WROW, 0, 0, R, F, B, G) ||
               find_shape(h, s, LDPC_ALGO_CIRC, 0, 0, R, F, B, G);
    };
    for (int s = lo; s <= hi; ++s) any |= built(s);
    if (!any)
        return fail(LDPC_ENOTSUP, "shape R=%d F=%d B=%d G=%d not built for Z=%d D=%d", R, F, B, G, h->Z, h->D);
    for (int s = lo; s <= hi; ++s)
        if (reset || built(s)) {
            h->shape[s][0] = R;
            h->shape[s][1] = F;
            h->shape[s][2] = B;
            h->shape[s][3] = G;
        }
    return 0;
}

extern "C" int ldpc_list_shapes_algo(const ldpc_handle* h, int storage, int algo, int32_t* shapes, int max_shapes) {
    if (!h || storage < 0 || storage > 2 || algo < 0 || algo > 3 || (max_shapes > 0 && !shapes))
        return fail(LDPC_EINVAL, "bad arguments");
    int n = 0;
    if (h->kind != LDPC_KERNEL_QC) {
        if (algo != LDPC_ALGO_AMIN && algo != LDPC_ALGO_NMS) return 0;
        // the step kernel at every resident-CTA count worth timing, and the warp kernel
        static const int32_t step_ctas[] = {0, 24, 16};
        int32_t list[4][4];
        if (h->gen.sdt)
            for (int32_t b : step_ctas) {
                list[n][0] = 1; list[n][1] = 1; list[n][2] = b; list[n][3] = GEN_LAYOUT_STEP;
                ++n;
            }
        list[n][0] = 1; list[n][1] = GEN_WARPS; list[n][2] = 0; list[n][3] = GEN_LAYOUT_WARP;
        ++n;
        for (int i = 0; i < n && i < max_shapes; ++i) std::copy(list[i], list[i] + 4, shapes + 4 * i);
        return n;
    }
    // weights with one class per row: the per-row weighted kernels' shapes, where any are built
    if (algo == LDPC_ALGO_WAMIN && h->w_row && default_shape_exists(h, storage, ALGO_WROW)) algo = ALGO_WROW;
    for (const QcTable* t = qc_tables(); t; t = t->next)
        for (int i = 0; i < t->count; ++i) {
            const QcKey& k = t->entries[i].key;
            if (k.Z != h->Z || k.D != h->D || k.mode != storage || k.algo != algo || k.clip || k.ext) continue;
            if ((k.G == 5 || k.G == 6) && h->fix < 0) continue;
            if (n < max_shapes) {
                shapes[4 * n] = k.R;
                shapes[4 * n + 1] = k.F;
                shapes[4 * n + 2] = k.B;
                shapes[4 * n + 3] = k.G;
            }
            ++n;
        }
    return n;
}

extern "C" int ldpc_list_shapes(const ldpc_handle* h, int storage, int32_t* shapes, int max_shapes) {
    return ldpc_list_shapes_algo(h, storage, LDPC_ALGO_AMIN, shapes, max_shapes);
}

static int check_params(const ldpc_handle* h, const ldpc_run_params* p) {
    if (!h) return fail(LDPC_EINVAL, "handle is NULL");
    if (!p) return fail(LDPC_EINVAL, "params are NULL");
    if (p->max_iter < 0 || p->max_iter > 1000000) return fail(LDPC_EINVAL, "max_iter %d out of range", p->max_iter);
    if (p->storage < 0 || p->storage > 2) return fail(LDPC_EINVAL, "unknown storage mode %d", p->storage);
    if (p->algo < 0 || p->algo > 3) return fail(LDPC_EINVAL, "unknown algorithm %d", p->algo);
    if (p->algo == LDPC_ALGO_CIRC) {
        if (h->kind != LDPC_KERNEL_QC || h->D != 6)
            return fail(LDPC_ENOTSUP, "the circulant engine's decoder needs a QC code with rows of degrees 3 and 6");
        if (p->l_max > 0.0f || p->r_max > 0.0f || p->l_post_max > 0.0f)
            return fail(LDPC_ENOTSUP, "the circulant engine's decoder takes no clips");
    }
    if (p->algo == LDPC_ALGO_WAMIN) {
        if (h->kind != LDPC_KERNEL_QC) return fail(LDPC_ENOTSUP, "the weighted decoder needs a QC code");
        if (h->w_iters <= 0) return fail(LDPC_EINVAL, "weighted decoding without weights (ldpc_set_weights)");
        if (p->l_max > 0.0f || p->r_max > 0.0f || p->l_post_max > 0.0f)
            return fail(LDPC_ENOTSUP, "the weighted decoder takes no clips");
    }
    if (!(p->l_max >= 0.0f) || !(p->r_max >= 0.0f) || !(p->l_post_max >= 0.0f))
        return fail(LDPC_EINVAL, "clips must be >= 0");
    if (!(p->sigma >= 0.0f) || p->mu != p->mu) return fail(LDPC_EINVAL, "bad channel mu/sigma");
    if (!(p->ebn0_lo_db > -100.0f && p->ebn0_lo_db < 100.0f) || !(p->ebn0_hi_db > -100.0f && p->ebn0_hi_db < 100.0f))
        return fail(LDPC_EINVAL, "per-frame Eb/N0 range must lie in (-100, 100) dB");
    return 0;
}

// A prepared QC launch: kernel, grid, block, dynamic shared memory and its parameter block.
struct QcLaunch {
    const void* fn = nullptr;
    unsigned grid = 0;
    int block = 0;
    size_t smem = 0;
    QcParams qp;
};

static double code_rate(const ldpc_handle* h) { return (double)(h->N - h->M) / (double)(h->N - h->P); }

// Chooses the QC kernel for these numerics and shape and fills its launch; grid_frac < 1 gives the
// launch that share of the GPU's resident CTA slots (for kernels that run side by side).
static int prepare_qc(ldpc_handle* h, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                      const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be,
                      double grid_frac, QcLaunch* out) {
    const bool clip = p->l_max > 0.0f || p->r_max > 0.0f || p->l_post_max > 0.0f;
    int sh[4];
    // the handle's shape for this storage, else the default shape of the algorithm
    auto lookup = [&](int algo) -> const void* {
        int s[4] = {h->shape[p->storage][0], h->shape[p->storage][1], h->shape[p->storage][2],
                    h->shape[p->storage][3]};
        const void* f = nullptr;
        if (s[0] || s[1] || s[2] || s[3])
            f = find_shape(h, p->storage, algo, clip, ext, s[0] ? s[0] : 1, s[1] ? s[1] : 1, s[2], s[3]);
        if (f) {
            s[0] = s[0] ? s[0] : 1;
            s[1] = s[1] ? s[1] : 1;
        } else if (default_shape(h, p->storage, algo, clip, ext, s)) {
            f = find_shape(h, p->storage, algo, clip, ext, s[0], s[1], s[2], s[3]);
        }
        if (f) std::copy(s, s + 4, sh);
        return f;
    };
    // weights with one class per row run on the per-row weighted kernels where they are built
    const bool wrow = p->algo == LDPC_ALGO_WAMIN && h->w_row && lookup(ALGO_WROW);
    const void* fn = lookup(wrow ? ALGO_WROW : p->algo);
    if (!fn) return LDPC_ENOTSUP;  // the caller falls back to the general kernel
    const int R = sh[0], F = sh[1], G = sh[3];
    QcParams& qp = out->qp;
    memset(&qp, 0, sizeof qp);
    memcpy(qp.blk_off, h->blk_off, sizeof qp.blk_off);
    memcpy(qp.shift, h->shift, sizeof qp.shift);
    qp.n_vars = h->N;
    qp.n_tx = h->N - h->P;
    qp.max_iter = p->max_iter;
    qp.mu = p->mu;
    qp.sigma = p->sigma;
    qp.l_max = p->l_max;
    qp.r_max = p->r_max;
    qp.l_post_max = p->l_post_max;
    qp.seed_lo = (uint32_t)p->seed;
    qp.seed_hi = (uint32_t)(p->seed >> 32);
    qp.stream = p->stream;
    qp.first_frame = first;
    qp.n_frames = n;
    qp.llr_in = d_llr;
    qp.post_out = d_post;
    qp.iters_out = d_it;
    qp.synd_out = d_sf;
    qp.be_out = d_be;
    qp.tally = h->d_tally;
    qp.hist = h->d_hist;
    qp.hist_bins = h->hist_bins;
    qp.work = h->d_work;
    qp.ebn0_lo = p->ebn0_lo_db;
    qp.ebn0_hi = p->ebn0_hi_db;
    qp.rate = (float)code_rate(h);
    qp.snr_bins = h->d_snr;
    if (p->algo == LDPC_ALGO_WAMIN) {
        qp.wtab = wrow ? h->d_wtab_row : h->d_wtab;
        qp.w_iters = h->w_iters;
        qp.w_slots = wrow ? QC_LAYERS : h->w_slots;
    }
    if (p->algo == LDPC_ALGO_CIRC) {
        // the engine's edge order is ascending column: inside a layer every edge has its own column
        // block, so sort the layer's edges by block (the messages follow the same order)
        for (int l = 0; l < QC_LAYERS; ++l) {
            const int d = l < 4 ? QC_DEG_LOW : h->D;
            for (int a = 1; a < d; ++a)
                for (int b = a; b > 0 && qp.blk_off[l][b - 1] > qp.blk_off[l][b]; --b) {
                    std::swap(qp.blk_off[l][b - 1], qp.blk_off[l][b]);
                    std::swap(qp.shift[l][b - 1], qp.shift[l][b]);
                }
        }
        const bool sfpu = h->circ.numerics == LDPC_CIRC_SFPU;
        // the SFPU kernel's constants are bf16 (sFloat16b truncates the fp32 value)
        auto c = [&](float v) {
            uint32_t u;
            memcpy(&u, &v, 4);
            if (sfpu) u &= 0xFFFF0000u;
            memcpy(&v, &u, 4);
            return v;
        };
        qp.circ_c[0] = c(0.69315f);
        qp.circ_c[1] = c(-0.40f);
        qp.circ_c[2] = c(0.65715f);
        qp.circ_c[3] = c(-0.328f);
        qp.circ_damping = h->circ.damping;
        qp.circ_sfpu = sfpu ? 1 : 0;
        qp.stop_rule = h->circ.stop == LDPC_CIRC_STOP_GENIE ? QC_STOP_GENIE : QC_STOP_SYNDROME;
        qp.n_info = h->N - h->M;
    }
    const int T = h->Z / R;
    int32_t off = 0;
    for (int l = 0; l < QC_LAYERS; ++l) {
        qp.layer_off[l] = off;  // the global-message layout keeps edges in pairs: odd degrees padded
        off += h->Z * (((l < 4 ? QC_DEG_LOW : h->D) + 1) & ~1);
    }
    qp.slot_elems = off;
    const size_t esz = p->storage == LDPC_STORE_BF16 ? 2 : 4;
    const size_t lstride = (size_t)((h->N + 7) & ~7);
    // the kernel's layout: L slots, hard-decision words, [16-byte aligned] offset table (G = 2), weights
    size_t smem = (size_t)F * lstride * esz + (size_t)F * (h->N / 32) * 4;
    if (G == 2 || p->algo == LDPC_ALGO_WAMIN) smem = (smem + 15) & ~(size_t)15;
    if (G == 2) smem += (size_t)T * (QC_DEG_LOW * 4 + h->D * 8) * 4;
    if (p->algo == LDPC_ALGO_WAMIN) smem += (size_t)qp.w_iters * qp.w_slots * sizeof(float2);
    if (smem > 48 * 1024) CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, smem));
    if (per_sm <= 0) return fail(LDPC_ENOTSUP, "QC kernel does not fit on an SM (smem %zu)", smem);
    const uint64_t want = (n + F - 1) / F;
    const uint64_t cap = std::max<uint64_t>(1, (uint64_t)((double)per_sm * h->n_sm * std::min(1.0, grid_frac) + 0.5));
    const uint64_t grid = std::min<uint64_t>(want, cap);
    out->fn = fn;
    out->grid = (unsigned)grid;
    out->block = T;
    out->smem = smem;
    if (grid == 0) return 0;
    if (G == 1 || G == 5 || G == 7) {
        int rc;
        const size_t rsz = p->storage == LDPC_STORE_FP32 ? 4 : 2;
        if ((rc = ensure_cap(&h->d_rmsg, &h->rmsg_cap, grid * F * (size_t)qp.slot_elems * rsz))) return rc;
        qp.r_base = h->d_rmsg;
    }
    return 0;
}

static int launch_qc(ldpc_handle* h, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                     const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be) {
    QcLaunch L;
    int rc = prepare_qc(h, p, ext, n, first, d_llr, d_post, d_it, d_sf, d_be, 1.0, &L);
    if (rc || L.grid == 0) return rc;
    void* args[] = {&L.qp};
    CU(cudaLaunchKernel(L.fn, dim3(L.grid), dim3(L.block), args, L.smem, h->stream));
    h->launches++;
    return 0;
}

static int reset_counters(ldpc_handle* h) {
    CU(cudaMemsetAsync(h->d_tally, 0, TALLY_WORDS * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(h->d_work, 0, 64, h->stream));
    CU(cudaMemsetAsync(h->d_hist, 0, h->hist_bins * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(h->d_snr, 0, 4 * SNR_BINS * sizeof(unsigned long long), h->stream));
    return 0;
}

static int read_tally(ldpc_handle* h, ldpc_tally* out) {
    CU(cudaMemcpyAsync(h->h_tally, h->d_tally, TALLY_WORDS * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (out) {
        out->frames = h->h_tally[T_FRAMES];
        out->bit_errors = h->h_tally[T_BIT_ERR];
        out->frame_errors = h->h_tally[T_FRAME_ERR];
        out->iter_sum = h->h_tally[T_ITER_SUM];
        out->unconverged = h->h_tally[T_UNCONVERGED];
        out->max_iters = h->h_tally[T_MAX_ITER];
        out->kernel_ms = ms;
        out->reserved1 = 0.0f;
        out->bit_errors_sq = h->h_tally[T_BIT_ERR_SQ];
    }
    return 0;
}

// Splits a request into launches of at most 2^31 frames (the kernel's claim counter is 32-bit).
static constexpr uint64_t kMaxLaunchFrames = 1ull << 31;

// Channel LLRs in host memory for ldpc_decode_llr / ldpc_decode_llr_bf16.
struct HostLlr {
    const void* src;  // [n][N-P] elements
    int elem;         // 4: fp32; 2: bf16 bit patterns
    bool pageable;    // not page-locked: staged through the pinned ring
};

// bf16 bit patterns -> fp32 (exact): eight values per thread and step when both arrays allow it.
__global__ void widen_bf16_kernel(const uint16_t* __restrict__ in, float* __restrict__ out, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const bool vec = (reinterpret_cast<uintptr_t>(in) % 16 == 0) && (reinterpret_cast<uintptr_t>(out) % 16 == 0);
    uint64_t head = 0;
    if (vec) {
        const uint64_t n8 = n / 8;
        for (uint64_t i = t; i < n8; i += stride) {
            const uint4 v = reinterpret_cast<const uint4*>(in)[i];
            float4 a, b;
            a.x = __uint_as_float(v.x << 16); a.y = __uint_as_float(v.x & 0xFFFF0000u);
            a.z = __uint_as_float(v.y << 16); a.w = __uint_as_float(v.y & 0xFFFF0000u);
            b.x = __uint_as_float(v.z << 16); b.y = __uint_as_float(v.z & 0xFFFF0000u);
            b.z = __uint_as_float(v.w << 16); b.w = __uint_as_float(v.w & 0xFFFF0000u);
            reinterpret_cast<float4*>(out)[2 * i] = a;
            reinterpret_cast<float4*>(out)[2 * i + 1] = b;
        }
        head = n8 * 8;
    }
    for (uint64_t i = head + t; i < n; i += stride) out[i] = __uint_as_float((uint32_t)in[i] << 16);
}

// Host copies on a pool of persistent threads (one per host thread, at most 16): the caller splits a
// copy into equal parts, each worker takes one, the caller takes the first and waits for the rest.
class CopyPool {
  public:
    static CopyPool& get() {
        static CopyPool pool;
        return pool;
    }
    void copy(void* dst, const void* src, size_t bytes) {
        constexpr size_t kMinPart = 1u << 20;
        const size_t nt = std::min<size_t>(workers_.size() + 1, std::max<size_t>(1, bytes / kMinPart));
        if (nt <= 1) {
            memcpy(dst, src, bytes);
            return;
        }
        std::lock_guard<std::mutex> serial(call_mu_);  // one copy at a time (handles on other threads wait)
        const size_t part = (bytes / nt + 63) & ~(size_t)63;
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = static_cast<char*>(dst);
            src_ = static_cast<const char*>(src);
            bytes_ = bytes;
            part_ = part;
            parts_ = nt;
            pending_ = nt - 1;
            ++gen_;
        }
        cv_.notify_all();
        memcpy(dst, src, std::min(bytes, part));
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

  private:
    CopyPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned n = std::min(16u, hw) - 1;
        for (unsigned i = 0; i < n; ++i) workers_.emplace_back([this, i] { run(i + 1); });
    }
    void run(size_t k) {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            if (k >= parts_) continue;  // fewer parts than workers this time
            char* d = dst_;
            const char* s = src_;
            const size_t a = std::min(bytes_, k * part_), b = std::min(bytes_, (k + 1) * part_);
            lk.unlock();
            if (a < b) memcpy(d + a, s + a, b - a);
            lk.lock();
            if (--pending_ == 0) done_cv_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_, call_mu_;
    std::condition_variable cv_, done_cv_;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0, part_ = 0, parts_ = 0, pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

static void par_memcpy(void* dst, const void* src, size_t bytes) { CopyPool::get().copy(dst, src, bytes); }

// Host -> device copy of `bytes` from a pageable array through the pinned ring, on the copy stream:
// each piece waits for its slot's previous copy, is copied into the slot by host threads, then
// copied to the device asynchronously, so the host fills one slot while others travel.
static int stage_h2d(ldpc_handle* h, void* dst, const char* src, size_t bytes) {
    for (int i = 0; i < ldpc_handle::kStageSlots; ++i) {
        if (!h->stage[i] && cudaMallocHost(&h->stage[i], ldpc_handle::kStageBytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(LDPC_ENOMEM, "pinned staging buffer allocation failed");
        }
        if (!h->stage_ev[i] && cudaEventCreateWithFlags(&h->stage_ev[i], cudaEventDisableTiming) != cudaSuccess)
            return fail(LDPC_EIO, "staging event creation failed");
    }
    for (size_t done = 0; done < bytes;) {
        const size_t piece = std::min(ldpc_handle::kStageBytes, bytes - done);
        const int k = h->stage_next;
        h->stage_next = (k + 1) % ldpc_handle::kStageSlots;
        if (h->stage_busy[k]) CU(cudaEventSynchronize(h->stage_ev[k]));
        par_memcpy(h->stage[k], src + done, piece);
        CU(cudaMemcpyAsync(static_cast<char*>(dst) + done, h->stage[k], piece, cudaMemcpyHostToDevice, h->cstream));
        CU(cudaEventRecord(h->stage_ev[k], h->cstream));
        h->stage_busy[k] = true;
        done += piece;
    }
    return 0;
}

// hin (optional): the channel LLRs of the n frames in host memory, copied into d_llr one chunk at a
// time on the handle's copy stream (bf16 through d_llr16 and the widening kernel) while the
// previous chunk decodes; chunk <= kMaxLaunchFrames.
static int run_frames(ldpc_handle* h, const ldpc_run_params* p, bool ext, uint64_t n, const float* d_llr,
                      float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be, const HostLlr* hin = nullptr,
                      uint64_t chunk = kMaxLaunchFrames) {
    int rc;
    if ((rc = reset_counters(h))) return rc;
    if (n == 0) CU(cudaEventRecord(h->ev0, h->stream));
    const uint64_t ntx = (uint64_t)(h->N - h->P);
    for (uint64_t off = 0; off < n; off += chunk) {
        const uint32_t cnt = (uint32_t)std::min<uint64_t>(chunk, n - off);
        if (hin) {
            const size_t bytes = (size_t)cnt * ntx * hin->elem;
            const char* src = static_cast<const char*>(hin->src) + off * ntx * hin->elem;
            void* dst = hin->elem == 4 ? static_cast<void*>(const_cast<float*>(d_llr) + off * ntx)
                                       : static_cast<void*>(h->d_llr16 + off * ntx);
            if (hin->pageable) {
                if ((rc = stage_h2d(h, dst, src, bytes))) return rc;
            } else {
                CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->cstream));
            }
            if (hin->elem == 2) {
                widen_bf16_kernel<<<h->n_sm * 4, 256, 0, h->cstream>>>(h->d_llr16 + off * ntx,
                                                                       const_cast<float*>(d_llr) + off * ntx,
                                                                       (uint64_t)cnt * ntx);
                CU(cudaGetLastError());
            }
            CU(cudaEventRecord(h->cev, h->cstream));
            CU(cudaStreamWaitEvent(h->stream, h->cev, 0));
        }
        if (off == 0) CU(cudaEventRecord(h->ev0, h->stream));
        if (off) CU(cudaMemsetAsync(h->d_work, 0, 64, h->stream));
        const float* llr = d_llr ? d_llr + off * (uint64_t)(h->N - h->P) : nullptr;
        float* post = d_post ? d_post + off * (uint64_t)h->N : nullptr;
        int32_t* it = d_it ? d_it + off : nullptr;
        int32_t* sf = d_sf ? d_sf + off : nullptr;
        int32_t* be = d_be ? d_be + off : nullptr;
        rc = LDPC_ENOTSUP;
        if (h->kind == LDPC_KERNEL_QC) rc = launch_qc(h, p, ext, cnt, p->first_frame + off, llr, post, it, sf, be);
        if (rc == LDPC_ENOTSUP && p->algo == LDPC_ALGO_WAMIN)
            return fail(LDPC_ENOTSUP, "the weighted decoder is not built for Z=%d D=%d with storage %d", h->Z, h->D,
                        p->storage);
        if (rc == LDPC_ENOTSUP && p->algo == LDPC_ALGO_CIRC)
            return fail(LDPC_ENOTSUP, "the circulant engine's decoder is not built for Z=%d with storage %d", h->Z,
                        p->storage);
        if (rc == LDPC_ENOTSUP) {  // no QC variant for these options: the general kernel decodes any matrix
            if (!h->gen_built) {
                if ((rc = build_general(h->rows.data(), h->N, h->M, h->P, h->dmax, &h->gen, g_err)) != 0) return rc;
                h->gen_built = true;
            }
            // the step kernel unless the shape asks for the warp kernel (or the step kernel does not
            // run these numerics / this matrix)
            const int* sh = h->shape[p->storage];
            h->gen.step_ctas = sh[3] == GEN_LAYOUT_STEP ? sh[2] : 0;
            if (sh[3] != GEN_LAYOUT_WARP)
                rc = launch_general_step(&h->gen, p, ext, cnt, p->first_frame + off, llr, post, it, sf, be,
                                         h->d_tally, h->d_hist, h->hist_bins, h->d_work, h->n_sm, h->stream, g_err,
                                         h->d_snr);
            if (rc == LDPC_ENOTSUP)
                rc = launch_general(&h->gen, p, ext, cnt, p->first_frame + off, llr, post, it, sf, be, h->d_tally,
                                    h->d_hist, h->hist_bins, h->d_work, h->n_sm, h->stream, g_err, h->d_snr);
            if (!rc) h->launches++;
        }
        if (rc) return rc;
    }
    CU(cudaEventRecord(h->ev1, h->stream));
    CU(cudaGetLastError());
    return 0;
}

extern "C" int ldpc_run_chunk(ldpc_handle* h, const ldpc_run_params* p, ldpc_tally* out) {
    int rc;
    if ((rc = check_params(h, p))) return rc;
    CU(cudaSetDevice(h->device));
    if ((rc = run_frames(h, p, false, p->n_frames, nullptr, nullptr, nullptr, nullptr, nullptr))) return rc;
    return read_tally(h, out);
}

// ldpc_decode_llr and ldpc_decode_llr_bf16: caller LLRs of `elem` bytes each (4: fp32, 2: bf16).
static int decode_host(ldpc_handle* h, const ldpc_run_params* p, const void* llr, int elem, int64_t n, float* post,
                       int32_t* iters, int32_t* synd_fail, int32_t* bit_errors, ldpc_tally* out) {
    int rc;
    if ((rc = check_params(h, p))) return rc;
    if (n < 0) return fail(LDPC_EINVAL, "n_frames < 0");
    if (n > 0 && !llr) return fail(LDPC_EINVAL, "llr is NULL");
    CU(cudaSetDevice(h->device));
    const size_t ntx = (size_t)(h->N - h->P);
    const size_t nb = (size_t)n;
    if (nb) {
        if ((rc = ensure_cap((void**)&h->d_llr, &h->llr_cap, nb * ntx * sizeof(float)))) return rc;
        if (elem == 2 && (rc = ensure_cap((void**)&h->d_llr16, &h->llr16_cap, nb * ntx * sizeof(uint16_t))))
            return rc;
        if (post && (rc = ensure_cap((void**)&h->d_post, &h->post_cap, nb * h->N * sizeof(float)))) return rc;
        if ((rc = ensure_cap((void**)&h->d_frame_out, &h->frame_cap, 3 * nb * sizeof(int32_t)))) return rc;
    }
    if (!h->cstream && cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(LDPC_EIO, "copy stream creation failed");
    if (!h->cev && cudaEventCreateWithFlags(&h->cev, cudaEventDisableTiming) != cudaSuccess)
        return fail(LDPC_EIO, "copy event creation failed");
    // A page-locked array is copied by DMA straight from the caller's memory; a pageable one through
    // the handle's pinned ring, filled by host threads.
    bool pageable = true;
    if (nb) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, llr) == cudaSuccess)
            pageable = a.type == cudaMemoryTypeUnregistered;
        else
            cudaGetLastError();
    }
    // Large calls copy the LLRs in chunks on the copy stream, so that the decoding of one chunk
    // overlaps the copy of the next; small ones are one chunk.
    constexpr uint64_t kMinChunk = 8192;
    uint64_t chunk = kMaxLaunchFrames;
    if (nb >= 2 * kMinChunk) chunk = std::min<uint64_t>(kMaxLaunchFrames, std::max<uint64_t>(kMinChunk, (nb + 7) / 8));
    const HostLlr hin{llr, elem, pageable};
    ldpc_run_params q = *p;
    q.first_frame = 0;
    q.n_frames = nb;
    int32_t* d_it = h->d_frame_out;
    int32_t* d_sf = d_it ? d_it + nb : nullptr;
    int32_t* d_be = d_sf ? d_sf + nb : nullptr;
    if ((rc = run_frames(h, &q, true, nb, h->d_llr, post ? h->d_post : nullptr, d_it, d_sf, d_be,
                         nb ? &hin : nullptr, chunk)))
        return rc;
    if (nb) {
        if (post) CU(cudaMemcpyAsync(post, h->d_post, nb * h->N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        if (iters) CU(cudaMemcpyAsync(iters, d_it, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
        if (synd_fail) CU(cudaMemcpyAsync(synd_fail, d_sf, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
        if (bit_errors) CU(cudaMemcpyAsync(bit_errors, d_be, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    }
    return read_tally(h, out);
}

extern "C" int ldpc_decode_llr(ldpc_handle* h, const ldpc_run_params* p, const float* llr, int64_t n,
                               float* post, int32_t* iters, int32_t* synd_fail, int32_t* bit_errors,
                               ldpc_tally* out) {
    return decode_host(h, p, llr, 4, n, post, iters, synd_fail, bit_errors, out);
}

extern "C" int ldpc_decode_llr_bf16(ldpc_handle* h, const ldpc_run_params* p, const uint16_t* llr, int64_t n,
                                    float* post, int32_t* iters, int32_t* synd_fail, int32_t* bit_errors,
                                    ldpc_tally* out) {
    return decode_host(h, p, llr, 2, n, post, iters, synd_fail, bit_errors, out);
}

// Channel only: the Philox/Box-Muller LLRs of a range of frames, for checking the generator.
__global__ void channel_kernel(float* out, int ntx, uint64_t first, uint64_t n, uint32_t seed_lo, uint32_t seed_hi,
                               uint32_t stream, float mu0, float sigma0, float lo, float hi, float rate) {
    const int nq = ntx >> 2;
    const uint64_t total = n * (uint64_t)nq;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t f = i / nq;
        const int qd = (int)(i % nq);
        const uint64_t gf = first + f;
        float mu = mu0, sigma = sigma0;
        int bin;
        if (hi > lo) frame_snr(lo, hi, rate, gf, stream, seed_lo, seed_hi, mu, sigma, bin);
        float v[4];
        if (sigma > 0.0f) {
            const U32x4 x = philox4x32_10(U32x4{(uint32_t)qd, (uint32_t)gf, (uint32_t)(gf >> 32), stream}, seed_lo, seed_hi);
            box_muller(x.x, x.y, v[0], v[1]);
            box_muller(x.z, x.w, v[2], v[3]);
            for (int k = 0; k < 4; ++k) v[k] = __fmaf_rn(sigma, v[k], mu);
        } else {
            v[0] = v[1] = v[2] = v[3] = mu;
        }
        reinterpret_cast<float4*>(out + f * ntx)[qd] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

extern "C" int ldpc_channel_llr(ldpc_handle* h, const ldpc_run_params* p, float* llr) {
    int rc;
    if ((rc = check_params(h, p))) return rc;
    if (!llr && p->n_frames) return fail(LDPC_EINVAL, "llr is NULL");
    const int ntx = h->N - h->P;
    if (ntx % 4) return fail(LDPC_ENOTSUP, "channel export needs N-P divisible by 4");
    CU(cudaSetDevice(h->device));
    const size_t bytes = (size_t)p->n_frames * ntx * sizeof(float);
    if (!bytes) return 0;
    if ((rc = ensure_cap((void**)&h->d_llr, &h->llr_cap, bytes))) return rc;
    channel_kernel<<<h->n_sm * 8, 256, 0, h->stream>>>(h->d_llr, ntx, p->first_frame, p->n_frames, (uint32_t)p->seed,
                                                       (uint32_t)(p->seed >> 32), p->stream, p->mu, p->sigma,
                                                       p->ebn0_lo_db, p->ebn0_hi_db, (float)code_rate(h));
    h->launches++;
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(llr, h->d_llr, bytes, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return 0;
}

extern "C" int ldpc_channel_llr_device(ldpc_handle* h, const ldpc_run_params* p, float* d_llr, void* stream) {
    int rc;
    if ((rc = check_params(h, p))) return rc;
    if (!d_llr && p->n_frames) return fail(LDPC_EINVAL, "d_llr is NULL");
    if (!p->n_frames) return 0;
    const int ntx = h->N - h->P;
    if (ntx % 4) return fail(LDPC_ENOTSUP, "channel export needs N-P divisible by 4");
    if (reinterpret_cast<uintptr_t>(d_llr) % 16) return fail(LDPC_EINVAL, "d_llr must be 16-byte aligned");
    CU(cudaSetDevice(h->device));
    channel_kernel<<<h->n_sm * 8, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_llr, ntx, p->first_frame, p->n_frames, (uint32_t)p->seed, (uint32_t)(p->seed >> 32), p->stream, p->mu,
        p->sigma, p->ebn0_lo_db, p->ebn0_hi_db, (float)code_rate(h));
    h->launches++;
    CU(cudaGetLastError());
    return 0;
}

extern "C" int ldpc_decode_llr_static(const ldpc_matrix* h, const ldpc_run_params* p, const float* d_llr,
                                      int64_t n, float* d_post, int32_t* d_iters, int32_t* d_synd_fail,
                                      int32_t* d_bit_errors, ldpc_tally* out, void* stream) {
    return decode_llr_static(h, p, d_llr, n, d_post, d_iters, d_synd_fail, d_bit_errors, out,
                             static_cast<cudaStream_t>(stream), g_err);
}

extern "C" int ldpc_iter_histogram(ldpc_handle* h, uint64_t* hist, int n_bins) {
    if (!h || !hist || n_bins <= 0) return fail(LDPC_EINVAL, "bad arguments");
    CU(cudaSetDevice(h->device));
    std::vector<unsigned long long> tmp(h->hist_bins);
    CU(cudaMemcpyAsync(tmp.data(), h->d_hist, h->hist_bins * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < n_bins; ++i) hist[i] = 0;
    for (int i = 0; i < h->hist_bins; ++i) hist[std::min(i, n_bins - 1)] += tmp[i];
    return 0;
}

extern "C" int ldpc_snr_bins(ldpc_handle* h, uint64_t* out) {
    if (!h || !out) return fail(LDPC_EINVAL, "bad arguments");
    CU(cudaSetDevice(h->device));
    unsigned long long tmp[4 * SNR_BINS];
    CU(cudaMemcpyAsync(tmp, h->d_snr, sizeof tmp, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < 4 * SNR_BINS; ++i) out[i] = tmp[i];
    return 0;
}

// ----------------------------------------------------------------------------- batched launch
// Several codes decoded by one CUDA graph launch: per code, memset nodes for its counters followed by
// its persistent kernel; the codes' kernels have no dependencies on one another and run side by
// side, each on its share of the GPU's CTA slots, each claiming frames from its own queue.  The graph
// is built and instantiated once and relaunched: a call updates its kernel nodes in place
// (cudaGraphExecKernelNodeSetParams: arguments, kernel, grid and shared-memory size may all change),
// and rebuilds the graph only when the set of codes with frames changes (a code's kernel node
// appears or goes) or an update is refused.

struct ldpc_batch {
    int device = 0;
    std::vector<ldpc_handle*> hs;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int64_t launches = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<char> key;                // per code: 1 if it has a kernel node
    std::vector<cudaGraphNode_t> knode;   // per code, its kernel node in `graph`
    int64_t builds = 0;
    int order = LDPC_BATCH_IN_TURN;         // LDPC_BATCH_*: dependencies between the kernel nodes
    int built_order = -1;                   // the order `graph` was built with
};

extern "C" int ldpc_batch_create(ldpc_handle* const* handles, int n, ldpc_batch** out) {
    if (!out || !handles || n <= 0) return fail(LDPC_EINVAL, "bad arguments");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!handles[i]) return fail(LDPC_EINVAL, "handle %d is NULL", i);
        if (handles[i]->device != handles[0]->device) return fail(LDPC_EINVAL, "handles on different devices");
        if (handles[i]->kind != LDPC_KERNEL_QC)
            return fail(LDPC_ENOTSUP, "handle %d does not have the QC structure (batches take QC codes)", i);
    }
    ldpc_batch* b = new (std::nothrow) ldpc_batch();
    if (!b) return fail(LDPC_ENOMEM, "host allocation failed");
    b->device = handles[0]->device;
    b->hs.assign(handles, handles + n);
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
        cudaGetLastError();
        ldpc_batch_destroy(b);
        return fail(LDPC_EIO, "stream/event creation failed");
    }
    *out = b;
    return 0;
}

extern "C" void ldpc_batch_destroy(ldpc_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

extern "C" int64_t ldpc_batch_graph_builds(const ldpc_batch* b) { return b ? b->builds : -1; }

extern "C" int ldpc_batch_set_order(ldpc_batch* b, int order) {
    if (!b) return fail(LDPC_EINVAL, "batch is NULL");
    if (order < LDPC_BATCH_SIDE_BY_SIDE || order > LDPC_BATCH_GLOBAL_IN_TURN)
        return fail(LDPC_EINVAL, "unknown batch order %d", order);
    b->order = order;
    return 0;
}

static int add_memset(cudaGraph_t g, void* dst, size_t bytes, cudaGraphNode_t* node) {
    cudaMemsetParams mp = {};
    mp.dst = dst;
    mp.value = 0;
    mp.elementSize = 4;
    mp.width = bytes / 4;
    mp.height = 1;
    mp.pitch = 0;
    CU(cudaGraphAddMemsetNode(node, g, nullptr, 0, &mp));
    return 0;
}

extern "C" int ldpc_batch_run(ldpc_batch* b, const ldpc_run_params* params, const float* share, ldpc_tally* out,
                              float* graph_ms) {
    if (!b || !params) return fail(LDPC_EINVAL, "bad arguments");
    CU(cudaSetDevice(b->device));
    const int n = (int)b->hs.size();
    double work_total = 0.0;
    std::vector<double> w(n, 0.0);
    for (int i = 0; i < n; ++i) {
        int rc;
        if ((rc = check_params(b->hs[i], &params[i]))) return rc;
        if (params[i].n_frames > kMaxLaunchFrames) return fail(LDPC_EINVAL, "code %d: at most 2^31 frames per batch", i);
        w[i] = share ? (double)share[i] : 1.0;
        if (!(w[i] >= 0.0)) return fail(LDPC_EINVAL, "share %d is negative", i);
        work_total += params[i].n_frames ? w[i] : 0.0;
    }
    // every code's launch first (prepare_qc may grow a code's message scratch, so its arguments
    // change from call to call even when nothing else does)
    std::vector<QcLaunch> Ls(n);
    std::vector<char> key(n, 0);
    int rc = 0;
    int64_t kernels = 0;
    for (int i = 0; i < n; ++i) {
        if (!params[i].n_frames) continue;
        // no shares: every kernel gets its full persistent grid and the block scheduler starts the
        // next code's CTAs as the previous code's retire
        const double frac = (share && work_total > 0.0) ? w[i] / work_total : 1.0;
        rc = prepare_qc(b->hs[i], &params[i], false, (uint32_t)params[i].n_frames, params[i].first_frame, nullptr,
                        nullptr, nullptr, nullptr, nullptr, frac, &Ls[i]);
        if (rc == LDPC_ENOTSUP) return fail(LDPC_ENOTSUP, "code %d: no QC kernel for these options", i);
        if (rc) return rc;
        if (!Ls[i].grid) continue;
        key[i] = 1;
        ++kernels;
    }
    auto kparams = [&](int i, void** args) {
        cudaKernelNodeParams kp = {};
        kp.func = const_cast<void*>(Ls[i].fn);
        kp.gridDim = dim3(Ls[i].grid);
        kp.blockDim = dim3(Ls[i].block);
        kp.sharedMemBytes = (unsigned)Ls[i].smem;
        kp.kernelParams = args;
        return kp;
    };
    // the kernels chained one after another (LDPC_BATCH_IN_TURN: all of them; GLOBAL_IN_TURN: those
    // with a message scratch in global memory); the chain's membership is part of the graph's shape
    for (int i = 0; i < n; ++i)
        if (key[i] && (b->order == LDPC_BATCH_IN_TURN ||
                       (b->order == LDPC_BATCH_GLOBAL_IN_TURN && Ls[i].qp.r_base != nullptr)))
            key[i] = 2;
    bool reuse = b->exec && b->built_order == b->order && b->key.size() == key.size() &&
                 std::equal(key.begin(), key.end(), b->key.begin());
    if (reuse) {
        for (int i = 0; i < n && reuse; ++i) {
            if (!key[i]) continue;
            void* args[] = {&Ls[i].qp};
            const cudaKernelNodeParams kp = kparams(i, args);
            if (cudaGraphExecKernelNodeSetParams(b->exec, b->knode[i], &kp) != cudaSuccess) {
                cudaGetLastError();
                reuse = false;  // rebuild below
            }
        }
    }
    if (!reuse) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->graph) cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
        b->key.clear();
        b->knode.assign(n, nullptr);
        cudaGraph_t g = nullptr;
        CU(cudaGraphCreate(&g, 0));
        b->graph = g;
        cudaGraphNode_t chain = nullptr;  // the last chained kernel node
        for (int i = 0; i < n && !rc; ++i) {
            ldpc_handle* h = b->hs[i];
            cudaGraphNode_t deps[5];
            if ((rc = add_memset(g, h->d_tally, TALLY_WORDS * sizeof(unsigned long long), &deps[0])) ||
                (rc = add_memset(g, h->d_work, 64, &deps[1])) ||
                (rc = add_memset(g, h->d_hist, h->hist_bins * sizeof(unsigned long long), &deps[2])) ||
                (rc = add_memset(g, h->d_snr, 4 * SNR_BINS * sizeof(unsigned long long), &deps[3])))
                break;
            if (!key[i]) continue;
            int nd = 4;
            if (key[i] == 2 && chain) deps[nd++] = chain;
            void* args[] = {&Ls[i].qp};
            const cudaKernelNodeParams kp = kparams(i, args);
            const cudaError_t e = cudaGraphAddKernelNode(&b->knode[i], g, deps, nd, &kp);
            if (e != cudaSuccess) rc = fail(LDPC_EIO, "cudaGraphAddKernelNode: %s", cudaGetErrorString(e));
            if (key[i] == 2) chain = b->knode[i];
        }
        if (!rc) {
            const cudaError_t e = cudaGraphInstantiate(&b->exec, g, 0);
            if (e != cudaSuccess) {
                b->exec = nullptr;
                rc = fail(LDPC_EIO, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
            }
        }
        if (rc) return rc;
        b->key = key;
        b->built_order = b->order;
        ++b->builds;
    }
    {
        cudaError_t e = cudaEventRecord(b->e0, b->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->e1, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) rc = fail(LDPC_EIO, "graph launch: %s", cudaGetErrorString(e));
    }
    if (rc) return rc;
    b->launches += kernels;
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, b->e0, b->e1));
    if (graph_ms) *graph_ms = ms;
    for (int i = 0; i < n; ++i) {
        ldpc_handle* h = b->hs[i];
        h->launches += params[i].n_frames ? 1 : 0;
        unsigned long long t[TALLY_WORDS];
        CU(cudaMemcpy(t, h->d_tally, sizeof t, cudaMemcpyDeviceToHost));
        if (out) {
            out[i].frames = t[T_FRAMES];
            out[i].bit_errors = t[T_BIT_ERR];
            out[i].frame_errors = t[T_FRAME_ERR];
            out[i].iter_sum = t[T_ITER_SUM];
            out[i].unconverged = t[T_UNCONVERGED];
            out[i].max_iters = t[T_MAX_ITER];
            out[i].kernel_ms = ms;
            out[i].reserved1 = 0.0f;
            out[i].bit_errors_sq = t[T_BIT_ERR_SQ];
        }
    }
    return 0;
}

// ----------------------------------------------------------------------------- weighted decoder (training)
struct WLayout {
    size_t ckpt, rwork, stash, gr, total;  // offsets (elements of the real type) and total bytes
};

static int wcheck(const ldpc_handle* h, const ldpc_wdec_config* c, int64_t n, WLayout* lay) {
    if (!h || !c) return fail(LDPC_EINVAL, "handle or config is NULL");
    if (h->kind != LDPC_KERNEL_QC) return fail(LDPC_ENOTSUP, "the weighted decoder needs a QC code");
    const int rb = c->fp64 ? 8 : 4;
    if (!weighted_supported(h->Z, h->D, rb))
        return fail(LDPC_ENOTSUP, "the %s weighted decoder is not built for Z=%d D=%d", c->fp64 ? "double" : "float",
                    h->Z, h->D);
    if (c->n_iter < 1 || c->n_iter > W_MAX_ITER || c->n_classes < 1 || c->n_classes > W_MAX_CLASSES ||
        c->ckpt_every < 1 || c->ckpt_every > c->n_iter || n < 0 || n > (1 << 24))
        return fail(LDPC_EINVAL, "bad weighted-decoder configuration");
    for (int l = 0; l < QC_LAYERS; ++l)
        for (int e = 0; e < (l < 4 ? QC_DEG_LOW : h->D); ++e)
            if (c->edge_class[l][e] < 0 || c->edge_class[l][e] >= c->n_classes)
                return fail(LDPC_EINVAL, "edge class of layer %d edge %d out of range", l, e);
    const size_t E = (size_t)h->Z * (4 * QC_DEG_LOW + 8 * h->D);
    const size_t n_ckpt = (c->n_iter + c->ckpt_every - 1) / c->ckpt_every;
    lay->ckpt = 0;
    lay->rwork = lay->ckpt + n_ckpt * n * (h->N + E);
    lay->stash = lay->rwork + n * E;
    lay->gr = lay->stash + (size_t)n * c->ckpt_every * E;
    lay->total = (lay->gr + n * E) * rb;
    return 0;
}

static void wparams_fill(const ldpc_handle* h, const ldpc_wdec_config* c, int64_t n, WParams* p) {
    memset(p, 0, sizeof *p);
    memcpy(p->blk_off, h->blk_off, sizeof p->blk_off);
    memcpy(p->shift, h->shift, sizeof p->shift);
    memcpy(p->edge_class, c->edge_class, sizeof p->edge_class);
    int32_t off = 0;
    for (int l = 0; l < QC_LAYERS; ++l) {
        p->layer_off[l] = off;
        off += h->Z * (l < 4 ? QC_DEG_LOW : h->D);
    }
    p->n_vars = h->N;
    p->n_tx = h->N - h->P;
    p->n_edges = off;
    p->n_iter = c->n_iter;
    p->n_classes = c->n_classes;
    p->ckpt_every = c->ckpt_every;
    p->post_all = c->post_all ? 1 : 0;
    p->n_frames = (int32_t)n;
}

extern "C" int64_t ldpc_wdec_workspace_bytes(const ldpc_handle* h, const ldpc_wdec_config* c, int64_t n) {
    WLayout lay;
    int rc = wcheck(h, c, n, &lay);
    return rc ? rc : (int64_t)lay.total;
}

extern "C" int ldpc_wdec_forward(ldpc_handle* h, const ldpc_wdec_config* c, const void* d_llr, int64_t n,
                                 const void* d_alpha, const void* d_beta, void* d_post, void* d_ws, void* stream) {
    WLayout lay;
    int rc;
    if ((rc = wcheck(h, c, n, &lay))) return rc;
    if (n && (!d_llr || !d_alpha || !d_beta || !d_post || !d_ws)) return fail(LDPC_EINVAL, "NULL device pointer");
    CU(cudaSetDevice(h->device));
    WParams p;
    wparams_fill(h, c, n, &p);
    char* ws = static_cast<char*>(d_ws);
    const size_t rb = c->fp64 ? 8 : 4;
    p.llr = d_llr;
    p.alpha = d_alpha;
    p.beta = d_beta;
    p.post = d_post;
    p.ckpt = ws + lay.ckpt * rb;
    p.rwork = ws + lay.rwork * rb;
    if ((rc = weighted_forward(p, h->Z, h->D, (int)rb, static_cast<cudaStream_t>(stream), g_err))) return rc;
    h->launches += n ? 1 : 0;
    return 0;
}

extern "C" int ldpc_wdec_backward(ldpc_handle* h, const ldpc_wdec_config* c, int64_t n, const void* d_alpha,
                                  const void* d_beta, const void* d_gpost, void* d_galpha, void* d_gbeta,
                                  void* d_gllr, void* d_ws, void* stream) {
    WLayout lay;
    int rc;
    if ((rc = wcheck(h, c, n, &lay))) return rc;
    if (!d_alpha || !d_beta || !d_galpha || !d_gbeta || (n && (!d_gpost || !d_ws)))
        return fail(LDPC_EINVAL, "NULL device pointer");
    CU(cudaSetDevice(h->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int rb = c->fp64 ? 8 : 4;
    const size_t tc = (size_t)c->n_iter * c->n_classes * rb;
    CU(cudaMemsetAsync(d_galpha, 0, tc, s));
    CU(cudaMemsetAsync(d_gbeta, 0, tc, s));
    WParams p;
    wparams_fill(h, c, n, &p);
    char* ws = static_cast<char*>(d_ws);
    p.alpha = d_alpha;
    p.beta = d_beta;
    p.ckpt = ws + lay.ckpt * rb;
    p.rwork = ws + lay.rwork * rb;
    p.stash = ws + lay.stash * rb;
    p.gr = ws + lay.gr * rb;
    p.gpost = d_gpost;
    p.galpha = d_galpha;
    p.gbeta = d_gbeta;
    p.gllr = d_gllr;
    if ((rc = weighted_backward(p, h->Z, h->D, rb, s, g_err))) return rc;
    h->launches += n ? 1 : 0;
    return 0;
}
