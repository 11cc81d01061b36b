/*
 * libldpcb200 — C ABI of the B200 AR4JA LDPC Monte Carlo engine.
 *
 * The reference runs its Monte Carlo hot path (channel -> layered Approximate-Min* decoding ->
 * error tallies) inside one C++ function, run_ldpc_worker
 * (engines/scalar_5w/ldpc_decoder_core.h:214-232), which its host harness drives one batch at a
 * time (engines/scalar_5w/ldpc_sim_scalar.cpp:421-632) after parsing the parity-check matrix
 * (ldpc_sim_scalar.cpp:116-269).  This header is the boundary that replaces that pair: a handle
 * made from a parity-check matrix, a call that simulates one chunk of frames and returns the tallies
 * the harness sums, and a call that decodes caller-supplied channel LLRs (the path of the
 * reference's CPU steppers, tests/test_circulant_dma_stepper.cpp:861-990).
 *
 * Conventions: plain C types only; every function returns 0 on success or a negative errno-style
 * code (LDPC_E*), never aborts, and leaves a message for ldpc_last_error() (per calling thread).
 * The caller owns host buffers; the library owns device memory.  A handle is used by one thread at a
 * time and issues its work on its own CUDA stream.
 */
#ifndef LDPCB200_H
#define LDPCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDPCB200_ABI_VERSION 1

/* Error codes (negative errno values). */
#define LDPC_OK 0
#define LDPC_EINVAL (-22)  /* bad argument */
#define LDPC_ENOMEM (-12)  /* device or host allocation failed */
#define LDPC_ENODEV (-19)  /* no usable CUDA device / kernel image */
#define LDPC_ENOTSUP (-95) /* combination not built (e.g. a storage mode for a code shape) */
#define LDPC_EIO (-5)      /* a CUDA call failed; see ldpc_last_error() */

/* Message storage (engines/scalar_5w/ldpc_decoder_core.h:84-90, 476-520). */
#define LDPC_STORE_BF16 0 /* L and r rounded to bf16 after every update: the reference numerics */
#define LDPC_STORE_FP32 1 /* L and r in fp32 */
#define LDPC_STORE_FP16 2 /* L in fp32, r rounded to IEEE fp16 */

/* Check-node rule (ldpc_decoder_core.h:320-475; the reference's -n flag selects NMS). */
#define LDPC_ALGO_AMIN 0 /* Approximate-Min* (Jones, MILCOM 2003) */
#define LDPC_ALGO_NMS 1  /* normalised min-sum, alpha = 0.75 */
#define LDPC_ALGO_WAMIN 2 /* weighted Approximate-Min* with the handle's weights (ldpc_set_weights) */
#define LDPC_ALGO_CIRC 3  /* the circulant engine's decoder with the handle's settings (ldpc_set_circulant) */

/* Decoder family chosen for a matrix (ldpc_kernel_kind). */
#define LDPC_KERNEL_QC 0      /* quasi-cyclic layered kernel (AR4JA structure detected) */
#define LDPC_KERNEL_GENERAL 1 /* any matrix, file order kept where rows share a variable (ldpc_row_schedule) */

typedef struct ldpc_handle ldpc_handle;

/* A parity-check matrix: replaces the reference's ChinnMatrix (ldpc_sim_scalar.cpp:108-114).
 * rows[m * max_check_deg + d] is the 0-based column of edge d of check m, in the order the matrix
 * file lists it, -1 after the row's last edge (an edge after a -1 is rejected with LDPC_EINVAL).  The
 * last n_punct columns are punctured. */
typedef struct {
    int32_t n_vars;        /* N */
    int32_t n_checks;      /* M (checks) */
    int32_t n_punct;       /* P */
    int32_t max_check_deg; /* row stride of rows */
    const int32_t* rows;   /* [n_checks][max_check_deg] */
} ldpc_matrix;

/* One chunk of simulation: replaces run_ldpc_worker's arguments (ldpc_decoder_core.h:214-232)
 * and the per-batch runtime arguments of ldpc_sim_scalar.cpp:501-523.  Frame f of the chunk is
 * global frame first_frame + f; its channel depends only on (seed, stream, global frame index). */
typedef struct {
    float mu;           /* channel LLR mean,  4 R Eb/N0       (ldpc_sim_scalar.cpp:351-355) */
    float sigma;        /* channel LLR sigma, sqrt(8 R Eb/N0); 0 = noiseless (LLR = mu) */
    uint64_t seed;      /* Philox key */
    uint32_t stream;    /* Philox counter word 3: independent streams for one seed */
    uint32_t reserved0;
    uint64_t first_frame;
    uint64_t n_frames;  /* frames in this chunk, >= 0 */
    int32_t max_iter;   /* >= 0 */
    int32_t storage;    /* LDPC_STORE_* */
    int32_t algo;       /* LDPC_ALGO_* */
    float l_max;        /* channel LLR clip (-L / -G), 0 = off  (ldpc_decoder_core.h:266-275) */
    float r_max;        /* check message clip (-R), 0 = off      (:487) */
    float l_post_max;   /* posterior clip (-V), 0 = off          (:492-495) */
    float ebn0_lo_db;   /* per-frame Eb/N0: when ebn0_hi_db > ebn0_lo_db every frame draws its Eb/N0 */
    float ebn0_hi_db;   /* uniformly in [lo, hi) from its own counter, and mu/sigma are ignored */
} ldpc_run_params;

/* Bins of the per-frame Eb/N0 range (ldpc_snr_bins). */
#define LDPC_SNR_BINS 32

/* Tallies of one call: the per-worker stats of run_ldpc_worker (ldpc_decoder_core.h:580-585)
 * summed over all frames of the chunk. */
typedef struct {
    uint64_t frames;
    uint64_t bit_errors;   /* sign bits set over the first N-P positions, summed */
    uint64_t frame_errors; /* frames with at least one such bit */
    uint64_t iter_sum;     /* executed iterations, including the one that met the syndrome */
    uint64_t unconverged;  /* frames whose syndrome still fails after decoding */
    uint64_t max_iters;    /* largest iteration count of one frame */
    float kernel_ms;       /* device time of the decode kernel (CUDA events on the handle's stream;
                              for a large ldpc_decode_llr, from the first launch to the end of the
                              last, waits for later chunks' LLR copies included) */
    float reserved1;
    uint64_t bit_errors_sq; /* sum over frames of (bit errors of the frame)^2: the frame-level variance
                               of the bit-error count, for confidence intervals on BER */
} ldpc_tally;

/* Replaces parse_chinn + the device setup of ldpc_sim_scalar.cpp:204-269, 319-392.  Copies the
 * matrix; detects the quasi-cyclic AR4JA layer structure (12 layers of Z rows, degrees 3 and D)
 * and selects the layered QC kernel, otherwise the general kernel.  device < 0 = current. */
int ldpc_create(const ldpc_matrix* h, int device, ldpc_handle** out);

/* Releases the handle and its device memory. */
void ldpc_destroy(ldpc_handle* h);

/* LDPC_KERNEL_QC or LDPC_KERNEL_GENERAL, or a negative error. */
int ldpc_kernel_kind(const ldpc_handle* h);

/* The row schedule the general kernel runs a matrix with (host only, needs no GPU).  The reference
 * updates the rows one after another in file order (ldpc_decoder_core.h:314-522); rows that share no
 * variable commute bit for bit, so the kernel runs the rows in steps of at most 32 rows sharing no
 * variable, with every pair of rows that share one in file order: rows sorted by their earliest level
 * (1 + the highest level among the earlier rows they share a variable with; file order inside a
 * level), cut greedily into steps.  Writes the file rows in schedule order to order[M] and the first
 * position of every step followed by M to starts[M + 1]; returns the number of steps, or a negative
 * error for a bad matrix. */
int ldpc_row_schedule(const ldpc_matrix* h, int32_t* order, int32_t* starts);

/* The schedule the step kernel (the general kernel for rows of degree at most 10, the one the shipped
 * matrix file runs on) uses instead (host only, needs no GPU).  The same rule keeps the file order of
 * every pair of rows sharing a variable, but each step takes rows of one degree class: low (degree
 * at most half the kernel's degree bound: 3 for files of degree up to 6) or high, so that a low step
 * runs the kernel's short row body.  Steps are filled by list scheduling, the rows with the longest
 * chain of dependants first.  Writes order[M], starts[M + 1] (as ldpc_row_schedule) and low[M]
 * (1 for a low step, one entry per step); returns the number of steps, or a negative error. */
int ldpc_step_schedule(const ldpc_matrix* h, int32_t* order, int32_t* starts, int32_t* low);

/* Simulates p->n_frames frames (channel generation, decoding, tallies) on the device; replaces one
 * batch of ldpc_sim_scalar.cpp:421-589 (EnqueueMeshWorkload + ReadShard + host sums).  Blocks until
 * the tallies are on the host. */
int ldpc_run_chunk(ldpc_handle* h, const ldpc_run_params* p, ldpc_tally* out);

/* Decodes n_frames caller-supplied frames: llr [n_frames][N-P] fp32 channel LLRs (host; pinned
 * memory copies fastest, and from 16384 frames on the copy of each chunk of frames overlaps the
 * decoding of the previous one).  Uses
 * p->max_iter, storage, algo and the clips (mu/sigma/seed ignored).  Outputs (each may be NULL):
 * post [n_frames][N] final L as stored (bf16/fp16 values widened to float), iters, synd_fail (rows
 * failing after decoding), bit_errors. */
int ldpc_decode_llr(ldpc_handle* h, const ldpc_run_params* p, const float* llr, int64_t n_frames,
                    float* post, int32_t* iters, int32_t* synd_fail, int32_t* bit_errors,
                    ldpc_tally* out);

/* As ldpc_decode_llr with the channel LLRs as bf16 values (the bit patterns, uint16 each), the form in
 * which the reference's decoder holds its channel LLRs (ldpc_decoder_core.h:262-283): half the
 * host->device bytes.  The values are widened to fp32 exactly on the device, so the results equal
 * ldpc_decode_llr on the same values given as fp32.  A pageable array (either entry point) is
 * staged through a ring of page-locked buffers that host threads fill while earlier pieces copy. */
int ldpc_decode_llr_bf16(ldpc_handle* h, const ldpc_run_params* p, const uint16_t* llr, int64_t n_frames,
                         float* post, int32_t* iters, int32_t* synd_fail, int32_t* bit_errors,
                         ldpc_tally* out);

/* Writes the channel LLRs the simulation would decode for frames first_frame .. +n_frames-1
 * (before storage rounding): llr [n_frames][N-P] (host).  For checking the channel. */
int ldpc_channel_llr(ldpc_handle* h, const ldpc_run_params* p, float* llr);

/* As ldpc_channel_llr into a caller-owned device array d_llr [n_frames][N-P] (16-byte aligned),
 * queued on the stream (NULL: the legacy default stream) without waiting: training frames for the
 * weighted decoder come from the simulator's own channel.  No counterpart in the reference. */
int ldpc_channel_llr_device(ldpc_handle* h, const ldpc_run_params* p, float* d_llr, void* stream);

/* Iteration histogram of the last ldpc_run_chunk / ldpc_decode_llr: hist[i] = frames that used i
 * iterations (the last bin also counts every larger value). */
int ldpc_iter_histogram(ldpc_handle* h, uint64_t* hist, int n_bins);

/* Per-Eb/N0 tallies of the last ldpc_run_chunk with a per-frame Eb/N0 range: out[k * LDPC_SNR_BINS + b]
 * for k = frames, frame errors, bit errors, iterations, and bin b of [lo, hi) in LDPC_SNR_BINS equal
 * steps. */
int ldpc_snr_bins(ldpc_handle* h, uint64_t* out);

/* Launch shape of the QC kernel's simulation path for one storage mode (-1 = all): rows per thread,
 * frames per CTA, the resident CTAs per SM its register allocation must allow (a register cap;
 * 0 = the compiler's choice), and the layout (global_messages): 0 = check messages in registers,
 * 1 = in global memory (codes too large for the register file), 2 = in registers, with each
 * thread's column offsets precomputed in shared memory, 5 = as 1 with the code's layer descriptors
 * compiled into the kernel (built for the K = 16384 AR4JA codes and the rate-4/5 codes at K = 1024
 * and 4096, in makeH order, offered only when the matrix's descriptors are exactly those), 6 = as 0
 * with the descriptors compiled in (rates 1/2 and 2/3 at K = 1024 and 4096), 7 = as 1 with the
 * degree-D layers in a loop that is not unrolled, its descriptors read by layer index (rate 4/5 at
 * K = 1024 and 4096, rate 2/3 at K = 1024: any matrix of that shape); layouts 3 and 4 are the
 * general kernels'.
 * All zero restores the default.
 * LDPC_ENOTSUP if the shape is not built for this code.  Used by the autotuner
 * (ldpcb200.capi.Decoder.autotune).  Options with no QC variant built (e.g. clips on a K = 16384
 * code) run on the general kernel. */
int ldpc_set_launch_shape(ldpc_handle* h, int storage, int rows_per_thread, int frames_per_cta,
                          int min_ctas_per_sm, int global_messages);

/* The QC shapes built for this code and storage mode: writes up to max_shapes quadruples
 * (rows per thread, frames per CTA, min CTAs per SM, layout) and returns how many exist. */
int ldpc_list_shapes(const ldpc_handle* h, int storage, int32_t* shapes, int max_shapes);

/* As ldpc_list_shapes for the simulation variants of one algorithm (LDPC_ALGO_*). */
int ldpc_list_shapes_algo(const ldpc_handle* h, int storage, int algo, int32_t* shapes, int max_shapes);

/* Number of kernel launches the handle issued since creation (for launch accounting). */
int64_t ldpc_launch_count(const ldpc_handle* h);

/* Bytes of the kernel argument block one decode launch copies to the device (the only host-to-
 * device traffic of ldpc_run_chunk besides the launch itself). */
int64_t ldpc_launch_param_bytes(const ldpc_handle* h);

/* Size of the device scratch ldpc_decode_llr_static works in (16 MiB per GPU). */
#define LDPC_STATIC_SCRATCH_BYTES (16u << 20)

/* Decoding without any allocation.  No counterpart in the reference (its workers decode in buffers
 * the host set up once).  For callers that must not let a library allocate device memory: an
 * application that reserves all of a GPU's memory up front for its own pool, or one whose device
 * footprint has to be fixed and known before it runs.  Decodes n_frames frames of the matrix h from
 * d_llr [n_frames][N-P] fp32 (device memory) into device buffers d_post [n_frames][N], d_iters,
 * d_synd_fail, d_bit_errors (each may be NULL), on `stream` (a cudaStream_t; NULL = the legacy
 * default stream), and returns the tallies in *out.  Same decoder and results as ldpc_decode_llr
 * (the general file-order kernel); no cudaMalloc, cudaFree or host allocation.
 *
 * Its scratch (code tables, check messages, claim counter, tallies) is one static device array of
 * LDPC_STATIC_SCRATCH_BYTES that every GPU loading the library holds until exit.  A matrix needing
 * more than that for one CTA of frame slots (4 slots, or 1 when a frame's posteriors are too large
 * for 4 to share a CTA, as in ldpc_decode_llr) is rejected with LDPC_ENOMEM; smaller ones run with as
 * many frame slots as fit.  Any n_frames >= 0 is accepted (decoded in launches of at most 2^31
 * frames).  The first call on a device looks the array up on that device.  Every call reuses the
 * same array: calls whose work can overlap on the
 * GPU race and must be serialised by the caller.  Each call synchronises `stream` before it returns,
 * so the outputs are ready when it does. */
int ldpc_decode_llr_static(const ldpc_matrix* h, const ldpc_run_params* p, const float* d_llr,
                           int64_t n_frames, float* d_post, int32_t* d_iters, int32_t* d_synd_fail,
                           int32_t* d_bit_errors, ldpc_tally* out, void* stream);

/* Weights of the weighted Approximate-Min* decoder for LDPC_ALGO_WAMIN runs of this handle (host
 * arrays, copied): alpha/beta [n_iter][n_classes] (iteration t >= n_iter uses row n_iter - 1) and
 * edge_class [12][18], the class of edge e of layer l.  The check-node output becomes
 * sign * max(alpha[t][c] * m - beta[t][c], 0) in the simulation kernels (with syndrome stop and
 * tallies, like every other algorithm).  The table is expanded to one pair per iteration and edge of a
 * row-layer set, n_iter x (12 + 8 D) x 8 bytes, at most 64 KB (n_iter <= 52 for D = 18).
 * n_iter = 0 removes the weights.  QC codes only; no clips.  No counterpart in the reference. */
int ldpc_set_weights(ldpc_handle* h, const float* alpha, const float* beta, int n_iter, int n_classes,
                     const int32_t* edge_class);

/* The circulant engine's decoder for LDPC_ALGO_CIRC runs of this handle: the check-node arithmetic
 * of engines/circulant_dma_4cw/compute_trisc.cpp:299-658 as its golden stepper states it
 * (tests/test_circulant_dma_stepper.cpp:39-565, run_monte_carlo :708-822).  Replaces the
 * per-invocation settings of ldpc_sim_circulant_dma.cpp:526-572 and of the stepper's command line.
 *   - rows of degree 3 and 6 only (the rate-1/2 AR4JA codes), degree-6 layers first (the engine's
 *     tile schedule: rows 512..1535, then 0..511, for K = 1024), edges in ascending column order;
 *   - degree-6 magnitudes from the pairwise min* tree (pairs (0,3), (1,4), (2,5)), degree 3 from the
 *     other two edges; min* g = max(min - max(c1 - 0.4 d, c2 - 0.328 d, 0), 0), c1 = 0.69315,
 *     c2 = 0.65715 (not the scalar engine's piecewise form);
 *   - numerics LDPC_CIRC_SFPU: the SFPU kernel (constants truncated to bf16, q = L - r rounded to the
 *     storage, magnitudes times damping, L = store(q + store(r)));  LDPC_CIRC_SCALAR: the stepper's
 *     scalar path (exact constants, q unrounded, L = store(q + r)), damping must be 1;
 *   - stop LDPC_CIRC_STOP_SYNDROME: the stepper (full syndrome after every iteration; a frame that
 *     never meets it is a frame error, with bit errors = info positions holding a value <= 0);
 *     LDPC_CIRC_STOP_GENIE: the engine on silicon (stop once no info position has its sign bit set;
 *     bit errors = info sign bits of a frame that never stopped, reader_brisc.cpp:166-198,
 *     writer_ncrisc.cpp:265-337).  Info positions are the first N - M columns.
 * Tallies and per-frame outputs of LDPC_ALGO_CIRC runs follow that engine (ldpc_tally.bit_errors
 * then counts info positions).  The defaults (before any call) are the silicon engine: SFPU,
 * damping 0.9375, genie stop.  LDPC_ENOTSUP for codes whose rows are not of degrees 3 and 6. */
#define LDPC_CIRC_SCALAR 0
#define LDPC_CIRC_SFPU 1
#define LDPC_CIRC_STOP_SYNDROME 0
#define LDPC_CIRC_STOP_GENIE 1
typedef struct {
    int32_t numerics;  /* LDPC_CIRC_SFPU or LDPC_CIRC_SCALAR */
    int32_t stop;      /* LDPC_CIRC_STOP_SYNDROME or LDPC_CIRC_STOP_GENIE */
    float damping;     /* in (0, 1]; the engine's beta = 15/16 */
    int32_t reserved0; /* 0 */
} ldpc_circ_config;
int ldpc_set_circulant(ldpc_handle* h, const ldpc_circ_config* c);

/* ---- Weighted Approximate-Min* decoder (training path; no counterpart in the reference) ----
 * Layered decoding of the handle's QC code for exactly n_iter iterations (no early stop) with
 * r_e = sign_e * relu(alpha[t][c] * m_e - beta[t][c]): m_e the Approximate-Min* magnitude of edge e,
 * t the iteration, c = edge_class[l][e] the protograph edge class of edge e of layer l.  The real
 * type is float (fp64 = 0; alpha = 1, beta = 0 then reproduces the plain fp32 decoder bit for bit)
 * or double (fp64 = 1, for checking the adjoint against finite differences; rate 1/2 and 4/5 at
 * K = 1024 only): every array argument below is of that type.  All pointers are device memory owned
 * by the caller; the workspace holds the activation checkpoints between the forward and the
 * backward call of the same frames.  Work is queued on the stream; the calls do not wait for it. */
typedef struct {
    int32_t n_iter;              /* T, 1..64 */
    int32_t n_classes;           /* C, 1..64 */
    int32_t ckpt_every;          /* iterations between activation checkpoints, 1..T */
    int32_t post_all;            /* 1: posteriors after every iteration [T][n][N]; 0: after the last [1][n][N] */
    int32_t fp64;                /* 0: float arrays; 1: double arrays */
    int32_t reserved0;
    int32_t edge_class[12][18];  /* class of edge e of layer l */
} ldpc_wdec_config;

int64_t ldpc_wdec_workspace_bytes(const ldpc_handle* h, const ldpc_wdec_config* c, int64_t n_frames);

/* d_llr [n][N-P] channel LLRs, d_alpha/d_beta [T][C] -> d_post (see post_all). */
int ldpc_wdec_forward(ldpc_handle* h, const ldpc_wdec_config* c, const void* d_llr, int64_t n_frames,
                      const void* d_alpha, const void* d_beta, void* d_post, void* d_workspace, void* stream);

/* Adjoint of the last forward with this workspace: d_grad_post (shaped like d_post) in; gradients
 * of alpha and beta ([T][C], overwritten) and of the channel LLRs ([n][N-P], may be NULL) out. */
int ldpc_wdec_backward(ldpc_handle* h, const ldpc_wdec_config* c, int64_t n_frames, const void* d_alpha,
                       const void* d_beta, const void* d_grad_post, void* d_grad_alpha, void* d_grad_beta,
                       void* d_grad_llr, void* d_workspace, void* stream);

/* A batch of codes on one device decoded by one CUDA graph launch (the mixed-code workload).  The
 * reference runs one code per process (run_simulation.py:164-193); this has no counterpart there.
 * Every handle must have the QC structure. */
typedef struct ldpc_batch ldpc_batch;
int ldpc_batch_create(ldpc_handle* const* handles, int n_handles, ldpc_batch** out);
void ldpc_batch_destroy(ldpc_batch* b);

/* One graph launch: per handle i, params[i] (n_frames may be 0; at most 2^31) decoded by its
 * persistent kernel, in the order ldpc_batch_set_order chose.  With share NULL each kernel gets its
 * full persistent grid (kernels without a dependency between them: the hardware block scheduler
 * starts a code's CTAs as the CTAs launched before it retire); otherwise kernel i is limited to the
 * fraction share[i] / sum(share) of the GPU's CTA slots.
 * out[i] receives handle i's tallies (kernel_ms = the whole graph's device time), *graph_ms the
 * device time of the launch.  ldpc_snr_bins(handle i) then gives its per-Eb/N0 tallies. */
int ldpc_batch_run(ldpc_batch* b, const ldpc_run_params* params, const float* share, ldpc_tally* out,
                   float* graph_ms);

/* Order of the batch's kernels inside its graph:
 *   LDPC_BATCH_SIDE_BY_SIDE  no dependencies between the kernels (the block scheduler interleaves
 *                            their CTAs as resources free up);
 *   LDPC_BATCH_IN_TURN       each code's kernel starts when the previous code's has finished, so every
 *                            kernel has the GPU (and its L2) to itself;
 *   LDPC_BATCH_GLOBAL_IN_TURN  the kernels that keep their check messages in global memory (the
 *                            K = 16384 codes and the register-capped degree-18 shapes, whose message
 *                            scratch lives in L2) run in turn, the others side by side with them.
 * A change of order rebuilds the graph at the next ldpc_batch_run.  Default: LDPC_BATCH_IN_TURN (on the
 * nine-code workload it equals the sum of each code's kernel run alone, and is the steadiest). */
#define LDPC_BATCH_SIDE_BY_SIDE 0
#define LDPC_BATCH_IN_TURN 1
#define LDPC_BATCH_GLOBAL_IN_TURN 2
int ldpc_batch_set_order(ldpc_batch* b, int order);

/* How many times the batch built and instantiated its CUDA graph.  The graph is built by the first
 * ldpc_batch_run and relaunched by later ones with its kernel nodes updated in place (arguments,
 * kernel, grid, shared memory: other frame counts, storage modes, shapes or shares); a call that
 * changes which codes have frames rebuilds it. */
int64_t ldpc_batch_graph_builds(const ldpc_batch* b);

/* Copies the last error message of the calling thread into buf (NUL-terminated); returns its
 * length. */
int ldpc_last_error(char* buf, size_t len);

/* LDPCB200_ABI_VERSION */
int ldpc_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LDPCB200_H */
