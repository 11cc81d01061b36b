// Decoder for an arbitrary parity-check matrix with the reference's serial row order.
//
// The reference updates rows one after another in file order (engines/scalar_5w/ldpc_decoder_core.h:
// 314-522).  The host reorders the rows into steps of at most 32 rows that share no variable, keeping
// every pair of rows that share one in file order (general_schedule in general.cu); rows of one step
// are independent, so updating them at once gives the serial result bit for bit.  One warp owns one
// frame: lanes take the rows of a step, __syncwarp between steps.  L lives in shared memory; the
// messages r of a slot live in a global-memory scratch area laid out [position in the schedule][edge],
// so a lane reads and writes its row's messages with a few vector accesses and a step's rows are
// contiguous (the area of all resident slots stays mostly in L2).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ldpcb200.h"
#include "ldpc_device.cuh"

namespace ldpcb200 {

constexpr int GEN_WARPS = 4;  // frame slots (warps) per CTA

// Kernels for a general matrix: the step kernel (general_step.cu) when the matrix's degree allows
// it and the numerics are ones it runs, else the warp kernel (general.cu).
// Layout numbers of the two kernels in ldpc_set_launch_shape (0-2 are the QC kernel's layouts).
enum GenLayout : int { GEN_LAYOUT_STEP = 3, GEN_LAYOUT_WARP = 4 };

struct GeneralCode {
    int N = 0, M = 0, P = 0, dmax = 0, n_runs = 0, dt = 0;  // dt: compiled degree bound
    int32_t* d_cols = nullptr;  // [M][gen_dtc(dt)] columns of the row at schedule position k (-1 pad)
    int32_t* d_runs = nullptr;  // [n_runs + 1] first position of each step, then M
    void* d_r = nullptr;        // message scratch of either kernel (one slot per resident frame)
    size_t r_cap = 0;
    // step kernel: the same steps, each padded to 32 rows (lane j takes row j of the step); a lane
    // without a row and an edge past its row's degree point at the dummy posterior slot N
    int sdt = 0;                          // its degree bound (0: the matrix needs the warp kernel)
    int32_t* d_scols[2] = {nullptr, nullptr};  // byte offsets for 2- and 4-byte posteriors, step_table layout
    int32_t* d_slot[2] = {nullptr, nullptr};   // [N] the shared-memory slot of each variable, per element size
    int s_steps = 0;                      // steps of the step kernel's own schedule (step_schedule)
    int32_t* d_slow = nullptr;            // [s_steps] 1: every row of the step has degree <= sdt / 2
    int step_ctas = 0;                    // step kernel CTAs per SM (0: as many as fit)
};

struct GenParams {
    const int32_t* cols;
    const int32_t* runs;
    int32_t n_runs, N, M, n_tx, dmax, max_iter;
    float mu, sigma, l_max, r_max, l_post_max;
    uint32_t seed_lo, seed_hi, stream;
    uint64_t first_frame;
    uint32_t n_frames;
    void* r_base;
    const float* llr_in;
    float* post_out;
    int32_t* iters_out;
    int32_t* synd_out;
    int32_t* be_out;
    unsigned long long* tally;
    unsigned long long* hist;
    int32_t hist_bins;
    unsigned int* work;
    float ebn0_lo, ebn0_hi, rate;         // per-frame Eb/N0 (see QcParams)
    unsigned long long* snr_bins;
    const int32_t* scols;                 // step kernel: its column table (byte offsets)
    const int32_t* slot;                  // step kernel: [N] shared-memory slot of each variable
    const int32_t* slow;                  // step kernel: [n_steps] 1 for a step of low-degree rows
    int32_t n_steps;
};

void general_schedule(const int32_t* rows, int N, int M, int dmax, std::vector<int32_t>& order,
                      std::vector<int32_t>& starts);
int build_general(const int32_t* rows, int N, int M, int P, int dmax, GeneralCode* g, std::string& err);
void free_general(GeneralCode* g);
// No-allocation variant of ldpc_decode_llr (device buffers, static scratch); see general.cu.
int decode_llr_static(const ldpc_matrix* h, const ldpc_run_params* p, const float* d_llr, int64_t n,
                      float* d_post, int32_t* d_iters, int32_t* d_synd, int32_t* d_be, ldpc_tally* out,
                      cudaStream_t stream, std::string& err);
// The step kernel's degree bound for rows of at most maxdeg edges (6, 8 or 10), or 0 when the
// matrix needs the warp kernel.
int step_dt(int maxdeg);
// The step kernel's schedule (general_step.cu): steps of up to 32 rows of one degree class (low:
// degree <= dl), each row after the earlier rows it shares a variable with.  low[s] = 1 for a low step.
void step_schedule(const int32_t* rows, int N, int M, int dmax, int dl, std::vector<int32_t>& order,
                   std::vector<int32_t>& starts, std::vector<uint8_t>& low);
// Builds the step kernel's schedule and tables for the matrix of build_general.
int build_general_steps(const int32_t* rows, int dmax, GeneralCode* g, std::string& err);
// The step kernel; LDPC_ENOTSUP when it does not run these numerics or this matrix (the caller then
// takes the warp kernel).
int launch_general_step(GeneralCode* g, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                        const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be,
                        unsigned long long* d_tally, unsigned long long* d_hist, int hist_bins, unsigned int* d_work,
                        int n_sm, cudaStream_t stream, std::string& err, unsigned long long* d_snr_bins);
int launch_general(GeneralCode* g, const ldpc_run_params* p, bool ext, uint32_t n, uint64_t first,
                   const float* d_llr, float* d_post, int32_t* d_it, int32_t* d_sf, int32_t* d_be,
                   unsigned long long* d_tally, unsigned long long* d_hist, int hist_bins, unsigned int* d_work,
                   int n_sm, cudaStream_t stream, std::string& err, unsigned long long* d_snr_bins = nullptr);

}  // namespace ldpcb200
