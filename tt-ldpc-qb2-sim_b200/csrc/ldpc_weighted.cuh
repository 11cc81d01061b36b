// Weighted Approximate-Min* decoder with a hand-written adjoint (training path).
//
// Row update of the layered decoder with per-iteration t, per-protograph-edge-class c parameters
// (scale alpha[t][c], offset beta[t][c]):
//     q_e = L_v - r_e
//     m_e = Approximate-Min* magnitude of edge e (as in the plain decoder: the recursive min* over the
//           row's other edges, ldpc_decoder_core.h:176-201)
//     r_e = sign_e * relu(alpha[t][c_e] * m_e - beta[t][c_e]),   sign_e = parity(q) * sign(q_e)
//     L_v = q_e + r_e
// With alpha = 1 and beta = 0 every value equals the plain fp32 decoder's bit for bit.  T iterations
// are unrolled with no early stop (the training graph); the posteriors after every iteration (or after
// the last) are the outputs.  The backward pass recomputes each segment of ckpt_every iterations from
// an activation checkpoint (L and r at the segment's start), stashing every layer's q, then walks the
// layers in reverse: adjoints of L in shared memory, of r in global memory, parameter gradients
// reduced per warp into shared memory.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "ldpc_qc.cuh"

namespace ldpcb200 {

constexpr int W_MAX_ITER = 64;
constexpr int W_MAX_CLASSES = 64;

struct WParams {
    int32_t blk_off[QC_LAYERS][QC_DMAX];
    int32_t shift[QC_LAYERS][QC_DMAX];
    int32_t edge_class[QC_LAYERS][QC_DMAX];
    int32_t layer_off[QC_LAYERS];  // element offset of layer l in a frame's [edge][row] message array
    int32_t n_vars, n_tx, n_edges;  // N, N - P, E
    int32_t n_iter, n_classes, ckpt_every, post_all;
    int32_t n_frames;
    // arrays of the kernel's real type (float, or double for adjoint checks)
    const void* llr;       // [B][n_tx]
    const void* alpha;     // [T][C]
    const void* beta;      // [T][C]
    void* post;            // [T or 1][B][N]
    void* ckpt;            // [ceil(T / every)][B][N + E]
    void* rwork;           // [B][E] message state
    void* stash;           // [B][every][E] q of every layer of one segment
    void* gr;              // [B][E] adjoint of the messages
    const void* gpost;     // [T or 1][B][N] adjoint of the posteriors
    void* galpha;          // [T][C] (accumulated)
    void* gbeta;           // [T][C] (accumulated)
    void* gllr;            // [B][n_tx] (optional)
};

// Host side (weighted.cu); real_bytes 4 (float) or 8 (double).
int weighted_forward(const WParams& p, int Z, int D, int real_bytes, cudaStream_t stream, std::string& err);
int weighted_backward(const WParams& p, int Z, int D, int real_bytes, cudaStream_t stream, std::string& err);
bool weighted_supported(int Z, int D, int real_bytes);
size_t weighted_smem_bytes(const WParams& p, bool fwd, int real_bytes);

}  // namespace ldpcb200
