// Kernel variants for Z = 128, D = 6: AR4JA rate 1/2, K = 1024 (N = 2560, 1536 checks).
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_r12k1[] = {
    // simulation (Philox channel), Approximate-Min*, no clips: the benchmarked path
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 2, STORE_FP32, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false),
    // paired: two interleaved frames per thread, packed f32x2 arithmetic (16-bit messages)
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_BF16, false, 0),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_BF16, false, 4),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_BF16, false, 5),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_FP16, false, 0),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_FP16, false, 4),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_FP16, false, 5),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_BF16, true, 0),
    LDPC_QC_ENTRY_PAIR(128, 6, STORE_FP16, true, 0),
    // register caps for more resident warps: 5 CTAs/SM (<= 96 registers), 6 (<= 80), 8 (<= 64)
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 5),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 5),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 8),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 5),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 8),
    // caller-supplied LLRs (parity tests, ldpc_decode_llr)
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, true),
    // reference-engine options: -n (NMS) and the -L/-R/-V/-G clips, reference numerics
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, true, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_NMS, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_NMS, true, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, true, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_NMS, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_NMS, true, true),
    // column offset table in shared memory (no circulant index arithmetic per edge)
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 5),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 8),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 8),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, true, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, true, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, true, 0),
    // layout 6: messages in registers, the code's layer descriptors compiled in (no offset table)
    LDPC_QC_ENTRY_RF(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0, 5),
    LDPC_QC_ENTRY_RF(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 5, 5),
    LDPC_QC_ENTRY_RF(128, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 6, 5),
    LDPC_QC_ENTRY_RF(128, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 8, 5),
    LDPC_QC_ENTRY_RF(128, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 6, 5),
    // weighted Approximate-Min* (trained weights, LDPC_ALGO_WAMIN): simulation and caller-supplied LLRs
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 5),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 6),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 8),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, false, 5),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_WAMIN, false, true),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, false, 5),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 6),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, true, 0),
    // the same shapes with one (alpha, beta) per row (weights of one class per protograph check row)
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_WROW, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP16, ALGO_WROW, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_WROW, false, false),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_WROW, false, false, 5),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_WROW, false, false, 6),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP16, ALGO_WROW, false, false, 8),
    LDPC_QC_ENTRY_B(128, 6, 1, 1, STORE_FP32, ALGO_WROW, false, false, 5),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_WROW, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP16, ALGO_WROW, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_WROW, false, true),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_WROW, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_WROW, false, false, 5),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP16, ALGO_WROW, false, false, 6),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_FP32, ALGO_WROW, false, true, 0),
};
LDPC_QC_REGISTER(qc_r12k1)
