// Kernel variants for Z = 128, D = 18: AR4JA rate 4/5, K = 4096 (N = 5632, 1536 checks).
// FP32 message storage is not built for D = 18: 156 fp32 messages per thread do not fit the
// register file next to the working set (16-bit storage packs them into 78 registers).
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_r45k4[] = {
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, true, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_NMS, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_NMS, true, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, true, true),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_NMS, false, true),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_NMS, true, true),
    // weighted Approximate-Min* (trained weights, LDPC_ALGO_WAMIN): simulation and caller-supplied LLRs
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, true),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_WAMIN, false, true),
    // column offset table in shared memory (layout 2)
    LDPC_QC_ENTRY_OT(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 18, 1, 1, STORE_BF16, ALGO_WAMIN, false, false, 0),
    // the same shapes with one (alpha, beta) per row (weights of one class per protograph check row)
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_FP16, ALGO_WROW, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_WROW, false, false),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_FP16, ALGO_WROW, false, true),
    LDPC_QC_ENTRY(128, 18, 1, 1, STORE_BF16, ALGO_WROW, false, true),
    LDPC_QC_ENTRY_OT(128, 18, 1, 1, STORE_FP16, ALGO_WROW, false, false, 0),
    LDPC_QC_ENTRY_OT(128, 18, 1, 1, STORE_BF16, ALGO_WROW, false, false, 0),
    // check messages in global memory (layout 1): the 156 per-thread message registers of the
    // register layout leave room for only 8-10 warps per SM; without them the kernel holds more frames
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    // the same capped at 64 registers (8 CTAs of 128 threads per SM)
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 8),
    // layout 5: the register-capped shapes with the code's layer descriptors compiled in
    // (ar4ja_fixed_tables.h entry 4)
    LDPC_QC_ENTRY_GF(128, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 8, 4),
    LDPC_QC_ENTRY_GF(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 8, 4),
    LDPC_QC_ENTRY_GF(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 8, 4),
    // the weighted decoders in the same layout (per-edge and per-row weights)
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_BF16, ALGO_WAMIN, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP32, ALGO_WAMIN, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP32, ALGO_WAMIN, false, true, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_BF16, ALGO_WROW, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP16, ALGO_WROW, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP32, ALGO_WROW, false, false, 8),
    LDPC_QC_ENTRY_G(128, 18, 1, 1, STORE_FP32, ALGO_WROW, false, true, 8),
    // layout 7: the degree-18 layers in a loop that is not unrolled (the instruction cache; 4-6
    // CTAs per SM at 80-112 registers): fp32 6.92 -> 8.32, bf16 6.45 -> 7.63 M frames/s at
    // threshold + 1.25 dB; and the weighted decoders in the same layout
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 4),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 5),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP32, ALGO_WAMIN, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_BF16, ALGO_WAMIN, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP32, ALGO_WROW, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_BF16, ALGO_WROW, false, false, 6),
    LDPC_QC_ENTRY_GR(128, 18, 1, 1, STORE_FP16, ALGO_WROW, false, false, 6),
};
LDPC_QC_REGISTER(qc_r45k4)
