// Kernel variants for Z = 64, D = 10: AR4JA rate 2/3, K = 1024 (N = 1792, 768 checks).
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_r23k1[] = {
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, true, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_NMS, false, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_NMS, true, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, true, true),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_NMS, false, true),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_BF16, ALGO_NMS, true, true),
    // weighted Approximate-Min* (trained weights, LDPC_ALGO_WAMIN): simulation and caller-supplied LLRs
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP16, ALGO_WAMIN, false, true),
    LDPC_QC_ENTRY(64, 10, 1, 1, STORE_FP32, ALGO_WAMIN, false, true),
    // column offset table in shared memory (layout 2)
    LDPC_QC_ENTRY_OT(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(64, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(64, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    // layout 6: the code's descriptors compiled in, no offset table
    LDPC_QC_ENTRY_RF(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0, 8),
    // layout 7: messages in global memory with the degree-10 layers in a loop that is not unrolled:
    // fp32 24.2 (offset table) -> 25.7, bf16 21.1 (layout 6) -> 22.4 M frames/s at threshold + 1.25 dB
    LDPC_QC_ENTRY_GR(64, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_GR(64, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 16),
    LDPC_QC_ENTRY_GR(64, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 16),
};
LDPC_QC_REGISTER(qc_r23k1)
