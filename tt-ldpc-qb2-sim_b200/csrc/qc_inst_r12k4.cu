// Kernel variants for Z = 512, D = 6: AR4JA rate 1/2, K = 4096 (N = 10240, 6144 checks).
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_r12k4[] = {
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_AMIN, true, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_NMS, false, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_NMS, true, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_AMIN, true, true),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_NMS, false, true),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_NMS, true, true),
    // weighted Approximate-Min* (trained weights, LDPC_ALGO_WAMIN): simulation and caller-supplied LLRs
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP16, ALGO_WAMIN, false, true),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_FP32, ALGO_WAMIN, false, true),
    // column offset table in shared memory (layout 2)
    LDPC_QC_ENTRY_OT(512, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(512, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(512, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    // layout 6: the code's descriptors compiled in, no offset table (its 120 KB held one CTA per SM)
    LDPC_QC_ENTRY_RF(512, 6, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 1, 6),
    LDPC_QC_ENTRY_RF(512, 6, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 2, 6),
    LDPC_QC_ENTRY_RF(512, 6, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 2, 6),
};
LDPC_QC_REGISTER(qc_r12k4)
