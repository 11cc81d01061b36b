// Kernel variants for Z = 256, D = 10: AR4JA rate 2/3, K = 4096 (N = 7168, 3072 checks).
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_r23k4[] = {
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_AMIN, true, false),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_NMS, false, false),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_NMS, true, false),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_AMIN, true, true),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_NMS, false, true),
    LDPC_QC_ENTRY(256, 10, 1, 1, STORE_BF16, ALGO_NMS, true, true),
    // column offset table in shared memory (layout 2)
    LDPC_QC_ENTRY_OT(256, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(256, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(256, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    // layout 6: the code's descriptors compiled in, no offset table
    LDPC_QC_ENTRY_RF(256, 10, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 2, 7),
    LDPC_QC_ENTRY_RF(256, 10, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 2, 7),
    LDPC_QC_ENTRY_RF(256, 10, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 3, 7),
};
LDPC_QC_REGISTER(qc_r23k4)
