// Kernel variants of the circulant engine's decoder (ALGO_CIRC: pairwise min* tree, damping, its
// stop rules and tally) for the rate-1/2 AR4JA codes, the only ones with rows of degrees 3 and 6.
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_circ[] = {
    // K = 1024 (Z = 128): bf16 is the engine's storage; fp32 keeps L and r unrounded
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_CIRC, false, false),
    LDPC_QC_ENTRY_OT(128, 6, 1, 1, STORE_BF16, ALGO_CIRC, false, false, 0),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_BF16, ALGO_CIRC, false, true),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_CIRC, false, false),
    LDPC_QC_ENTRY(128, 6, 1, 1, STORE_FP32, ALGO_CIRC, false, true),
    // K = 4096 (Z = 512)
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_CIRC, false, false),
    LDPC_QC_ENTRY(512, 6, 1, 1, STORE_BF16, ALGO_CIRC, false, true),
    // K = 16384 (Z = 2048): check messages in global memory, 512 threads x 4 rows
    LDPC_QC_ENTRY_G(2048, 6, 4, 1, STORE_BF16, ALGO_CIRC, false, false, 0),
    LDPC_QC_ENTRY_G(2048, 6, 4, 1, STORE_BF16, ALGO_CIRC, false, true, 0),
};
LDPC_QC_REGISTER(qc_circ)
