// Kernel variants for the K = 16384 AR4JA codes.  Their check messages (94,208 to 122,880 edges per
// frame) do not fit the register file, so they live in an L2-resident global scratch (RG kernels):
//   rate 1/2: Z = 2048, D = 6  (N = 40960, 24576 checks), 512 threads x 4 rows
//   rate 2/3: Z = 1024, D = 10 (N = 28672, 12288 checks), 512 threads x 2 rows
//   rate 4/5: Z = 512,  D = 18 (N = 22528,  6144 checks), 512 threads x 1 row
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

#define K16_SHAPE(Z, D, R)                                                          \
    LDPC_QC_ENTRY_G(Z, D, R, 1, STORE_BF16, ALGO_AMIN, false, false, 0),            \
    LDPC_QC_ENTRY_G(Z, D, R, 1, STORE_FP16, ALGO_AMIN, false, false, 0),            \
    LDPC_QC_ENTRY_G(Z, D, R, 1, STORE_FP32, ALGO_AMIN, false, false, 0),            \
    LDPC_QC_ENTRY_G(Z, D, R, 1, STORE_BF16, ALGO_AMIN, false, true, 0),             \
    LDPC_QC_ENTRY_G(Z, D, R, 1, STORE_FP16, ALGO_AMIN, false, true, 0),             \
    LDPC_QC_ENTRY_G(Z, D, R, 1, STORE_FP32, ALGO_AMIN, false, true, 0)

static const QcEntry qc_k16[] = {
    K16_SHAPE(2048, 6, 4),
    K16_SHAPE(1024, 10, 2),
    K16_SHAPE(512, 18, 1),
    // register cap of 64 (2 CTAs of 512 threads per SM) for the codes whose kernels need 77-110
    LDPC_QC_ENTRY_G(1024, 10, 2, 1, STORE_BF16, ALGO_AMIN, false, false, 2),
    LDPC_QC_ENTRY_G(1024, 10, 2, 1, STORE_FP16, ALGO_AMIN, false, false, 2),
    LDPC_QC_ENTRY_G(512, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 2),
    LDPC_QC_ENTRY_G(512, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 2),
    // layout 5: the same kernels with the code's layer descriptors compiled in (ar4ja_fixed_tables.h:
    // 0 = rate 1/2, 1 = rate 2/3, 2 = rate 4/5), so a circulant index costs no constant-bank operands
    LDPC_QC_ENTRY_GF(2048, 6, 4, 1, STORE_BF16, ALGO_AMIN, false, false, 0, 0),
    LDPC_QC_ENTRY_GF(2048, 6, 4, 1, STORE_FP16, ALGO_AMIN, false, false, 0, 0),
    LDPC_QC_ENTRY_GF(2048, 6, 4, 1, STORE_BF16, ALGO_AMIN, false, true, 0, 0),
    LDPC_QC_ENTRY_GF(1024, 10, 2, 1, STORE_BF16, ALGO_AMIN, false, false, 0, 1),
    LDPC_QC_ENTRY_GF(1024, 10, 2, 1, STORE_BF16, ALGO_AMIN, false, false, 2, 1),
    LDPC_QC_ENTRY_GF(1024, 10, 2, 1, STORE_FP16, ALGO_AMIN, false, false, 2, 1),
    LDPC_QC_ENTRY_GF(512, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0, 2),
    LDPC_QC_ENTRY_GF(512, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 2, 2),
    LDPC_QC_ENTRY_GF(512, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 2, 2),
};
LDPC_QC_REGISTER(qc_k16)
