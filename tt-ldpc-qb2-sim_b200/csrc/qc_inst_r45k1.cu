// Kernel variants for Z = 32, D = 18: AR4JA rate 4/5, K = 1024 (N = 1408, 384 checks).
// FP32 message storage is not built for D = 18: 156 fp32 messages per thread do not fit the
// register file next to the working set (16-bit storage packs them into 78 registers).
#include "ldpc_qc.cuh"
#include "ldpc_registry.h"

using namespace ldpcb200;

static const QcEntry qc_r45k1[] = {
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, true, false),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_NMS, false, false),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_NMS, true, false),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, true),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, true, true),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_NMS, false, true),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_BF16, ALGO_NMS, true, true),
    // weighted Approximate-Min* (trained weights, LDPC_ALGO_WAMIN): simulation and caller-supplied LLRs
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, false),
    LDPC_QC_ENTRY(32, 18, 1, 1, STORE_FP16, ALGO_WAMIN, false, true),
    // column offset table in shared memory (layout 2)
    LDPC_QC_ENTRY_OT(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_OT(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    // check messages in global memory (layout 1): the 156 per-thread message registers of the
    // register layout leave room for only 8-10 warps per SM; without them the kernel holds more frames
    LDPC_QC_ENTRY_G(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_G(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 0),
    LDPC_QC_ENTRY_G(32, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 0),
    // the same capped at 64 registers (32 CTAs of 32 threads per SM)
    LDPC_QC_ENTRY_G(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 32),
    LDPC_QC_ENTRY_G(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 32),
    LDPC_QC_ENTRY_G(32, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 32),
    // layout 5: the register-capped shapes with the code's layer descriptors compiled in
    // (ar4ja_fixed_tables.h entry 3)
    LDPC_QC_ENTRY_GF(32, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 32, 3),
    LDPC_QC_ENTRY_GF(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 32, 3),
    LDPC_QC_ENTRY_GF(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 32, 3),
    // layout 7: the eight degree-18 layers in a loop that is not unrolled.  The unrolled body does
    // not fit the instruction cache, and with one-warp CTAs each warp is somewhere else in it (ncu:
    // 9 no-instruction stalls per issue, issue 46 %).  Rolled, at 16-24 CTAs per SM (80-112
    // registers, no 64-register spills, a message scratch that stays in L2): fp32 23.1 -> 34.5,
    // bf16 21.3 -> 30.9 M frames/s at threshold + 1.25 dB.
    LDPC_QC_ENTRY_GR(32, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 24),
    LDPC_QC_ENTRY_GR(32, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 20),
    LDPC_QC_ENTRY_GR(32, 18, 1, 1, STORE_FP32, ALGO_AMIN, false, false, 16),
    LDPC_QC_ENTRY_GR(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 24),
    LDPC_QC_ENTRY_GR(32, 18, 1, 1, STORE_BF16, ALGO_AMIN, false, false, 16),
    LDPC_QC_ENTRY_GR(32, 18, 1, 1, STORE_FP16, ALGO_AMIN, false, false, 16),
};
LDPC_QC_REGISTER(qc_r45k1)
