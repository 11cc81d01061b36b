// Registry of compiled kernel variants.  Each instantiation unit (qc_inst_*.cu, general.cu) adds its
// kernels to a table the host API searches by shape; a shape that was not built is reported as
// LDPC_ENOTSUP instead of being emulated.
#pragma once
#include <cstdint>

namespace ldpcb200 {

struct QcKey {
    int Z, D, R, F, mode, algo, clip, ext, B;  // B: min resident CTAs per SM (register cap), 0 = none
    int G;                                     // layout: 0 registers, 1 messages in global memory (RG
                                               // kernel), 2 registers + column offset table (OT),
                                               // 5 as 1 with a known code's descriptors compiled in,
                                               // 6 as 0 with them compiled in, 7 as 1 with the
                                               // degree-D layers in a loop not unrolled
    // F = 2 with 16-bit storage, Approximate-Min*, no clips is the paired kernel (two interleaved
    // slots per thread, packed f32x2 arithmetic).
    bool operator==(const QcKey& o) const {
        return Z == o.Z && D == o.D && R == o.R && F == o.F && mode == o.mode && algo == o.algo &&
               clip == o.clip && ext == o.ext && B == o.B && G == o.G;
    }
};

struct QcEntry {
    QcKey key;
    const void* fn;  // __global__ void (const QcParams)
};

struct QcTable {
    const QcEntry* entries;
    int count;
    const QcTable* next;
};

// Linked at static-initialisation time by each instantiation unit.
void register_qc_table(QcTable* t);
const QcTable* qc_tables();

}  // namespace ldpcb200

#define LDPC_QC_ENTRY(Z, D, R, F, MODE, ALGO, CLIP, EXT) LDPC_QC_ENTRY_B(Z, D, R, F, MODE, ALGO, CLIP, EXT, 0)
#define LDPC_QC_ENTRY_B(Z, D, R, F, MODE, ALGO, CLIP, EXT, B)                  \
    {{Z, D, R, F, MODE, ALGO, CLIP, EXT, B, 0},                                \
     reinterpret_cast<const void*>(&::ldpcb200::qc_decode_kernel<Z, D, R, F, MODE, ALGO, CLIP, EXT, B>)}
#define LDPC_QC_ENTRY_G(Z, D, R, F, MODE, ALGO, CLIP, EXT, B)                  \
    {{Z, D, R, F, MODE, ALGO, CLIP, EXT, B, 1},                                \
     reinterpret_cast<const void*>(                                            \
         &::ldpcb200::qc_decode_kernel<Z, D, R, F, MODE, ALGO, CLIP, EXT, B, false, true>)}

// Layout 5: the global-message kernel with the layer descriptors of fixed-table code FIX compiled in.
#define LDPC_QC_ENTRY_GF(Z, D, R, F, MODE, ALGO, CLIP, EXT, B, FIX)           \
    {{Z, D, R, F, MODE, ALGO, CLIP, EXT, B, 5},                                \
     reinterpret_cast<const void*>(                                            \
         &::ldpcb200::qc_decode_kernel<Z, D, R, F, MODE, ALGO, CLIP, EXT, B, false, true, false, FIX>)}

// Layout 6: messages in registers with the layer descriptors of fixed-table code FIX compiled in.
#define LDPC_QC_ENTRY_RF(Z, D, R, F, MODE, ALGO, CLIP, EXT, B, FIX)           \
    {{Z, D, R, F, MODE, ALGO, CLIP, EXT, B, 6},                                \
     reinterpret_cast<const void*>(                                            \
         &::ldpcb200::qc_decode_kernel<Z, D, R, F, MODE, ALGO, CLIP, EXT, B, false, false, false, FIX>)}

// Layout 7: the global-message kernel with its degree-D layers in a loop that is not unrolled.
#define LDPC_QC_ENTRY_GR(Z, D, R, F, MODE, ALGO, CLIP, EXT, B)                 \
    {{Z, D, R, F, MODE, ALGO, CLIP, EXT, B, 7},                                \
     reinterpret_cast<const void*>(                                            \
         &::ldpcb200::qc_decode_kernel<Z, D, R, F, MODE, ALGO, CLIP, EXT, B, false, true, false, -1, true>)}

#define LDPC_QC_ENTRY_OT(Z, D, R, F, MODE, ALGO, CLIP, EXT, B)                 \
    {{Z, D, R, F, MODE, ALGO, CLIP, EXT, B, 2},                                \
     reinterpret_cast<const void*>(                                            \
         &::ldpcb200::qc_decode_kernel<Z, D, R, F, MODE, ALGO, CLIP, EXT, B, false, false, true>)}

#define LDPC_QC_ENTRY_PAIR(Z, D, MODE, EXT, B)                                 \
    {{Z, D, 1, 2, MODE, ::ldpcb200::ALGO_AMIN, 0, EXT, B, 0},                  \
     reinterpret_cast<const void*>(                                            \
         &::ldpcb200::qc_decode_kernel<Z, D, 1, 2, MODE, ::ldpcb200::ALGO_AMIN, false, EXT, B, true>)}

#define LDPC_QC_REGISTER(name)                                                           \
    namespace {                                                                          \
    struct name##_reg {                                                                  \
        name##_reg() {                                                                   \
            static ::ldpcb200::QcTable t{name, (int)(sizeof(name) / sizeof(name[0])), nullptr}; \
            ::ldpcb200::register_qc_table(&t);                                           \
        }                                                                                \
    } name##_reg_instance;                                                               \
    }
