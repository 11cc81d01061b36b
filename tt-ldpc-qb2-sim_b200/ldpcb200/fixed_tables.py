"""Layer descriptors compiled into the global-message kernels (csrc/ar4ja_fixed_tables.h): the K = 16384
codes and the degree-18 rate-4/5 codes at K = 1024 and 4096.

The QC kernel reads each edge's column block offset and circulant shift from its launch parameters
(the constant bank); with the descriptors of a known code compiled in, they become immediate
operands and the circulant index of an edge costs an add and a mask less per row.  The header holds
the descriptors exactly as ldpc_create detects them from a makeH-order matrix file (edge e of layer
l = the e-th column of the layer's first row: block * Z and shift), and the library offers the
compiled kernels (launch layout 5) only for a matrix whose detected descriptors equal them.

    python -m ldpcb200.fixed_tables            writes the header
    python -m ldpcb200.fixed_tables --check    exits 1 if the header differs from what it would write
"""
from __future__ import annotations

import os
import sys
from typing import List, Tuple

from . import ar4ja

CODES = ((16384, "1/2"), (16384, "2/3"), (16384, "4/5"), (1024, "4/5"), (4096, "4/5"), (1024, "1/2"),
         (4096, "1/2"), (4096, "2/3"), (1024, "2/3"))
LAYERS, DMAX = 12, 18
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "csrc", "ar4ja_fixed_tables.h")


def descriptors(code: ar4ja.QcCode) -> Tuple[int, int, List[List[int]], List[List[int]]]:
    """(Z, D, blk_off[12][18], shift[12][18]) as ldpc_create's structure detection finds them."""
    rows = code.row_matrix()
    Z = code.n_checks // LAYERS
    blk = [[0] * DMAX for _ in range(LAYERS)]
    sh = [[0] * DMAX for _ in range(LAYERS)]
    D = 0
    for l in range(LAYERS):
        r0 = [int(c) for c in rows[l * Z] if c >= 0]
        if l >= 4:
            D = len(r0)
        for e, c in enumerate(r0):
            blk[l][e] = (c // Z) * Z
            sh[l][e] = c % Z
    return Z, D, blk, sh


def _rows(t: List[List[int]]) -> str:
    return ",\n".join("         {" + ", ".join(str(v) for v in r) + "}" for r in t)


def _initializer() -> str:
    entries = []
    for K, rate in CODES:
        Z, D, blk, sh = descriptors(ar4ja.make_code(K, rate))
        entries.append(f"    // AR4JA rate {rate}, K = {K}\n"
                       f"    {{{Z}, {D},\n      {{\n{_rows(blk)}}},\n      {{\n{_rows(sh)}}}}}")
    return "{\n" + ",\n".join(entries) + "}"


def header_text() -> str:
    init = _initializer()
    return f"""// Generated by `python -m ldpcb200.fixed_tables` from ldpcb200.ar4ja (the makeH construction): the
// layer descriptors of the codes whose global-message kernels compile them in (launch layout 5).
// Edge e of layer l: column block * Z and circulant shift, as ldpc_create detects them.  Do not edit.
#pragma once
#include <cstdint>

namespace ldpcb200 {{

struct QcFixedTable {{
    int32_t Z, D;
    int32_t blk_off[{LAYERS}][{DMAX}];
    int32_t shift[{LAYERS}][{DMAX}];
}};

constexpr int QC_FIXED_COUNT = {len(CODES)};

// host copy (kernel selection)
static constexpr QcFixedTable kQcFixedHost[QC_FIXED_COUNT] = {init};

// device copy (read at compile-time indices, so the values become immediate operands)
static __device__ constexpr QcFixedTable kQcFixedDev[QC_FIXED_COUNT] = {init};

}}  // namespace ldpcb200
"""


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    text = header_text()
    if "--check" in argv:
        with open(HEADER) as f:
            return 0 if f.read() == text else 1
    with open(HEADER, "w") as f:
        f.write(text)
    print(HEADER)
    return 0


if __name__ == "__main__":
    sys.exit(main())
