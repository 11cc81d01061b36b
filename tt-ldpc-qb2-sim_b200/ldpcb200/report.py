"""Headless result report: the confidence-interval table of the reference's result consumer, without
plotting.

The reference's sweep driver appends one row per Eb/N0 point to
``Results/results_<matrix>_..._<cores>.csv`` (``EbN0_dB,Total_Blocks,Total_Bit_Errors,
Total_Block_Errors,BER,FER``, ``run_simulation.py:158-159,249-252``), and its consumer
``combine_and_plot_results.py`` reads those files, computes SER = bit errors / (blocks x 2560)
(``:99-115``), adds exact 95 % Poisson intervals on the frame-error count (``add_confidence_intervals``,
``:30-61``, with ``poisson_ci_95`` of ``tools/import_jpl_results.py:66-80``), merges the sources into
one CSV (``:118-163``) and plots it with matplotlib (absent here).  This module does all of that but
the plot, and adds Clopper-Pearson intervals on FER:

    python -m ldpcb200.report Results/results_*.csv [--jpl JPL.txt] [--out combined.csv]

Every input file is one source (its name without the extension, or ``--label``); rows of a file with
the same Eb/N0 keep the first (the consumer's ``drop_duplicates``) or, with ``--chunked``, the row with
the most blocks (the circulant engine writes one cumulative row per chunk).  ``--jpl`` adds a
historical JPL result file in the format ``tools/import_jpl_results.py`` reads (``%`` comment lines,
then ``SNR FER symbol_errors frame_errors blocks iterations`` with SNR = Es/N0, converted to Eb/N0 by
10 log10(1/R)).  The combined table goes to ``--out`` (CSV) and to stdout as text.
"""
from __future__ import annotations

import argparse
import csv
import math
import os
import sys
from typing import Dict, List, Optional, Sequence, Tuple

from . import stats

BLOCK_LENGTH = 2560  # the consumer's SER denominator per block (combine_and_plot_results.py:106,113)

COLUMNS = ("Source", "EbN0_dB", "Total_Blocks", "Total_Symbol_Errors", "Total_Block_Errors", "SER",
           "SER_ci_lower", "SER_ci_upper", "FER", "FER_ci_lower", "FER_ci_upper", "FER_err_minus",
           "FER_err_plus", "SER_err_minus", "SER_err_plus", "FER_cp_lower", "FER_cp_upper", "BER",
           "Mean_Iterations")


def poisson_ci_95(k: float) -> Tuple[float, float]:
    """The reference's exact 95 % Poisson interval for a count k (tools/import_jpl_results.py:66-80,
    its scipy branch): 0.5 chi2.ppf(0.025, 2k) (0 for k = 0) and 0.5 chi2.ppf(0.975, 2(k + 1))."""
    from scipy.stats import chi2
    low = 0.5 * chi2.ppf(0.025, 2 * k) if k > 0 else 0.0
    high = 0.5 * chi2.ppf(0.975, 2 * (k + 1))
    return float(low), float(high)


def point(source: str, ebn0: float, blocks: int, bit_errors: int, block_errors: int,
          block_length: int = BLOCK_LENGTH, ber: Optional[float] = None, mean_iters: Optional[float] = None,
          fer: Optional[float] = None) -> Dict[str, object]:
    """One row of the combined table (combine_and_plot_results.py:30-61 for the Poisson columns)."""
    n, k = int(blocks), int(block_errors)
    fer = (k / n if n > 0 else 0.0) if fer is None else float(fer)
    ser = bit_errors / (n * float(block_length)) if n > 0 else 0.0
    if n > 0 and k > 0:
        k_l, k_h = poisson_ci_95(k)
        f_lo, f_hi = k_l / n, k_h / n
        s_lo, s_hi = ser * (k_l / k), ser * (k_h / k)
    else:
        f_lo = f_hi = s_lo = s_hi = 0.0
    cp_lo, cp_hi = stats.clopper_pearson(k, n)
    return {
        "Source": source, "EbN0_dB": round(float(ebn0), 2), "Total_Blocks": n,
        "Total_Symbol_Errors": int(bit_errors), "Total_Block_Errors": k, "SER": ser,
        "SER_ci_lower": s_lo, "SER_ci_upper": s_hi, "FER": fer, "FER_ci_lower": f_lo, "FER_ci_upper": f_hi,
        "FER_err_minus": max(0.0, fer - f_lo), "FER_err_plus": max(0.0, f_hi - fer),
        "SER_err_minus": max(0.0, ser - s_lo), "SER_err_plus": max(0.0, s_hi - ser),
        "FER_cp_lower": cp_lo, "FER_cp_upper": cp_hi,
        "BER": ber if ber is not None else float("nan"),
        "Mean_Iterations": mean_iters if mean_iters is not None else float("nan"),
    }


def read_results_csv(path: str, label: str = "", chunked: bool = False,
                     block_length: int = BLOCK_LENGTH) -> List[Dict[str, object]]:
    """A sweep result CSV (run_simulation.py's, or the circulant engine's --out CSV) as table rows."""
    source = label or os.path.splitext(os.path.basename(path))[0]
    with open(path, newline="") as f:
        rows = list(csv.DictReader(f))
    need = ("EbN0_dB", "Total_Blocks", "Total_Bit_Errors", "Total_Block_Errors")
    if rows and any(c not in rows[0] for c in need):
        raise ValueError(f"{path}: missing columns {[c for c in need if c not in rows[0]]}")
    keep: Dict[float, Dict[str, str]] = {}
    order: List[float] = []
    for r in rows:
        eb = round(float(r["EbN0_dB"]), 6)
        if eb not in keep:
            keep[eb] = r
            order.append(eb)
        elif chunked and int(float(r["Total_Blocks"])) > int(float(keep[eb]["Total_Blocks"])):
            keep[eb] = r
    out = []
    for eb in sorted(order):
        r = keep[eb]
        mi = r.get("Mean_Iterations")
        out.append(point(source, float(r["EbN0_dB"]), int(float(r["Total_Blocks"])), int(float(r["Total_Bit_Errors"])),
                         int(float(r["Total_Block_Errors"])), block_length,
                         ber=float(r["BER"]) if r.get("BER") not in (None, "") else None,
                         mean_iters=float(mi) if mi not in (None, "") else None,
                         fer=float(r["FER"]) if r.get("FER") not in (None, "") else None))
    return out


def read_jpl(path: str, code_rate: float = 0.5, block_length: int = BLOCK_LENGTH,
             label: str = "JPL") -> List[Dict[str, object]]:
    """A historical JPL result file (tools/import_jpl_results.py:100-200): lines starting with '%'
    are comments; a data line holds SNR (Es/N0, dB), FER, symbol errors, frame errors, blocks run and
    total iterations; Eb/N0 = SNR + 10 log10(1/R), FER recomputed from the counts."""
    out = []
    with open(path, encoding="utf-8", errors="replace") as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("%"):
                continue
            tok = s.split()
            if len(tok) < 6:
                continue
            try:
                snr, _, sym, fe, blocks, iters = (float(t) for t in tok[:6])
            except ValueError:
                continue
            n = int(blocks)
            out.append(point(label, snr + 10.0 * math.log10(1.0 / code_rate), n, int(sym), int(fe), block_length,
                             ber=sym / (n * block_length) if n > 0 else 0.0,
                             mean_iters=iters / n if n > 0 else 0.0))
    out.sort(key=lambda r: r["EbN0_dB"])
    return out


def combine(tables: Sequence[List[Dict[str, object]]]) -> List[Dict[str, object]]:
    """All sources in one table sorted by (Eb/N0, source) (combine_and_plot_results.py:160-161)."""
    rows = [r for t in tables for r in t]
    return sorted(rows, key=lambda r: (r["EbN0_dB"], r["Source"]))


def write_csv(rows: Sequence[Dict[str, object]], path: str) -> None:
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=COLUMNS)
        w.writeheader()
        for r in rows:
            w.writerow({k: r[k] for k in COLUMNS})


def text_table(rows: Sequence[Dict[str, object]]) -> str:
    head = f"{'source':<40} {'Eb/N0':>6} {'blocks':>14} {'frame err':>10} {'FER':>10} " \
           f"{'FER 95% (Poisson)':>23} {'FER 95% (Clopper-Pearson)':>25} {'SER':>10}"
    lines = [head, "-" * len(head)]
    for r in rows:
        lines.append(f"{str(r['Source'])[:40]:<40} {r['EbN0_dB']:>6.2f} {r['Total_Blocks']:>14d} "
                     f"{r['Total_Block_Errors']:>10d} {r['FER']:>10.3e} "
                     f"[{r['FER_ci_lower']:.3e}, {r['FER_ci_upper']:.3e}] "
                     f"[{r['FER_cp_lower']:.3e}, {r['FER_cp_upper']:.3e}] {r['SER']:>10.3e}")
    return "\n".join(lines)


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("csv", nargs="*", help="sweep result CSV files (one source each)")
    ap.add_argument("--label", action="append", default=[], help="source name per CSV, in order")
    ap.add_argument("--chunked", action="store_true",
                    help="per Eb/N0 keep the row with the most blocks (cumulative per-chunk rows)")
    ap.add_argument("--jpl", action="append", default=[], help="JPL result text file(s)")
    ap.add_argument("--jpl-rate", type=float, default=0.5, help="code rate for the JPL Es/N0 -> Eb/N0 shift")
    ap.add_argument("--block-length", type=int, default=BLOCK_LENGTH, help="SER denominator per block")
    ap.add_argument("--out", default="", help="combined CSV to write")
    a = ap.parse_args(argv)
    if not a.csv and not a.jpl:
        ap.error("give at least one result CSV or --jpl file")
    tables = []
    for i, p in enumerate(a.csv):
        tables.append(read_results_csv(p, a.label[i] if i < len(a.label) else "", a.chunked, a.block_length))
    for p in a.jpl:
        tables.append(read_jpl(p, a.jpl_rate, a.block_length, label="JPL " + os.path.basename(p)))
    rows = combine(tables)
    if a.out:
        write_csv(rows, a.out)
    print(text_table(rows))
    return 0


if __name__ == "__main__":
    sys.exit(main())
