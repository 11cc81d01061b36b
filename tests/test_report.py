"""ldpcb200.report: the reference consumer's confidence-interval table without plotting, checked
against the reference's own code run on the same synthetic tables (tests/golden/make_report_ci.py):
add_confidence_intervals (combine_and_plot_results.py:30-61) and load_jpl_results
(tools/import_jpl_results.py:100-240).  Tolerance: 1e-12 relative (the same scipy quantiles; the
report forms the ratios in the same order)."""
import csv
import os
import subprocess
import sys

import numpy as np

import conftest
from ldpcb200 import report, stats

G = os.path.join(conftest.REPO, "tests", "golden")


def _ref_rows(name):
    with open(os.path.join(G, name), newline="") as f:
        return list(csv.DictReader(f))


def _close(a, b):
    return abs(float(a) - float(b)) <= 1e-12 * max(1.0, abs(float(b)))


def test_sweep_poisson_columns_equal_reference_consumer():
    rows = report.read_results_csv(os.path.join(G, "report_input_sweep.csv"))
    ref = _ref_rows("report_ci_reference.csv")
    assert len(rows) == len(ref) == 7
    for r, e in zip(rows, ref):
        assert r["EbN0_dB"] == round(float(e["EbN0_dB"]), 2)
        assert r["Total_Blocks"] == int(e["Total_Blocks"]) and r["Total_Block_Errors"] == int(e["Total_Block_Errors"])
        for k in ("SER", "FER", "FER_ci_lower", "FER_ci_upper", "SER_ci_lower", "SER_ci_upper", "FER_err_minus",
                  "FER_err_plus", "SER_err_minus", "SER_err_plus"):
            assert _close(r[k], e[k]), (k, r[k], e[k])


def test_jpl_file_equals_reference_importer():
    rows = report.read_jpl(os.path.join(G, "report_input_jpl.txt"))
    ref = _ref_rows("report_jpl_reference.csv")
    assert len(rows) == len(ref) == 4  # the commented-out data line is skipped, as the importer does
    for r, e in zip(rows, ref):
        assert abs(r["EbN0_dB"] - round(float(e["EbN0_dB"]), 2)) < 1e-9
        assert _close(r["SER"], e["BER"]) and _close(r["FER"], e["FER_calc"])
        assert _close(r["FER_ci_lower"], e["FER_ci_lower"]) and _close(r["FER_ci_upper"], e["FER_ci_upper"])
        assert _close(r["SER_ci_lower"], e["BER_ci_lower"]) and _close(r["SER_ci_upper"], e["BER_ci_upper"])
        assert _close(r["Mean_Iterations"], e["Avg_Iterations"])


def test_clopper_pearson_columns_bracket_the_estimate():
    for r in report.read_results_csv(os.path.join(G, "report_input_sweep.csv")):
        lo, hi = stats.clopper_pearson(r["Total_Block_Errors"], r["Total_Blocks"])
        assert (r["FER_cp_lower"], r["FER_cp_upper"]) == (lo, hi)
        assert lo <= r["Total_Block_Errors"] / r["Total_Blocks"] <= hi


def test_duplicates_keep_first_or_most_blocks(tmp_path):
    p = tmp_path / "chunks.csv"
    p.write_text("EbN0_dB,Total_Blocks,Total_Bit_Errors,Total_Block_Errors,BER,FER,Mean_Iterations\n"
                 "1.50,1000,50,4,1.9e-05,4.0e-03,12.5\n1.50,3000,170,11,2.2e-05,3.7e-03,12.4\n"
                 "1.00,2000,900,30,1.7e-04,1.5e-02,30.1\n")
    first = report.read_results_csv(str(p))
    assert [r["EbN0_dB"] for r in first] == [1.0, 1.5] and first[1]["Total_Blocks"] == 1000
    most = report.read_results_csv(str(p), chunked=True)
    assert most[1]["Total_Blocks"] == 3000 and most[1]["Mean_Iterations"] == 12.4


def test_cli_writes_the_combined_table(tmp_path):
    out = tmp_path / "combined.csv"
    r = subprocess.run([sys.executable, "-m", "ldpcb200.report", os.path.join(G, "report_input_sweep.csv"),
                        "--label", "gpu", "--jpl", os.path.join(G, "report_input_jpl.txt"), "--out", str(out)],
                       capture_output=True, text=True, timeout=120,
                       cwd=os.path.join(conftest.REPO, "tt-ldpc-qb2-sim_b200"))
    assert r.returncode == 0, r.stderr
    assert "FER 95% (Poisson)" in r.stdout
    with open(out, newline="") as f:
        rows = list(csv.DictReader(f))
    assert tuple(rows[0].keys()) == report.COLUMNS
    assert len(rows) == 11
    keys = [(float(x["EbN0_dB"]), x["Source"]) for x in rows]
    assert keys == sorted(keys)
    assert {x["Source"] for x in rows} == {"gpu", "JPL report_input_jpl.txt"}
    z = [x for x in rows if x["Total_Block_Errors"] == "0"]
    assert all(float(x["FER_ci_upper"]) == 0.0 and float(x["FER_cp_upper"]) > 0 for x in z)


def test_missing_columns_are_an_error(tmp_path):
    p = tmp_path / "bad.csv"
    p.write_text("EbN0_dB,Total_Blocks\n1.0,10\n")
    try:
        report.read_results_csv(str(p))
    except ValueError as e:
        assert "Total_Bit_Errors" in str(e)
    else:
        raise AssertionError("accepted a CSV without the error columns")
