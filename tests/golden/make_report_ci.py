"""Generates tests/golden/report_ci_reference.csv and report_jpl_reference.csv: the reference's own
confidence-interval code run on synthetic result tables, for checking ldpcb200.report.

* add_confidence_intervals (combine_and_plot_results.py:30-61 of the reference) and the SER column it
  is given (:106) on report_input_sweep.csv, a synthetic sweep table in run_simulation.py's CSV
  format.  That script imports matplotlib (absent here) at its top, so only the function's own
  definition is taken from its source (ast) and run beside the reference's poisson_ci_95.
* load_jpl_results (tools/import_jpl_results.py:100-240, imported as it is) on report_input_jpl.txt,
  a synthetic file in the JPL result format.

    python tests/golden/make_report_ci.py [REF]

REF: the argument, else LDPC_REFERENCE_TREE or the oracle recipe's print-ref.  The input tables are
synthetic (numbers chosen here to cover zero, one and many frame errors); the committed outputs are
what tests/test_report.py reads.
"""
import ast
import os
import sys

import numpy as np
import pandas as pd

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle import oracle as O  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else O.reference_tree()
if not REF or not os.path.isdir(REF):
    raise SystemExit("the reference tree is needed: pass its path or set LDPC_REFERENCE_TREE")

sys.path.insert(0, os.path.join(REF, "tools"))
import import_jpl_results as J  # noqa: E402

src = open(os.path.join(REF, "combine_and_plot_results.py")).read()
fn = next(n for n in ast.parse(src).body if isinstance(n, ast.FunctionDef) and n.name == "add_confidence_intervals")
ns = {"pd": pd, "np": np, "poisson_ci_95": J.poisson_ci_95}
exec(compile(ast.Module(body=[fn], type_ignores=[]), "add_confidence_intervals", "exec"), ns)

df = pd.read_csv(os.path.join(HERE, "report_input_sweep.csv"))
df["SER"] = df["Total_Bit_Errors"] / (df["Total_Blocks"] * 2560.0)
df = ns["add_confidence_intervals"](df)
df.to_csv(os.path.join(HERE, "report_ci_reference.csv"), index=False, float_format="%.17g")

jp = J.load_jpl_results(os.path.join(HERE, "report_input_jpl.txt"), code_rate=0.5, block_length=2560)
jp.to_csv(os.path.join(HERE, "report_jpl_reference.csv"), index=False, float_format="%.17g")
print("wrote report_ci_reference.csv and report_jpl_reference.csv")
