"""Confidence intervals for error-rate estimates.

Clopper-Pearson (exact binomial) intervals for FER and BER, and the Poisson interval the reference's
result importer uses (tools/import_jpl_results.py:66-80 of the reference), both from the chi-square /
beta quantiles in scipy.
"""
from __future__ import annotations

from typing import Tuple

from scipy import stats as _st


def clopper_pearson(k: int, n: int, conf: float = 0.95) -> Tuple[float, float]:
    """Exact two-sided binomial interval for k successes in n trials."""
    if n <= 0:
        return 0.0, 1.0
    a = 1.0 - conf
    lo = 0.0 if k <= 0 else float(_st.beta.ppf(a / 2, k, n - k + 1))
    hi = 1.0 if k >= n else float(_st.beta.ppf(1 - a / 2, k + 1, n - k))
    return lo, hi


def poisson_interval(k: int, conf: float = 0.95) -> Tuple[float, float]:
    """Exact Poisson interval for a count k (chi-square form)."""
    a = 1.0 - conf
    lo = 0.0 if k <= 0 else float(_st.chi2.ppf(a / 2, 2 * k) / 2)
    hi = float(_st.chi2.ppf(1 - a / 2, 2 * k + 2) / 2)
    return lo, hi


def intervals_overlap(a: Tuple[float, float], b: Tuple[float, float]) -> bool:
    return a[0] <= b[1] and b[0] <= a[1]
