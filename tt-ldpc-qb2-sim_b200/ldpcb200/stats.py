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


def ber_interval(bit_errors: int, bit_errors_sq: int, units: int, bits_per_unit: int,
                 conf: float = 0.95) -> Tuple[float, float]:
    """Interval for BER that respects error clustering: the independent unit is the frame (or the
    codeword pair), not the bit, because a failed frame carries hundreds of correlated bit errors.
    Normal interval on the mean bit-error count per unit from its sample variance (sum of squares);
    with no errors at all, the Clopper-Pearson bound on units with an error, times the unit's bits."""
    if units <= 1:
        return 0.0, 1.0
    z = float(_st.norm.ppf(0.5 + conf / 2))
    if bit_errors == 0:
        return 0.0, clopper_pearson(0, units, conf)[1]
    mean = bit_errors / units
    var = max(bit_errors_sq / units - mean * mean, 0.0) * units / (units - 1)
    half = z * (var / units) ** 0.5
    return max(0.0, mean - half) / bits_per_unit, (mean + half) / bits_per_unit


def intervals_overlap(a: Tuple[float, float], b: Tuple[float, float]) -> bool:
    return a[0] <= b[1] and b[0] <= a[1]
