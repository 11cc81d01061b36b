"""Iterative-decoding thresholds of the AR4JA protographs by protograph EXIT (PEXIT) analysis.

The reference does not define the "code threshold" its mixed-code configuration is expressed in, so
it is computed here: PEXIT analysis (G. Liva and M. Chiani, "Protograph LDPC codes design based on
EXIT analysis", IEEE GLOBECOM 2007) of the AR4JA protograph of each rate, on the BPSK-AWGN channel
with the punctured variable node receiving no channel information.  Mutual information uses the
J-function approximation of F. Brannstrom, L. K. Rasmussen and A. J. Grant ("Convergence analysis
and optimal scheduling for multiple concatenated codes", IEEE Trans. IT 2005):
J(s) = (1 - 2^(-H1 s^(2 H2)))^H3 with H1 = 0.3073, H2 = 0.8935, H3 = 1.1064.

The threshold is the smallest Eb/N0 (dB) at which the a-posteriori mutual information of every
variable node reaches 1 (to 1e-6) within the iteration budget; it depends on the protograph (the
rate), not on the lifting size K.
"""
from __future__ import annotations

from functools import lru_cache
from typing import Dict

import numpy as np

H1, H2, H3 = 0.3073, 0.8935, 1.1064

# AR4JA protographs: edge multiplicities per (check, variable) of the 3 x (5, 7, 11) base matrices
# (makeH_AR4JA.m:94-98: "I + P1" counts two edges, "P2 + P3 + P4" three).  The last column is
# punctured.
_B12 = [[0, 0, 1, 0, 2],
        [1, 1, 0, 1, 3],
        [1, 2, 0, 2, 1]]
_P23 = [[0, 0], [3, 1], [1, 3]]
_P45 = [[0, 0, 0, 0], [3, 1, 3, 1], [1, 3, 1, 3]]


def protograph(rate: str) -> np.ndarray:
    if rate == "1/2":
        rows = _B12
    elif rate == "2/3":
        rows = [p + r for p, r in zip(_P23, _B12)]
    elif rate == "4/5":
        rows = [a + b + c for a, b, c in zip(_P45, _P23, _B12)]
    else:
        raise ValueError(rate)
    return np.array(rows, dtype=np.int64)


def J(s):
    s = np.asarray(s, dtype=np.float64)
    return np.power(1.0 - np.power(2.0, -H1 * np.power(np.maximum(s, 0.0), 2.0 * H2)), H3)


def Jinv(i):
    i = np.clip(np.asarray(i, dtype=np.float64), 0.0, 1.0 - 1e-15)
    return np.power(-np.log2(1.0 - np.power(i, 1.0 / H3)) / H1, 1.0 / (2.0 * H2))


def converges(B: np.ndarray, ebn0_db: float, rate: float, iters: int = 2000, tol: float = 1e-6,
              punctured_last: bool = True) -> bool:
    """PEXIT recursion on protograph B at Eb/N0 (``rate`` = information bits per transmitted bit);
    the last column is punctured unless ``punctured_last`` is False."""
    m, n = B.shape
    sigma_ch2 = np.full(n, 8.0 * rate * 10.0 ** (ebn0_db / 10.0))  # variance of the channel LLR
    if punctured_last:
        sigma_ch2[-1] = 0.0
    E = B > 0
    Iac = np.zeros((m, n))  # check -> variable
    for _ in range(iters):
        # variable -> check
        jinv_c = Jinv(Iac) ** 2 * B  # sum over the multi-edges of column j
        tot_v = jinv_c.sum(axis=0) + sigma_ch2
        Iav = np.where(E, J(np.sqrt(np.maximum(tot_v[None, :] - Jinv(Iac) ** 2, 0.0))), 0.0)
        # check -> variable
        jinv_v = Jinv(1.0 - Iav) ** 2 * B
        tot_c = jinv_v.sum(axis=1)
        Iac = np.where(E, 1.0 - J(np.sqrt(np.maximum(tot_c[:, None] - Jinv(1.0 - Iav) ** 2, 0.0))), 0.0)
        app = J(np.sqrt((Jinv(Iac) ** 2 * B).sum(axis=0) + sigma_ch2))
        if np.all(app > 1.0 - tol):
            return True
    return False


def search(B: np.ndarray, rate: float, punctured_last: bool, lo: float = -1.0, hi: float = 4.0,
           tol: float = 1e-3) -> float:
    """Bisection for the smallest converging Eb/N0 (dB) of protograph B."""
    assert not converges(B, lo, rate, punctured_last=punctured_last)
    assert converges(B, hi, rate, punctured_last=punctured_last)
    while hi - lo > tol:
        mid = 0.5 * (lo + hi)
        if converges(B, mid, rate, punctured_last=punctured_last):
            hi = mid
        else:
            lo = mid
    return round(hi, 3)


@lru_cache(maxsize=None)
def threshold_db(rate: str) -> float:
    """PEXIT threshold of the AR4JA protograph of ``rate`` ("1/2", "2/3", "4/5") in Eb/N0 dB."""
    num, den = (int(x) for x in rate.split("/"))
    return search(protograph(rate), num / den, punctured_last=True)


def all_thresholds() -> Dict[str, float]:
    return {r: threshold_db(r) for r in ("1/2", "2/3", "4/5")}


if __name__ == "__main__":
    for r, t in all_thresholds().items():
        print(f"AR4JA rate {r}: PEXIT threshold {t:.3f} dB")
