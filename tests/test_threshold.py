"""PEXIT thresholds (the "code threshold" of the mixed-code workload, computed since the reference
does not define it)."""
import numpy as np

from ldpcb200 import threshold as T


def test_regular_36_ensemble_matches_textbook_threshold():
    # BP threshold of the (3,6)-regular ensemble on BPSK-AWGN: sigma* = 0.8809, Eb/N0 = 1.10 dB
    t = T.search(np.array([[3, 3]]), 0.5, punctured_last=False)
    assert abs(t - 1.10) < 0.02


def test_ar4ja_thresholds():
    th = T.all_thresholds()
    assert th["1/2"] < th["2/3"] < th["4/5"]
    assert abs(th["1/2"] - 0.639) < 0.01 and abs(th["2/3"] - 1.445) < 0.01 and abs(th["4/5"] - 2.400) < 0.01


def test_protographs_match_the_code_construction():
    from ldpcb200 import ar4ja
    for rate in ("1/2", "2/3", "4/5"):
        c = ar4ja.make_code(1024, rate)
        B = T.protograph(rate)
        rm = c.row_matrix()
        M = c.M
        for bi in range(3):
            for bj in range(B.shape[1]):
                block = rm[bi * M:(bi + 1) * M]
                cnt = ((block >= bj * M) & (block < (bj + 1) * M)).sum(axis=1)
                assert (cnt == B[bi, bj]).all()


def test_ber_interval_uses_frames_as_units():
    from ldpcb200.stats import ber_interval, clopper_pearson
    # 100 frames, 10 of them failed with 200 bit errors each, 2048 bits per frame
    be, be2, n = 10 * 200, 10 * 200 ** 2, 100
    lo, hi = ber_interval(be, be2, n, 2048)
    mean = be / (n * 2048)
    assert lo < mean < hi
    # much wider than a per-bit binomial interval, which would ignore the clustering
    blo, bhi = clopper_pearson(be, n * 2048)
    assert (hi - lo) > 5 * (bhi - blo)
    assert ber_interval(0, 0, n, 2048)[0] == 0.0
