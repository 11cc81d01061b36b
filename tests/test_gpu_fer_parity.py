"""Statistical parity of the whole Monte Carlo path with the reference's own CPU decoder.

The reference curves (tests/golden/fer_reference_*.json, made by tests/golden/make_fer_reference.py)
come from the reference's run_ldpc_worker with its xoshiro128+/polar channel, 10^4 frames per point,
Eb/N0 0.5 to 2.0 dB in 0.25 dB steps, at most 200 iterations.  The GPU path decodes the same code in
the same row order with its Philox/Box-Muller channel; the decoders are bit-identical given the same
LLRs (test_gpu_parity.py), so the curves may differ only through the noise realisations.  Bar: at
every point the 95% Clopper-Pearson intervals of FER overlap, and so do the 95% intervals of BER.
Bit errors cluster (a failed frame carries hundreds), so the BER interval takes the frame (GPU) or
the codeword pair (reference worker) as its independent unit, with the per-unit variance from the
tallied sums of squared bit-error counts (ldpcb200.stats.ber_interval).

fp32 message storage is a different, more precise decoder than the reference's bf16 one: its FER
intervals must still overlap the reference's, and its BER must not be worse (its interval's lower
end at most the reference interval's upper end); in the waterfall it is measurably better.
"""
import json
import os

import pytest

from conftest import REPO, golden_matrix
from ldpcb200 import ar4ja, capi
from ldpcb200.stats import ber_interval, clopper_pearson, intervals_overlap

pytestmark = pytest.mark.gpu

CURVES = {
    "makeh": os.path.join(REPO, "tests", "golden", "fer_reference_config1.json"),
    "shipped": os.path.join(REPO, "tests", "golden", "fer_reference_config1_shipped.json"),
}


def _rows(golden, which):
    if which == "makeh":
        c = ar4ja.make_code(1024, "1/2")
        return c.row_matrix(), c.N, c.P
    return golden_matrix(golden, "shipped")


@pytest.mark.parametrize("which,storage", [("makeh", "bf16"), ("makeh", "fp32"), ("shipped", "bf16")])
def test_fer_ber_within_reference_confidence_intervals(golden, gpu, which, storage):
    if not os.path.exists(CURVES[which]):
        pytest.skip("reference curve not generated")
    ref = json.load(open(CURVES[which]))
    rows, N, P = _rows(golden, which)
    ntx = N - P
    with capi.Decoder(rows, N, P, 0) as dec:
        for pt in ref["points"]:
            mu, sigma = capi.channel_mu_sigma(N, rows.shape[0], P, pt["ebn0"])
            r = dec.run_chunk(dec.params(mu=mu, sigma=sigma, seed=1, n_frames=pt["frames"], max_iter=ref["max_iter"],
                                         storage=storage))
            fer_g = clopper_pearson(r.frame_errors, r.frames)
            fer_r = clopper_pearson(pt["frame_errors"], pt["frames"])
            assert intervals_overlap(fer_g, fer_r), (pt["ebn0"], r.frame_errors, pt["frame_errors"])
            ber_g = ber_interval(r.bit_errors, r.bit_errors_sq, r.frames, ntx)
            ber_r = ber_interval(pt["bit_errors"], pt["bit_errors_sq_pairs"], pt["frames"] // 2, 2 * ntx)
            if storage == "bf16":
                assert intervals_overlap(ber_g, ber_r), (pt["ebn0"], r.bit_errors, pt["bit_errors"])
            else:
                assert ber_g[0] <= ber_r[1], (pt["ebn0"], r.bit_errors, pt["bit_errors"])
