"""GPU parity of the circulant engine's decoder (LDPC_ALGO_CIRC), called through the C ABI.

Against the reference's own circulant golden stepper (tests/golden/golden_circulant_stepper.npz,
made by tests/golden/make_golden_circ.py from tests/test_circulant_dma_stepper.cpp compiled from the
reference's sources) and against the CPU restatement in oracle/ (oracle_circ_decode), which the
fixture pins.  Bar: bit-exact (bf16 nodes, iteration counts, frame and bit errors), tolerance 0.
"""
import os

import numpy as np
import pytest

from ldpcb200 import ar4ja, capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_circulant_stepper.npz")


def _bits_to_f32(bits):
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _channel(rng, n, ntx, ebn0, rate=0.5):
    g = 10.0 ** (ebn0 / 10.0)
    x = (4.0 * rate * g + np.sqrt(8.0 * rate * g) * rng.standard_normal((n, ntx))).astype(np.float32)
    u = x.view(np.uint32).astype(np.uint64)  # bf16 values, as the engines hold their channel
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16).astype(np.uint32)).view(np.float32)


@pytest.fixture(scope="module")
def code_r12k1():
    c = ar4ja.make_code(1024, "1/2")
    return c, O.Code(c.row_matrix(), c.N, c.P)


@pytest.fixture(scope="module")
def dec_r12k1(gpu, code_r12k1):
    d = capi.Decoder.from_code(code_r12k1[0], 0)
    yield d
    d.close()


def _circ(dec, llr, numerics, stop, damping, max_iter, storage="bf16"):
    dec.set_circulant(numerics, stop, damping)
    p = dec.params(max_iter=max_iter, storage=storage, algo=capi.ALGO_CIRC)
    return dec.decode_llr(llr, p)


def _check_tally(tal, it, be, fe):
    b = be.astype(np.int64)
    assert tal.frames == len(be) and tal.iter_sum == int(it.sum())
    assert tal.bit_errors == int(b.sum()) and tal.bit_errors_sq == int((b * b).sum())
    assert tal.frame_errors == int(fe.sum())


@pytest.mark.parametrize("idx", range(7))
def test_circ_matches_reference_stepper(dec_r12k1, idx):
    """Every fixture case (scalar and SFPU stepper paths, damping 1 and 15/16, converging and capped
    runs): the GPU leaves the reference stepper's bf16 nodes and reports its iterations, frame
    errors and bit errors."""
    z = np.load(GOLDEN)
    llr = _bits_to_f32(z["llr_bits"][idx])
    num = capi.CIRC_SFPU if z["sfpu"][idx] else capi.CIRC_SCALAR
    post, it, sf, be, tal = _circ(dec_r12k1, llr, num, capi.CIRC_STOP_SYNDROME, float(z["damping"][idx]),
                                  int(z["max_iter"][idx]))
    want = _bits_to_f32(z["post_bits"][idx])
    assert np.array_equal(_u32(post), _u32(want))
    assert np.array_equal(it, z["iters"][idx])
    assert np.array_equal(be, z["bit_errors"][idx])
    _check_tally(tal, it, be, z["frame_error"][idx])


@pytest.mark.parametrize("numerics,stop,damping", [
    (capi.CIRC_SFPU, capi.CIRC_STOP_GENIE, 0.9375),      # the engine on silicon
    (capi.CIRC_SFPU, capi.CIRC_STOP_SYNDROME, 0.8),
    (capi.CIRC_SCALAR, capi.CIRC_STOP_SYNDROME, 1.0),   # the stepper's scalar path
    (capi.CIRC_SCALAR, capi.CIRC_STOP_GENIE, 1.0),
])
@pytest.mark.parametrize("storage", ["bf16", "fp32"])
def test_circ_matches_oracle(dec_r12k1, code_r12k1, numerics, stop, damping, storage):
    """Fresh frames from 0.5 to 3 dB against oracle_circ_decode, both stop rules, both storages."""
    c, code = code_r12k1
    rng = np.random.default_rng(1000 + 10 * numerics + stop + (storage == "fp32"))
    llr = np.concatenate([_channel(rng, 24, c.n_tx, eb) for eb in (0.5, 1.25, 2.0, 3.0)])
    post, it, sf, be, tal = _circ(dec_r12k1, llr, numerics, stop, damping, 40, storage)
    mode = O.STORE_BF16 if storage == "bf16" else O.STORE_FP32
    wp, wit, wsf, wbe, wfe = O.circ_decode(code, llr, numerics=numerics, damping=damping, stop=stop,
                                           max_iter=40, mode=mode)
    assert np.array_equal(_u32(post), _u32(wp))
    assert np.array_equal(it, wit) and np.array_equal(sf, wsf) and np.array_equal(be, wbe)
    _check_tally(tal, it, be, wfe)
    assert 0 < wfe.sum() < len(wfe)  # both outcomes occur


def test_circ_zero_and_one_iteration(dec_r12k1, code_r12k1):
    """max_iter 0 and 1: the degenerate caps of both stop rules and tallies."""
    c, code = code_r12k1
    llr = _channel(np.random.default_rng(9), 16, c.n_tx, 1.0)
    for stop in (capi.CIRC_STOP_SYNDROME, capi.CIRC_STOP_GENIE):
        for mi in (0, 1):
            post, it, sf, be, tal = _circ(dec_r12k1, llr, capi.CIRC_SFPU, stop, 0.9375, mi)
            wp, wit, wsf, wbe, wfe = O.circ_decode(code, llr, numerics=O.CIRC_SFPU, damping=0.9375, stop=stop,
                                                   max_iter=mi)
            assert np.array_equal(_u32(post), _u32(wp)) and np.array_equal(it, wit) and np.array_equal(be, wbe)
            _check_tally(tal, it, be, wfe)


def test_circ_offset_table_layout_equal(dec_r12k1, code_r12k1):
    """The offset-table layout of the bf16 kernel (layout 2) decodes every frame to the same bits."""
    c, _ = code_r12k1
    assert (1, 1, 0, 2) in dec_r12k1.shapes("bf16", capi.ALGO_CIRC)
    dec_r12k1.set_circulant(capi.CIRC_SFPU, capi.CIRC_STOP_GENIE, 0.9375)
    p = dec_r12k1.params(mu=3.17, sigma=2.52, seed=4, n_frames=1 << 14, max_iter=60, storage="bf16",
                         algo=capi.ALGO_CIRC)
    a = dec_r12k1.run_chunk(p)
    dec_r12k1.set_launch_shape(1, 1, 0, 2, storage="bf16")
    try:
        b = dec_r12k1.run_chunk(p)
    finally:
        dec_r12k1.set_launch_shape(0, 0, 0, 0, storage="bf16")
    assert (a.frames, a.bit_errors, a.frame_errors, a.iter_sum, a.bit_errors_sq) == \
           (b.frames, b.bit_errors, b.frame_errors, b.iter_sum, b.bit_errors_sq)


def test_circ_simulation_equals_decoding_its_channel(dec_r12k1):
    """ldpc_run_chunk with ALGO_CIRC decodes the same frames as ldpc_decode_llr fed that run's channel
    (ldpc_channel_llr): same tallies."""
    dec_r12k1.set_circulant(capi.CIRC_SFPU, capi.CIRC_STOP_GENIE, 0.9375)
    d = dec_r12k1
    mu, sigma = capi.channel_mu_sigma(d.N, d.M, d.P, 1.25)
    p = d.params(mu=mu, sigma=sigma, seed=77, first_frame=5000, n_frames=2048, max_iter=50,
                 storage="bf16", algo=capi.ALGO_CIRC)
    sim = d.run_chunk(p)
    llr = d.channel_llr(p)
    post, it, sf, be, tal = d.decode_llr(llr, p)
    assert (sim.frames, sim.bit_errors, sim.frame_errors, sim.iter_sum) == \
           (tal.frames, tal.bit_errors, tal.frame_errors, tal.iter_sum)
    assert sim.frame_errors > 0


@pytest.mark.parametrize("K", [4096, 16384])
def test_circ_larger_rate_half_codes(gpu, K):
    """K = 4096 (registers) and K = 16384 (messages in global memory) against the oracle."""
    c = ar4ja.make_code(K, "1/2")
    code = O.Code(c.row_matrix(), c.N, c.P)
    llr = _channel(np.random.default_rng(K), 4 if K == 16384 else 8, c.n_tx, 1.1)
    with capi.Decoder.from_code(c, 0) as dec:
        for num, stop, damp in ((capi.CIRC_SFPU, capi.CIRC_STOP_GENIE, 0.9375),
                                (capi.CIRC_SCALAR, capi.CIRC_STOP_SYNDROME, 1.0)):
            post, it, sf, be, tal = _circ(dec, llr, num, stop, damp, 25)
            wp, wit, wsf, wbe, wfe = O.circ_decode(code, llr, numerics=num, damping=damp, stop=stop, max_iter=25)
            assert np.array_equal(_u32(post), _u32(wp))
            assert np.array_equal(it, wit) and np.array_equal(be, wbe)
            _check_tally(tal, it, be, wfe)


def test_circ_rejections(gpu):
    """Codes without degree-6 rows, clips and bad settings are refused, not approximated."""
    c = ar4ja.make_code(1024, "2/3")
    with capi.Decoder.from_code(c, 0) as dec:
        with pytest.raises(capi.LdpcError) as e:
            dec.run_chunk(dec.params(mu=4.0, sigma=2.8, n_frames=4, algo=capi.ALGO_CIRC))
        assert e.value.code == -95
    c = ar4ja.make_code(1024, "1/2")
    with capi.Decoder.from_code(c, 0) as dec:
        with pytest.raises(capi.LdpcError):
            dec.run_chunk(dec.params(mu=4.0, sigma=2.8, n_frames=4, algo=capi.ALGO_CIRC, r_max=3.0))
        for args in ((capi.CIRC_SCALAR, capi.CIRC_STOP_GENIE, 0.9375), (capi.CIRC_SFPU, 0, 0.0),
                     (capi.CIRC_SFPU, 0, 1.5), (7, 0, 1.0), (capi.CIRC_SFPU, 5, 1.0)):
            with pytest.raises(capi.LdpcError) as e:
                dec.set_circulant(*args)
            assert e.value.code == -22


def test_circ_per_frame_snr_bins(dec_r12k1):
    """A per-frame Eb/N0 range: the per-bin tallies sum to the chunk's, frame errors by the engine's rule."""
    dec_r12k1.set_circulant(capi.CIRC_SFPU, capi.CIRC_STOP_SYNDROME, 0.9375)
    p = dec_r12k1.params(seed=3, n_frames=1 << 14, max_iter=30, storage="bf16", algo=capi.ALGO_CIRC,
                         ebn0_lo=0.5, ebn0_hi=2.0)
    r = dec_r12k1.run_chunk(p)
    bins = dec_r12k1.snr_bins()
    assert int(bins[0].sum()) == r.frames and int(bins[1].sum()) == r.frame_errors
    assert int(bins[2].sum()) == r.bit_errors and int(bins[3].sum()) == r.iter_sum
    fer = bins[1][:8].sum() / max(1, bins[0][:8].sum()), bins[1][-8:].sum() / max(1, bins[0][-8:].sum())
    assert fer[0] > fer[1]


def test_circ_cli(gpu, tmp_path, capsys):
    """ldpc_sim --circulant: a short point on the makeH r1/2 K=1024 file ends with the final JSON
    line; a matrix the decoder does not cover (rate 2/3) and an unbuilt storage fail cleanly."""
    import io
    import json

    from ldpcb200 import sim
    good = tmp_path / "r12.chinn.out"
    good.write_text(ar4ja.make_code(1024, "1/2").chinn_out_text())
    out = io.StringIO()
    rc = sim.main(["-c", str(good), "-e", "1.5", "-p", "512", "-s", "-k", "20000", "-b", "10000", "-i", "50",
                   "-t", "1000", "--circulant", "device"], out=out)
    lines = [json.loads(l) for l in out.getvalue().splitlines() if l.startswith("{")]
    assert rc == 0 and lines[-1]["blocks"] == 20000 and lines[-1]["frame_errors"] > 0
    bad = tmp_path / "r23.chinn.out"
    bad.write_text(ar4ja.make_code(1024, "2/3").chinn_out_text())
    assert sim.main(["-c", str(bad), "-e", "2.0", "-p", "256", "-s", "-k", "100", "--circulant", "device"],
                    out=io.StringIO()) == 1
    assert sim.main(["-c", str(good), "-e", "2.0", "-p", "512", "-s", "-k", "100", "--circulant", "device",
                     "--storage", "fp16"], out=io.StringIO()) == 1
    assert "circulant engine's decoder cannot run" in capsys.readouterr().err


def test_circ_fer_matches_reference_stepper_monte_carlo(dec_r12k1):
    """Statistical parity with the reference's own circulant Monte Carlo (its stepper's scalar path,
    its std::normal_distribution channel; tests/golden/fer_reference_circulant.json, made by
    tests/golden/make_fer_reference_circ.py): at every Eb/N0 point the 95% Clopper-Pearson intervals
    of the frame error rates overlap.  The GPU decodes 10^5 Philox frames per point with the same
    settings (scalar arithmetic, syndrome after every iteration, no damping, 200 iterations)."""
    import json

    from ldpcb200 import stats
    ref = json.load(open(os.path.join(os.path.dirname(GOLDEN), "fer_reference_circulant.json")))
    d = dec_r12k1
    d.set_circulant(capi.CIRC_SCALAR, capi.CIRC_STOP_SYNDROME, 1.0)
    for pt in ref["points"]:
        mu, sigma = capi.channel_mu_sigma(d.N, d.M, d.P, pt["ebn0"])
        r = d.run_chunk(d.params(mu=mu, sigma=sigma, seed=5, n_frames=100000, max_iter=200, storage="bf16",
                                 algo=capi.ALGO_CIRC))
        ours = stats.clopper_pearson(r.frame_errors, r.frames)
        theirs = stats.clopper_pearson(pt["frame_errors"], pt["frames"])
        assert stats.intervals_overlap(ours, theirs), (pt["ebn0"], r.frame_errors, pt["frame_errors"])


def test_circulant_engine_binary_drop_in(gpu, tmp_path):
    """ldpc_sim_circulant_dma (the drop-in for the reference's circulant engine binary): a short
    single-core run writes the engine's CSV rows and summary, and its totals equal ldpc_run_chunk with
    the same settings over the same frames."""
    import io

    from ldpcb200 import sim_circ
    csv = tmp_path / "c.csv"
    out = io.StringIO()
    rc = sim_circ.main(["1.5", "30000", "50", "--single-core", "--chunk-batches", "2500", "--min-fe", "1000000",
                        "--out", str(csv), "--seed", "17"], out=out)
    assert rc == 0
    rows = csv.read_text().splitlines()
    assert len(rows) == 1 + 3  # header + chunks of 10000, 10000, 10000
    blocks, be, fe = (int(x) for x in rows[-1].split(",")[1:4])
    assert blocks == 30000 and fe > 0
    c = ar4ja.make_code(1024, "1/2")
    with capi.Decoder.from_code(c, 0) as dec:
        dec.set_circulant(capi.CIRC_SFPU, capi.CIRC_STOP_GENIE, 0.9375)
        g = 10.0 ** 0.15
        p = dec.params(mu=float(np.float32(2.0 * g)), sigma=float(np.float32(np.sqrt(4.0 * g))), seed=17,
                       n_frames=30000, max_iter=50, storage="bf16", algo=capi.ALGO_CIRC)
        r = dec.run_chunk(p)
    assert (r.frames, r.bit_errors, r.frame_errors) == (blocks, be, fe)
    assert any(l.strip() == f"Frame Errors:     {fe}" for l in out.getvalue().splitlines())
