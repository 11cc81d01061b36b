"""The drop-in for the reference's circulant engine binary (ldpc_sim_circulant_dma): its command
line, chunk rule, CSV and summary, driven on the CPU through a deterministic stub engine."""
import io
import os

import pytest

from ldpcb200 import sim_circ


class Stub:
    """Frame i is in error when i % 5000 == 0 (9 bit errors); every frame takes 6 iterations."""

    def __init__(self):
        self.calls = []

    def run(self, mu, sigma, seed, first, n, max_iter):
        self.calls.append((mu, sigma, seed, first, n, max_iter))
        fe = len(range((first + 4999) // 5000 * 5000, first + n, 5000))
        return n, fe, 9 * fe, 6 * n

    def close(self):
        pass


def run(args):
    stub = Stub()
    out = io.StringIO()
    rc = sim_circ.main(args, engine_factory=lambda: stub, out=out)
    return rc, stub, out.getvalue().splitlines()


def test_arguments_and_defaults():
    o = sim_circ.parse_args([])
    assert (o.ebn0, o.max_blocks, o.max_iter, o.min_fe, o.chunk_batches, o.single_core) == \
        (2.5, 10_000_000_000, 200, 25, 2500, False)
    o = sim_circ.parse_args(["2.1", "5000000", "150", "--single-core", "--min-fe", "7", "--chunk-batches", "10",
                             "--out", "x.csv", "--seed", "42"])
    assert (o.ebn0, o.max_blocks, o.max_iter, o.single_core, o.min_fe, o.chunk_batches, o.out_csv, o.seed) == \
        (2.1, 5000000, 150, True, 7, 10, "x.csv", 42)
    assert sim_circ.parse_args(["--seed", "random"]).random_seed
    assert sim_circ.default_csv_name(2.5, 40_000_000_000).endswith("ebn0_2.50_40B.csv")
    assert sim_circ.default_csv_name(2.0, 13_200_000).endswith("ebn0_2.00_13M.csv")
    assert sim_circ.default_csv_name(1.0, 20_000).endswith("ebn0_1.00_20k.csv")
    for bad in (["--passthrough"], ["--max-steps", "3"]):
        assert sim_circ.main(bad, engine_factory=Stub, out=io.StringIO()) == 2


def test_chunks_stop_rule_csv_and_summary(tmp_path):
    csv = str(tmp_path / "c.csv")
    # single core: chunks of 1000 batches x 4 codewords; the last chunk is cut to what is left
    rc, stub, lines = run(["1.5", "10000", "60", "--single-core", "--chunk-batches", "1000", "--min-fe", "100",
                           "--out", csv, "--seed", "9"])
    assert rc == 0
    assert [c[4] for c in stub.calls] == [4000, 4000, 2000]
    assert [c[3] for c in stub.calls] == [0, 4000, 8000]  # frames numbered across chunks
    assert all(c[2] == 9 and c[5] == 60 for c in stub.calls)
    mu, sigma = stub.calls[0][:2]
    g = 10 ** 0.15
    assert mu == pytest.approx(2.0 * g, rel=1e-6) and sigma == pytest.approx((4.0 * g) ** 0.5, rel=1e-6)
    rows = open(csv).read().splitlines()
    assert rows[0].startswith("EbN0_dB,Total_Blocks,Total_Bit_Errors,Total_Block_Errors,BER,FER")
    assert rows[-1].split(",")[:4] == ["1.50", "10000", "18", "2"]
    assert any(l.strip() == "Total Blocks:     10000" for l in lines)
    assert any(l.strip() == "Frame Errors:     2" for l in lines)
    assert any(l.strip().startswith("BER:              1.7578e-06") for l in lines)  # 18 / (10000 x 1024)
    # the mesh accounting (440 cores) and the frame-error stop
    rc, stub, _ = run(["1.5", "100000000", "--chunk-batches", "10", "--min-fe", "5", "--out", csv])
    # chunks of 10 x 4 x 440 codewords; 4 frame errors after the first (frames 0, 5000, 10000, 15000),
    # 8 after the second: the run stops there
    assert [c[4] for c in stub.calls] == [17600, 17600]


def test_benchmark_is_noiseless_and_writes_no_default_csv(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    rc, stub, _ = run(["3.0", "8", "--single-core", "--benchmark", "--chunk-batches", "1"])
    assert rc == 0 and stub.calls[0][1] == 0.0
    assert not os.path.exists(tmp_path / "Results")
    rc, stub, _ = run(["3.0", "8", "--single-core", "--chunk-batches", "1"])
    assert os.path.exists(tmp_path / "Results" / "results_circulant_dma_4cw_ar4ja_r12_ebn0_3.00_0k.csv")
