"""Matrix-file parsing: formats and error behaviour of ldpc_sim_scalar.cpp:116-269."""
import pytest

from ldpcb200 import ar4ja, chinn


def test_chinn_out_with_comments_and_zero_values(tmp_path):
    p = tmp_path / "m.chinn.out"
    p.write_text("# comment\n\n1 1 1.0\n1 3 1.0\n2 2 1.0\n2 3 0.0\n2 1 1.0\n2 3 1.0\n2 3 0.0\n")
    m = chinn.parse_chinn(str(p))
    assert (m.M, m.N) == (2, 3)
    assert [list(r) for r in m.rows] == [[0, 2], [1, 0, 2]]  # file order kept, zero values skipped
    assert m.max_check_deg == 3 and m.max_var_deg == 2


def test_chinn_row_format(tmp_path):
    p = tmp_path / "m.chinn"
    p.write_text("4 2\n2 3\n3 1 2 4\n2 3 4\n")
    m = chinn.parse_chinn(str(p))
    assert (m.N, m.M, m.max_var_deg, m.max_check_deg) == (4, 2, 2, 3)
    assert [list(r) for r in m.rows] == [[0, 1, 3], [2, 3]]


def test_chinn_row_format_inline_degrees(tmp_path):
    p = tmp_path / "m.chinn"
    p.write_text("4 2 2 3\n3 1 2 4\n2 3 4\n")
    m = chinn.parse_chinn(str(p))
    assert [list(r) for r in m.rows] == [[0, 1, 3], [2, 3]]


@pytest.mark.parametrize("text,msg", [
    ("", "empty"),
    ("1 5 1.0\n2 3 0.0\n", "out of bounds"),
    ("0 1 1.0\n2 3 0.0\n", "out of bounds"),
])
def test_chinn_out_errors(tmp_path, text, msg):
    p = tmp_path / "bad.chinn.out"
    p.write_text(text)
    with pytest.raises(chinn.MatrixError, match=msg):
        chinn.parse_chinn(str(p))


def test_missing_file():
    with pytest.raises(chinn.MatrixError, match="Could not open"):
        chinn.parse_chinn("/nonexistent/file.chinn.out")


def test_truncated_row_list(tmp_path):
    p = tmp_path / "m.chinn"
    p.write_text("4 3\n2 3\n3 1 2 4\n")
    with pytest.raises(chinn.MatrixError, match="Unexpected EOF"):
        chinn.parse_chinn(str(p))


def test_degree_limit(tmp_path):
    n = chinn.MAX_CHECK_DEG + 1
    lines = [f"1 {c} 1.0" for c in range(1, n + 1)] + [f"1 {n} 0.0"]
    p = tmp_path / "wide.chinn.out"
    p.write_text("\n".join(lines) + "\n")
    with pytest.raises(chinn.MatrixError, match="exceeds MAX_DEG"):
        chinn.parse_chinn(str(p))


def test_conflict_free_runs_makeh_order():
    c = ar4ja.make_code(1024, "1/2")
    m = chinn.Matrix(N=c.N, M=c.n_checks, max_var_deg=6, max_check_deg=6, rows=c.rows())
    runs = chinn.conflict_free_runs(m)
    assert runs == [i * 128 for i in range(13)]  # exactly the 12 layers of Z = 128 rows


def test_chinn_out_text_round_trip(tmp_path):
    """A row table written as .chinn.out reads back with the same rows in the same edge order (the
    shipped matrix rebuilt from the committed fixture)."""
    import numpy as np
    import conftest
    g = np.load(conftest.GOLDEN)
    rows = g["shipped_rows"].astype(np.int32)
    p = tmp_path / "shipped.chinn.out"
    p.write_text(chinn.chinn_out_text(rows, 2560))
    m = chinn.parse_chinn(str(p))
    assert (m.M, m.N) == rows.shape[:1] + (2560,)
    for r, back in zip(rows, m.rows):
        assert back.tolist() == r[r >= 0].tolist()
    rr = np.array([[2, 0, -1], [1, -1, -1]], np.int32)  # an edge order that is not ascending
    p.write_text(chinn.chinn_out_text(rr, 3))
    assert [r.tolist() for r in chinn.parse_chinn(str(p)).rows] == [[2, 0], [1]]
