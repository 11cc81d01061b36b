"""The general kernel's row schedule (ldpc_row_schedule, host only): steps of at most 32 rows that
share no variable, every pair of rows sharing one kept in file order, so decoding in schedule order
gives the file order's bits (engines/scalar_5w/ldpc_decoder_core.h:314-522 updates the rows one after
another in file order)."""
import numpy as np
import pytest

from conftest import golden_matrix
from ldpcb200 import ar4ja, capi, chinn
from oracle import oracle as O


def _matrix(rows, N):
    return chinn.Matrix(N=N, M=rows.shape[0], max_var_deg=0, max_check_deg=rows.shape[1],
                        rows=[r[r >= 0] for r in rows])


def _check_schedule(rows, order, starts):
    M = rows.shape[0]
    assert sorted(order) == list(range(M))
    assert starts[0] == 0 and starts[-1] == M and all(b > a for a, b in zip(starts, starts[1:]))
    step = np.empty(M, np.int64)
    for k in range(len(starts) - 1):
        a, b = starts[k], starts[k + 1]
        assert b - a <= 32
        cols = np.concatenate([rows[m][rows[m] >= 0] for m in order[a:b]])
        assert len(cols) == len(set(cols.tolist())), k  # no shared variable inside a step
        step[order[a:b]] = k
    last = {}
    for m in range(M):  # rows sharing a variable: the earlier file row runs in an earlier step
        for c in rows[m][rows[m] >= 0].tolist():
            if c in last:
                assert step[last[c]] < step[m], (last[c], m)
            last[c] = m


def test_shipped_file_schedule(golden):
    rows, N, _ = golden_matrix(golden, "shipped")
    order, starts = chinn.row_schedule(_matrix(rows, N))
    _check_schedule(rows, np.array(order), starts)
    assert len(chinn.conflict_free_runs(_matrix(rows, N))) - 1 == 135  # file order
    assert len(starts) - 1 == 51                                         # the schedule


@pytest.mark.parametrize("K,rate", [(1024, "1/2"), (1024, "4/5"), (4096, "2/3")])
def test_makeh_order_schedule_is_the_layers(K, rate):
    c = ar4ja.make_code(K, rate)
    rows = c.row_matrix()
    order, starts = chinn.row_schedule(_matrix(rows, c.N))
    _check_schedule(rows, np.array(order), starts)
    assert order == list(range(c.n_checks))  # makeH order is already level order
    Z = c.n_checks // 12
    assert len(starts) - 1 == 12 * max(1, Z // 32)


def test_library_schedule_equals_restatement(golden):
    rng = np.random.default_rng(3)
    cases = [golden_matrix(golden, "shipped")[:2]]
    c = ar4ja.make_code(1024, "2/3")
    cases.append((c.row_matrix(), c.N))
    for _ in range(4):  # random sparse matrices with ragged rows and holes at the end
        N, M, d = int(rng.integers(20, 200)), int(rng.integers(5, 300)), int(rng.integers(1, 9))
        rows = np.full((M, d), -1, np.int32)
        for m in range(M):
            k = int(rng.integers(0, d + 1))
            rows[m, :k] = rng.choice(N, size=k, replace=False)
        cases.append((rows, N))
    for rows, N in cases:
        order, starts = capi.row_schedule(rows, N)
        o2, s2 = chinn.row_schedule(_matrix(rows, N))
        assert order.tolist() == list(o2) and starts.tolist() == list(s2)
        _check_schedule(rows, order, starts)


def test_bad_matrix_is_rejected():
    rows = np.array([[0, 5]], np.int32)
    with pytest.raises(capi.LdpcError):
        capi.row_schedule(rows, 4)  # column 5 of 4 variables


@pytest.mark.parametrize("mode", [O.STORE_BF16, O.STORE_FP32])
def test_schedule_order_decodes_as_the_file_order(golden, mode):
    """The oracle decoding the rows serially in schedule order gives the same posteriors, iteration
    counts and tallies as in file order (the shipped file, frames that converge and frames that
    do not)."""
    rows, N, P = golden_matrix(golden, "shipped")
    order, _ = chinn.row_schedule(_matrix(rows, N))
    file_code = O.Code(rows, N, P)
    sched_code = O.Code(rows[np.array(order)], N, P)
    rng = np.random.default_rng(11)
    mu, sigma = capi.channel_mu_sigma(N, rows.shape[0], P, 1.0)
    llr = (mu + sigma * rng.standard_normal((6, N - P))).astype(np.float32)
    a = O.decode(file_code, llr, mode=mode, max_iter=30)
    b = O.decode(sched_code, llr, mode=mode, max_iter=30)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert (a[2] > 0).any() and (a[2] == 0).any()  # some frames stop, some do not


# The step kernel's schedule (ldpc_step_schedule): the same ordering rule, steps of one degree class.

def _check_classes(rows, order, starts, low, dl):
    deg = (rows >= 0).sum(1)
    for k in range(len(starts) - 1):
        d = deg[np.array(order[starts[k]:starts[k + 1]])]
        assert (d <= dl).all() if low[k] else (d > dl).all(), k


def test_step_schedule_of_the_shipped_file(golden):
    """512 rows of degree 3 and 1024 of degree 6: 54 steps (18 of degree 3, 36 of degree 6, against
    the 16 and 32 that full steps would need) in place of the row schedule's 51 mixed steps."""
    rows, N, _ = golden_matrix(golden, "shipped")
    order, starts, low = capi.step_schedule(rows, N)
    _check_schedule(rows, order, starts)
    _check_classes(rows, order, starts, low, 3)
    assert len(starts) - 1 == 54 and int(low.sum()) == 18
    o2, s2, l2 = chinn.step_schedule(_matrix(rows, N), 3)
    assert order.tolist() == o2 and starts.tolist() == s2 and low.tolist() == l2


def test_step_schedule_equals_restatement():
    rng = np.random.default_rng(5)
    cases = []
    for K, rate in ((1024, "1/2"), (1024, "4/5"), (4096, "2/3")):
        c = ar4ja.make_code(K, rate)
        if c.row_matrix().shape[1] <= 10:
            cases.append((c.row_matrix(), c.N))
    for _ in range(6):  # random ragged matrices, degrees 0-10
        N, M, d = int(rng.integers(20, 300)), int(rng.integers(5, 400)), int(rng.integers(1, 11))
        rows = np.full((M, d), -1, np.int32)
        for m in range(M):
            k = int(rng.integers(0, d + 1))
            rows[m, :k] = rng.choice(N, size=k, replace=False)
        cases.append((rows, N))
    for rows, N in cases:
        maxdeg = int((rows >= 0).sum(1).max())
        dl = (6 if maxdeg <= 6 else 8 if maxdeg <= 8 else 10) // 2
        order, starts, low = capi.step_schedule(rows, N)
        o2, s2, l2 = chinn.step_schedule(_matrix(rows, N), dl)
        assert order.tolist() == o2 and starts.tolist() == s2 and low.tolist() == l2
        _check_schedule(rows, order, starts)
        _check_classes(rows, order, starts, low, dl)


def test_step_schedule_rejects_rows_above_degree_10():
    rows = np.arange(11, dtype=np.int32)[None, :]
    with pytest.raises(capi.LdpcError):
        capi.step_schedule(rows, 20)


@pytest.mark.parametrize("mode", [O.STORE_BF16, O.STORE_FP32])
def test_step_schedule_order_decodes_as_the_file_order(golden, mode):
    rows, N, P = golden_matrix(golden, "shipped")
    order, _, _ = capi.step_schedule(rows, N)
    rng = np.random.default_rng(12)
    mu, sigma = capi.channel_mu_sigma(N, rows.shape[0], P, 1.0)
    llr = (mu + sigma * rng.standard_normal((6, N - P))).astype(np.float32)
    a = O.decode(O.Code(rows, N, P), llr, mode=mode, max_iter=30)
    b = O.decode(O.Code(rows[np.array(order)], N, P), llr, mode=mode, max_iter=30)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
