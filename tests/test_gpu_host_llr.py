"""Caller LLRs from host memory: bf16 input (ldpc_decode_llr_bf16) and pageable arrays staged through
the pinned ring.  Bit-exact: bf16 values widened on the device decode exactly as the same values
given as fp32; a pageable array decodes exactly as the same data in page-locked memory."""
import numpy as np
import pytest

from conftest import golden_matrix
from ldpcb200 import ar4ja, capi

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _bf16(x):
    """fp32 -> bf16 bit patterns, round to nearest even (finite values)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def _widen(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


def _same(a, b):
    assert np.array_equal(_bits(a[0]), _bits(b[0])) if a[0] is not None else b[0] is None
    for k in (1, 2, 3):
        assert np.array_equal(a[k], b[k])
    ta, tb = a[4], b[4]
    assert (ta.frames, ta.bit_errors, ta.frame_errors, ta.iter_sum) == (tb.frames, tb.bit_errors, tb.frame_errors,
                                                                       tb.iter_sum)


def _pinned(a):
    """A page-locked copy of a (torch's pinned allocator) as a numpy view, and its owner."""
    import torch
    t = torch.empty(a.shape, dtype=torch.int16 if a.dtype == np.uint16 else torch.float32, pin_memory=True)
    v = t.numpy().view(a.dtype)
    v[...] = a
    return v, t


@pytest.mark.parametrize("n", [7, 20000])
def test_bf16_input_equals_fp32_of_the_same_values(n, gpu):
    c = ar4ja.make_code(1024, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.75)
    rng = np.random.default_rng(n)
    b = _bf16(mu + sigma * rng.standard_normal((n, c.n_tx)))
    with capi.Decoder.from_code(c, 0) as dec:
        p = dec.params(max_iter=60, storage="bf16")
        want_post = n < 100
        a = dec.decode_llr(_widen(b), p, want_post=want_post)
        z = dec.decode_llr(b, p, want_post=want_post)
    _same(a, z)


def test_bf16_input_on_general_matrix_with_odd_width(gpu):
    """A general matrix whose N - P is odd (the widening kernel's unaligned tail)."""
    rng = np.random.default_rng(3)
    N, M, P = 301, 150, 30
    rows = np.full((M, 6), -1, np.int32)
    for m in range(M):
        k = int(rng.integers(2, 7))
        rows[m, :k] = rng.choice(N, size=k, replace=False)
    b = _bf16(1.0 + 1.5 * rng.standard_normal((33, N - P)))
    with capi.Decoder(rows, N, P, 0) as dec:
        assert dec.kind == capi.KERNEL_GENERAL
        p = dec.params(max_iter=25, storage="fp32")
        _same(dec.decode_llr(_widen(b), p), dec.decode_llr(b, p))


@pytest.mark.parametrize("bf16", [False, True])
def test_pageable_equals_pinned(golden, gpu, bf16):
    """The shipped file, 40000 frames (five chunks, each larger than a staging slot for fp32): a
    pageable array through the staging ring and the same data page-locked give the same bits."""
    rows, N, P = golden_matrix(golden, "shipped")
    mu, sigma = capi.channel_mu_sigma(N, rows.shape[0], P, 2.0)
    rng = np.random.default_rng(11)
    x = (mu + sigma * rng.standard_normal((40000, N - P))).astype(np.float32)
    if bf16:
        x = _bf16(x)
    with capi.Decoder(rows, N, P, 0) as dec:
        p = dec.params(max_iter=100, storage="bf16")
        pin, owner = _pinned(x)
        a = dec.decode_llr(pin, p, want_post=False)
        z = dec.decode_llr(x.copy(), p, want_post=False)
    _same(a, z)
    assert a[4].frames == 40000
