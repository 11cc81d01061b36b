"""ctypes binding of libldpcb200 (include/ldpcb200.h).

There is no CPU path behind this module: if the library is missing, or no sm_100 GPU is present,
every call raises.  ``Decoder`` owns one handle (one CUDA stream); use it from one thread at a time.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libldpcb200.so")

STORE_BF16, STORE_FP32, STORE_FP16 = 0, 1, 2
ALGO_AMIN, ALGO_NMS, ALGO_WAMIN, ALGO_CIRC = 0, 1, 2, 3
CIRC_SCALAR, CIRC_SFPU = 0, 1
CIRC_STOP_SYNDROME, CIRC_STOP_GENIE = 0, 1
KERNEL_QC, KERNEL_GENERAL = 0, 1
STORAGE_NAMES = {"bf16": STORE_BF16, "fp32": STORE_FP32, "fp16": STORE_FP16}

# The entry points include/ldpcb200.h declares (tests check that the library exports each one).
EXPORTS = ("ldpc_create", "ldpc_destroy", "ldpc_kernel_kind", "ldpc_run_chunk", "ldpc_decode_llr",
           "ldpc_decode_llr_bf16",
           "ldpc_channel_llr", "ldpc_channel_llr_device", "ldpc_iter_histogram", "ldpc_snr_bins",
           "ldpc_set_launch_shape", "ldpc_list_shapes", "ldpc_list_shapes_algo", "ldpc_set_weights",
           "ldpc_set_circulant",
           "ldpc_wdec_workspace_bytes", "ldpc_wdec_forward", "ldpc_wdec_backward",
           "ldpc_launch_count", "ldpc_batch_create", "ldpc_batch_destroy", "ldpc_batch_run",
           "ldpc_batch_graph_builds", "ldpc_batch_set_order",
           "ldpc_launch_param_bytes", "ldpc_decode_llr_static", "ldpc_row_schedule", "ldpc_step_schedule",
           "ldpc_last_error",
           "ldpc_abi_version")


class LdpcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


class LibraryMissing(LdpcError):
    pass


class Matrix(C.Structure):
    _fields_ = [("n_vars", C.c_int32), ("n_checks", C.c_int32), ("n_punct", C.c_int32),
                ("max_check_deg", C.c_int32), ("rows", C.POINTER(C.c_int32))]


class RunParams(C.Structure):
    _fields_ = [("mu", C.c_float), ("sigma", C.c_float), ("seed", C.c_uint64), ("stream", C.c_uint32),
                ("reserved0", C.c_uint32), ("first_frame", C.c_uint64), ("n_frames", C.c_uint64),
                ("max_iter", C.c_int32), ("storage", C.c_int32), ("algo", C.c_int32),
                ("l_max", C.c_float), ("r_max", C.c_float), ("l_post_max", C.c_float),
                ("ebn0_lo_db", C.c_float), ("ebn0_hi_db", C.c_float)]


SNR_BINS = 32


class WdecConfig(C.Structure):
    _fields_ = [("n_iter", C.c_int32), ("n_classes", C.c_int32), ("ckpt_every", C.c_int32),
                ("post_all", C.c_int32), ("fp64", C.c_int32), ("reserved0", C.c_int32),
                ("edge_class", (C.c_int32 * 18) * 12)]


class CircConfig(C.Structure):
    """ldpc_circ_config: settings of ALGO_CIRC runs (the circulant engine's decoder)."""
    _fields_ = [("numerics", C.c_int32), ("stop", C.c_int32), ("damping", C.c_float), ("reserved0", C.c_int32)]


class Tally(C.Structure):
    _fields_ = [("frames", C.c_uint64), ("bit_errors", C.c_uint64), ("frame_errors", C.c_uint64),
                ("iter_sum", C.c_uint64), ("unconverged", C.c_uint64), ("max_iters", C.c_uint64),
                ("kernel_ms", C.c_float), ("reserved1", C.c_float), ("bit_errors_sq", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once).  Raises LibraryMissing if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LibraryMissing(-2, f"{path} is missing: build it with `python -m ldpcb200.build` "
                                 "(or __graft_entry__.build()); there is no CPU fallback")
    L = C.CDLL(path)
    P = C.POINTER
    L.ldpc_create.argtypes = [P(Matrix), C.c_int, P(C.c_void_p)]
    L.ldpc_destroy.argtypes = [C.c_void_p]
    L.ldpc_destroy.restype = None
    L.ldpc_kernel_kind.argtypes = [C.c_void_p]
    L.ldpc_run_chunk.argtypes = [C.c_void_p, P(RunParams), P(Tally)]
    L.ldpc_decode_llr.argtypes = [C.c_void_p, P(RunParams), P(C.c_float), C.c_int64, P(C.c_float),
                                  P(C.c_int32), P(C.c_int32), P(C.c_int32), P(Tally)]
    L.ldpc_decode_llr_bf16.argtypes = [C.c_void_p, P(RunParams), P(C.c_uint16), C.c_int64, P(C.c_float),
                                       P(C.c_int32), P(C.c_int32), P(C.c_int32), P(Tally)]
    L.ldpc_channel_llr.argtypes = [C.c_void_p, P(RunParams), P(C.c_float)]
    L.ldpc_iter_histogram.argtypes = [C.c_void_p, P(C.c_uint64), C.c_int]
    L.ldpc_snr_bins.argtypes = [C.c_void_p, P(C.c_uint64)]
    L.ldpc_batch_create.argtypes = [P(C.c_void_p), C.c_int, P(C.c_void_p)]
    L.ldpc_batch_destroy.argtypes = [C.c_void_p]
    L.ldpc_batch_destroy.restype = None
    L.ldpc_batch_run.argtypes = [C.c_void_p, P(RunParams), P(C.c_float), P(Tally), P(C.c_float)]
    L.ldpc_batch_graph_builds.argtypes = [C.c_void_p]
    L.ldpc_batch_graph_builds.restype = C.c_int64
    L.ldpc_batch_set_order.argtypes = [C.c_void_p, C.c_int]
    L.ldpc_step_schedule.argtypes = [C.POINTER(Matrix), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32)]
    L.ldpc_set_launch_shape.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.ldpc_list_shapes.argtypes = [C.c_void_p, C.c_int, P(C.c_int32), C.c_int]
    L.ldpc_list_shapes_algo.argtypes = [C.c_void_p, C.c_int, C.c_int, P(C.c_int32), C.c_int]
    L.ldpc_set_weights.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float), C.c_int, C.c_int, P(C.c_int32)]
    L.ldpc_set_circulant.argtypes = [C.c_void_p, P(CircConfig)]
    L.ldpc_channel_llr_device.argtypes = [C.c_void_p, P(RunParams), C.c_void_p, C.c_void_p]
    L.ldpc_wdec_workspace_bytes.argtypes = [C.c_void_p, P(WdecConfig), C.c_int64]
    L.ldpc_wdec_workspace_bytes.restype = C.c_int64
    L.ldpc_wdec_forward.argtypes = [C.c_void_p, P(WdecConfig), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    L.ldpc_wdec_backward.argtypes = [C.c_void_p, P(WdecConfig), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ldpc_launch_count.argtypes = [C.c_void_p]
    L.ldpc_launch_count.restype = C.c_int64
    L.ldpc_launch_param_bytes.argtypes = [C.c_void_p]
    L.ldpc_launch_param_bytes.restype = C.c_int64
    L.ldpc_decode_llr_static.argtypes = [P(Matrix), P(RunParams), C.c_void_p, C.c_int64, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p, P(Tally), C.c_void_p]
    L.ldpc_row_schedule.argtypes = [P(Matrix), P(C.c_int32), P(C.c_int32)]
    L.ldpc_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.ldpc_abi_version.argtypes = []
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().ldpc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def _check(rc: int):
    if rc < 0:
        raise LdpcError(rc, last_error())
    return rc


def channel_mu_sigma(N: int, M: int, P: int, ebn0_db: float):
    """mu = 4 R Eb/N0, sigma = sqrt(8 R Eb/N0) with R = (N-M)/(N-P), computed in double and rounded to
    float (engines/scalar_5w/ldpc_sim_scalar.cpp:351-355)."""
    rate = (N - M) / (N - P)
    snr = 10.0 ** (ebn0_db / 10.0)
    return float(np.float32(4.0 * rate * snr)), float(np.float32(math.sqrt(8.0 * rate * snr)))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


STATIC_SCRATCH_BYTES = 16 << 20


def decode_llr_static(rows: np.ndarray, n_vars: int, n_punct: int, p: RunParams, d_llr: int, n_frames: int,
                      d_post: int = 0, d_iters: int = 0, d_synd_fail: int = 0, d_bit_errors: int = 0,
                      stream: int = 0) -> "ChunkResult":
    """ldpc_decode_llr_static: decode frames whose LLRs are already in device memory into device
    buffers (addresses as integers), with no allocation by the library.  The caller owns every
    buffer; the library's scratch is a fixed static device array shared by all calls."""
    lib = load()
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    m = Matrix(int(n_vars), rows.shape[0], int(n_punct), rows.shape[1], _ip(rows))
    t = Tally()
    _check(lib.ldpc_decode_llr_static(C.byref(m), C.byref(p), d_llr or None, int(n_frames), d_post or None,
                                      d_iters or None, d_synd_fail or None, d_bit_errors or None, C.byref(t),
                                      stream or None))
    return ChunkResult(t.frames, t.bit_errors, t.frame_errors, t.iter_sum, t.unconverged, t.max_iters,
                       t.kernel_ms, t.bit_errors_sq)


def row_schedule(rows: np.ndarray, n_vars: int):
    """ldpc_row_schedule (host only, no GPU): the general kernel's row schedule of a [M, dmax] row
    table.  Returns (order, starts): the file rows in schedule order and the first position of every
    step followed by M."""
    lib = load()
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    M = rows.shape[0]
    m = Matrix(int(n_vars), M, 0, rows.shape[1], _ip(rows))
    order = np.zeros(M, np.int32)
    starts = np.zeros(M + 1, np.int32)
    n = _check(lib.ldpc_row_schedule(C.byref(m), _ip(order), _ip(starts)))
    return order, starts[:n + 1].copy()


def step_schedule(rows: np.ndarray, n_vars: int):
    """ldpc_step_schedule (host only, no GPU): the step kernel's schedule of a [M, dmax] row table,
    steps of one degree class.  Returns (order, starts, low): low[s] = 1 for a step of low-degree rows."""
    lib = load()
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    M = rows.shape[0]
    m = Matrix(int(n_vars), M, 0, rows.shape[1], _ip(rows))
    order = np.zeros(M, np.int32)
    starts = np.zeros(M + 1, np.int32)
    low = np.zeros(M, np.int32)
    n = _check(lib.ldpc_step_schedule(C.byref(m), _ip(order), _ip(starts), _ip(low)))
    return order, starts[:n + 1].copy(), low[:n].copy()


@dataclass
class ChunkResult:
    frames: int
    bit_errors: int
    frame_errors: int
    iter_sum: int
    unconverged: int
    max_iters: int
    kernel_ms: float
    bit_errors_sq: int = 0


class Decoder:
    """One parity-check matrix on one GPU.  ``rows``: [M, dmax] int32, 0-based columns in file order,
    -1 padded; the last ``n_punct`` of the ``n_vars`` columns are punctured."""

    def __init__(self, rows: np.ndarray, n_vars: int, n_punct: int, device: int = -1):
        self._lib = load()
        self.rows = np.ascontiguousarray(rows, dtype=np.int32)
        self.M, self.dmax = self.rows.shape
        self.N, self.P = int(n_vars), int(n_punct)
        self.n_tx = self.N - self.P
        m = Matrix(self.N, self.M, self.P, self.dmax, _ip(self.rows))
        h = C.c_void_p()
        _check(self._lib.ldpc_create(C.byref(m), device, C.byref(h)))
        self._h = h

    @classmethod
    def from_code(cls, code, device: int = -1) -> "Decoder":
        """From an ``ar4ja.QcCode`` (makeH order) or a ``chinn.Matrix`` plus punctured count."""
        return cls(code.row_matrix(), code.N, code.P, device)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ldpc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def kind(self) -> int:
        return _check(self._lib.ldpc_kernel_kind(self._h))

    @property
    def launches(self) -> int:
        return int(self._lib.ldpc_launch_count(self._h))

    @property
    def launch_param_bytes(self) -> int:
        return _check(int(self._lib.ldpc_launch_param_bytes(self._h)))

    def set_launch_shape(self, rows_per_thread: int = 0, frames_per_cta: int = 0, min_ctas_per_sm: int = 0,
                         global_messages: int = 0, storage=-1):
        if isinstance(storage, str):
            storage = STORAGE_NAMES[storage]
        _check(self._lib.ldpc_set_launch_shape(self._h, storage, rows_per_thread, frames_per_cta, min_ctas_per_sm,
                                               global_messages))

    def shapes(self, storage, algo: int = ALGO_AMIN) -> list:
        """Built launch shapes (rows per thread, frames per CTA, min CTAs per SM, layout) for a
        storage mode and algorithm: the QC kernel's, or for a general matrix the step kernel's
        (layout 3; third entry = resident CTAs per SM, 0 = as many as fit) and the warp kernel's
        (layout 4)."""
        if isinstance(storage, str):
            storage = STORAGE_NAMES[storage]
        buf = np.zeros(4 * 64, np.int32)
        n = _check(self._lib.ldpc_list_shapes_algo(self._h, storage, algo, _ip(buf), 64))
        return [tuple(int(x) for x in buf[4 * i:4 * i + 4]) for i in range(min(n, 64))]

    def autotune(self, mu: float, sigma: float, storages=("fp32", "fp16", "bf16"), frames: int = 1 << 18,
                 max_iter: int = 200, seed: int = 0x5EED, repeats: int = 2, algo: int = ALGO_AMIN):
        """Times every built launch shape of each storage mode on ``frames`` frames of this channel
        and keeps the fastest per mode.  Returns {storage: (best shape, {shape: Mframes/s})} and the
        fastest storage overall."""
        out = {}
        best_overall = None
        for st in storages:
            shapes = self.shapes(st, algo)
            timings = {}
            for sh in shapes:
                self.set_launch_shape(*sh, storage=st)
                p = self.params(mu=mu, sigma=sigma, seed=seed, n_frames=frames, max_iter=max_iter, storage=st,
                                algo=algo)
                self.run_chunk(p)  # warm-up
                ms = min(self.run_chunk(p).kernel_ms for _ in range(repeats))
                timings[sh] = frames / (ms * 1e-3) / 1e6
            if timings:
                best = max(timings, key=timings.get)
                self.set_launch_shape(*best, storage=st)
                out[st] = (best, timings)
                if best_overall is None or timings[best] > out[best_overall][1][out[best_overall][0]]:
                    best_overall = st
        return out, best_overall

    @staticmethod
    def params(mu=0.0, sigma=0.0, seed=1, stream=0, first_frame=0, n_frames=0, max_iter=200,
               storage=STORE_BF16, algo=ALGO_AMIN, l_max=0.0, r_max=0.0, l_post_max=0.0,
               ebn0_lo=0.0, ebn0_hi=0.0) -> RunParams:
        """Run parameters; ebn0_hi > ebn0_lo draws each frame's Eb/N0 uniformly in [lo, hi) dB."""
        if isinstance(storage, str):
            storage = STORAGE_NAMES[storage]
        return RunParams(mu, sigma, seed, stream, 0, first_frame, n_frames, max_iter, storage, algo,
                         l_max, r_max, l_post_max, ebn0_lo, ebn0_hi)

    def snr_bins(self) -> np.ndarray:
        """[4, SNR_BINS] frames, frame errors, bit errors, iterations per Eb/N0 bin of the last run."""
        out = np.zeros(4 * SNR_BINS, np.uint64)
        _check(self._lib.ldpc_snr_bins(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out.reshape(4, SNR_BINS)

    def run_chunk(self, p: RunParams) -> ChunkResult:
        t = Tally()
        _check(self._lib.ldpc_run_chunk(self._h, C.byref(p), C.byref(t)))
        return ChunkResult(t.frames, t.bit_errors, t.frame_errors, t.iter_sum, t.unconverged,
                           t.max_iters, t.kernel_ms, t.bit_errors_sq)

    def decode_llr(self, llr: np.ndarray, p: Optional[RunParams] = None, want_post: bool = True, **kw):
        """Decode caller-supplied channel LLRs [n, N-P]: fp32, or uint16 arrays holding bf16 bit
        patterns (ldpc_decode_llr_bf16).  Returns (post [n, N] or None, iters, synd_fail, bit_errors,
        ChunkResult)."""
        if p is None:
            p = self.params(**kw)
        bf16 = isinstance(llr, np.ndarray) and llr.dtype == np.uint16
        llr = np.ascontiguousarray(np.atleast_2d(llr), dtype=np.uint16 if bf16 else np.float32)
        if llr.shape[1] != self.n_tx:
            raise ValueError(f"llr has {llr.shape[1]} columns, expected N-P = {self.n_tx}")
        n = llr.shape[0]
        post = np.empty((n, self.N), np.float32) if want_post else None
        it = np.empty(n, np.int32)
        sf = np.empty(n, np.int32)
        be = np.empty(n, np.int32)
        t = Tally()
        if bf16:
            _check(self._lib.ldpc_decode_llr_bf16(self._h, C.byref(p), llr.ctypes.data_as(C.POINTER(C.c_uint16)),
                                                  n, _fp(post), _ip(it), _ip(sf), _ip(be), C.byref(t)))
        else:
            _check(self._lib.ldpc_decode_llr(self._h, C.byref(p), _fp(llr), n, _fp(post), _ip(it), _ip(sf),
                                             _ip(be), C.byref(t)))
        return post, it, sf, be, ChunkResult(t.frames, t.bit_errors, t.frame_errors, t.iter_sum,
                                             t.unconverged, t.max_iters, t.kernel_ms, t.bit_errors_sq)

    def channel_llr(self, p: RunParams) -> np.ndarray:
        out = np.empty((int(p.n_frames), self.n_tx), np.float32)
        _check(self._lib.ldpc_channel_llr(self._h, C.byref(p), _fp(out)))
        return out

    def channel_llr_device(self, p: RunParams, d_llr: int, stream: int = 0):
        """ldpc_channel_llr into a device array (address as an integer) on a CUDA stream (handle as
        an integer; 0 = the legacy default stream), without waiting."""
        _check(self._lib.ldpc_channel_llr_device(self._h, C.byref(p), d_llr or None, stream or None))

    def set_weights(self, alpha: np.ndarray, beta: np.ndarray, edge_class: np.ndarray):
        """Weights of ALGO_WAMIN runs: alpha/beta [T][C] (iterations past T use row T-1),
        edge_class [12][18]."""
        a = np.ascontiguousarray(alpha, dtype=np.float32)
        b = np.ascontiguousarray(beta, dtype=np.float32)
        ec = np.ascontiguousarray(edge_class, dtype=np.int32)
        if a.ndim != 2 or a.shape != b.shape or ec.shape != (12, 18):
            raise ValueError("alpha/beta must be [T][C] and edge_class [12][18]")
        _check(self._lib.ldpc_set_weights(self._h, _fp(a), _fp(b), a.shape[0], a.shape[1], _ip(ec)))

    def clear_weights(self):
        _check(self._lib.ldpc_set_weights(self._h, None, None, 0, 0, None))

    def set_circulant(self, numerics: int = CIRC_SFPU, stop: int = CIRC_STOP_GENIE, damping: float = 0.9375):
        """Settings of ALGO_CIRC runs: the circulant engine's arithmetic form (CIRC_SFPU: its device
        kernels; CIRC_SCALAR: its stepper's scalar path, damping 1), stop rule (CIRC_STOP_GENIE: the
        engine on silicon; CIRC_STOP_SYNDROME: the stepper's Monte Carlo loop) and damping factor."""
        _check(self._lib.ldpc_set_circulant(self._h, C.byref(CircConfig(numerics, stop, damping, 0))))

    def iter_histogram(self, n_bins: int = 256) -> np.ndarray:
        h = np.zeros(n_bins, np.uint64)
        _check(self._lib.ldpc_iter_histogram(self._h, h.ctypes.data_as(C.POINTER(C.c_uint64)), n_bins))
        return h


BATCH_SIDE_BY_SIDE, BATCH_IN_TURN, BATCH_GLOBAL_IN_TURN = 0, 1, 2
BATCH_ORDERS = {"side-by-side": BATCH_SIDE_BY_SIDE, "in-turn": BATCH_IN_TURN, "global-in-turn": BATCH_GLOBAL_IN_TURN}


class Batch:
    """Several decoders (codes) on one GPU run by one CUDA graph launch of their persistent kernels
    (ldpc_batch_* in include/ldpcb200.h); ``order`` says which kernels wait for one another."""

    def __init__(self, decoders):
        self._lib = load()
        self.decoders = list(decoders)
        arr = (C.c_void_p * len(self.decoders))(*[d._h for d in self.decoders])
        b = C.c_void_p()
        _check(self._lib.ldpc_batch_create(arr, len(self.decoders), C.byref(b)))
        self._b = b

    def run(self, params, share=None):
        """params: one RunParams per decoder; share: relative CTA shares (None = frames x checks).
        Returns (list of ChunkResult, graph milliseconds)."""
        n = len(self.decoders)
        P = (RunParams * n)(*params)
        T = (Tally * n)()
        S = (C.c_float * n)(*share) if share is not None else None
        ms = C.c_float()
        _check(self._lib.ldpc_batch_run(self._b, P, S, T, C.byref(ms)))
        res = [ChunkResult(t.frames, t.bit_errors, t.frame_errors, t.iter_sum, t.unconverged, t.max_iters,
                           t.kernel_ms, t.bit_errors_sq) for t in T]
        return res, ms.value

    def set_order(self, order):
        """BATCH_SIDE_BY_SIDE, BATCH_IN_TURN or BATCH_GLOBAL_IN_TURN (or its name)."""
        if isinstance(order, str):
            order = BATCH_ORDERS[order]
        _check(self._lib.ldpc_batch_set_order(self._b, int(order)))

    @property
    def graph_builds(self) -> int:
        """How many times the batch built its CUDA graph (once, unless a call changed a kernel)."""
        return int(self._lib.ldpc_batch_graph_builds(self._b))

    def close(self):
        if getattr(self, "_b", None):
            self._lib.ldpc_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
