"""The C ABI library without a GPU: it loads, exports every entry point include/ldpcb200.h
declares, and refuses politely when no device is present (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO, has_gpu
from ldpcb200 import capi

HEADER = os.path.join(REPO, "include", "ldpcb200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|int64_t)\s+(ldpc_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    assert sorted(capi.EXPORTS) == declared_functions()


def test_library_exports_every_symbol():
    lib = capi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.ldpc_abi_version() == 1


def test_struct_layouts():
    # sizes the C side uses (include/ldpcb200.h); a mismatch would corrupt every call
    assert C.sizeof(capi.Matrix) == 24
    assert C.sizeof(capi.RunParams) == 72
    assert C.sizeof(capi.Tally) == 64
    assert C.sizeof(capi.WdecConfig) == 6 * 4 + 12 * 18 * 4
    assert C.sizeof(capi.CircConfig) == 16


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    rows = np.array([[0, 1], [1, 2]], np.int32)
    with pytest.raises(capi.LdpcError) as e:
        capi.Decoder(rows, 3, 0)
    assert e.value.code in (-19, -5)
    assert capi.last_error()


def test_bad_arguments_are_rejected_before_any_device_work():
    lib = capi.load()
    h = C.c_void_p()
    assert lib.ldpc_create(None, 0, C.byref(h)) == -22
    rows = np.array([[0, 5]], np.int32)  # column 5 outside N = 3
    m = capi.Matrix(3, 1, 0, 2, rows.ctypes.data_as(C.POINTER(C.c_int32)))
    assert lib.ldpc_create(C.byref(m), 0, C.byref(h)) == -22
    assert "out of bounds" in capi.last_error()
    m = capi.Matrix(3, 1, 3, 2, rows.ctypes.data_as(C.POINTER(C.c_int32)))
    assert lib.ldpc_create(C.byref(m), 0, C.byref(h)) == -22
    holed = np.array([[0, -1, 2]], np.int32)  # an edge after the -1 that ends the row
    m = capi.Matrix(3, 1, 0, 3, holed.ctypes.data_as(C.POINTER(C.c_int32)))
    assert lib.ldpc_create(C.byref(m), 0, C.byref(h)) == -22
    assert "ends the row" in capi.last_error()
    with pytest.raises(capi.LdpcError):
        capi.row_schedule(holed, 3)
    with pytest.raises(capi.LdpcError):
        capi.decode_llr_static(holed, 3, 0, capi.RunParams(), 0, 0)
    t = capi.Tally()
    assert lib.ldpc_run_chunk(None, None, C.byref(t)) == -22
    assert lib.ldpc_set_circulant(None, C.byref(capi.CircConfig(1, 1, 0.9375, 0))) == -22
