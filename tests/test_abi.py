"""The C ABI (include/tlibttm.h) without a GPU: the library loads, exports every
declared entry point, and rejects bad arguments with the reference's texts."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from ttm_b200 import _lib
from test_oracle import bad_argument_sets

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in ("tlibttm.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        names |= set(re.findall(r"\b(tlibttm_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 12
    for name in syms:
        assert hasattr(L, name), name


def _abi_call(args, dtype=np.float64):
    q, p, a, na, wa, pia, b, nb, pib, c, nc, wc = args
    # Pointers are never dereferenced: the checks run before any device work.
    _lib.ttm_raw(_lib.F64 if dtype == np.float64 else _lib.F32, _lib.PREC_DEFAULT, q, p if p else 0,
                 a.ctypes.data, na, wa, pia, b.ctypes.data, nb, pib, c.ctypes.data, nc, wc)


def test_argument_errors_match_reference_texts(oracle_c):
    for args in bad_argument_sets():
        q, p, a, na, wa, pia, b, nb, pib, c, nc, wc = args
        with pytest.raises(RuntimeError) as e_ref:
            oracle_c.ttm(q, a, na, wa, pia, b, nb, pib, c, nc, wc)
        with pytest.raises(_lib.TtmError) as e_abi:
            _abi_call(args)
        assert str(e_abi.value) == str(e_ref.value)
        assert e_abi.value.code == _lib.ERR_ARG


def test_null_pointer_errors():
    L = _lib.lib()
    na = _lib.sz([2, 3])
    rc = L.tlibttm_ttm_f32(1, 2, None, na, na, _lib.sz([1, 2]), C.c_void_p(8), _lib.sz([2, 2]),
                           _lib.sz([1, 2]), C.c_void_p(16), na, na, None)
    assert rc == _lib.ERR_ARG
    assert L.tlibttm_last_error().decode() == \
        "Error in tlib::tensor_times_matrix: pointer to input tensor A should not be zero."
    rc = L.tlibttm_ttm_f32(1, 0, C.c_void_p(8), na, na, _lib.sz([1, 2]), C.c_void_p(8), _lib.sz([2, 2]),
                           _lib.sz([1, 2]), C.c_void_p(16), na, na, None)
    assert L.tlibttm_last_error().decode() == \
        "Error in tlib::tensor_times_matrix: input tensor order should be greater zero."
    # pib is dereferenced by the reference without a check; here it is an argument error.
    rc = L.tlibttm_ttm_f32(1, 2, C.c_void_p(8), na, _lib.sz([1, 2]), _lib.sz([1, 2]), C.c_void_p(8),
                           _lib.sz([2, 2]), None, C.c_void_p(16), na, _lib.sz([1, 2]), None)
    assert rc == _lib.ERR_ARG and "pib" in L.tlibttm_last_error().decode()


def test_c_extent_mismatch_is_an_error():
    a = np.zeros(24)
    with pytest.raises(_lib.TtmError, match="does not match A outside the contraction mode"):
        _lib.ttm_raw(_lib.F64, 0, 1, 3, a.ctypes.data, [2, 3, 4], [1, 2, 6], [1, 2, 3], a.ctypes.data,
                     [2, 2], [1, 2], a.ctypes.data, [2, 3, 5], [1, 2, 6])


def test_unknown_dtype_and_precision():
    a = np.zeros(4)
    with pytest.raises(_lib.TtmError):
        _lib.ttm_raw(7, 0, 1, 1, a.ctypes.data, [2], [1], [1], a.ctypes.data, [2, 2], [1, 2],
                     a.ctypes.data, [2], [1])
    with pytest.raises(_lib.TtmError):
        _lib.ttm_raw(0, 99, 1, 1, a.ctypes.data, [2], [1], [1], a.ctypes.data, [2, 2], [1, 2],
                     a.ctypes.data, [2], [1])


def test_precision_setting_roundtrip():
    old = _lib.set_precision("bf16x3")
    try:
        assert _lib.get_precision() == _lib.PREC_BF16X3
    finally:
        _lib.set_precision(old)
    assert _lib.lib().tlibttm_set_precision(42) == -1


def test_batched_plan_options_are_checked():
    """tlibttm_plan_batched_ex rejects a null plan pointer and unknown option bits before any
    device work."""
    L = _lib.lib()
    L.tlibttm_plan_batched_ex.restype = C.c_int
    L.tlibttm_plan_batched_ex.argtypes = [C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_uint, C.c_void_p]
    h = C.c_void_p(1)
    assert L.tlibttm_plan_batched_ex(_lib.F32, _lib.PREC_DEFAULT, 0, None, 0, None) == _lib.ERR_ARG
    assert "plan pointer is null" in L.tlibttm_last_error().decode()
    assert L.tlibttm_plan_batched_ex(_lib.F32, _lib.PREC_DEFAULT, 0, None, 2, C.byref(h)) == _lib.ERR_ARG
    assert "unknown flags" in L.tlibttm_last_error().decode()
    assert not h.value                      # the plan pointer is cleared on error
