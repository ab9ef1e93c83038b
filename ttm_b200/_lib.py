"""ctypes binding of the C ABI in include/tlibttm.h (libtlibttm_cuda.so).

The library is the only compute path: if it is missing or cannot be loaded
this module raises ImportError — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtlibttm_cuda.so")

OK, ERR_ARG, ERR_CUDA, ERR_ALLOC, ERR_UNSUPPORTED, ERR_DEVICE = range(6)
F32, F64 = 0, 1
PREC_DEFAULT, PREC_PLAIN, PREC_BF16X3, PREC_FP8, PREC_OZAKI, PREC_AUTO = range(6)
INJECT_NONE, INJECT_FAIL_ALLOC, INJECT_WAIT_NS, INJECT_SKIP_B_STAGE = range(4)
PRECISIONS = {"default": PREC_DEFAULT, "plain": PREC_PLAIN, "bf16x3": PREC_BF16X3, "fp8": PREC_FP8,
              "ozaki": PREC_OZAKI, "auto": PREC_AUTO}

_SZ = C.POINTER(C.c_size_t)
_lock = threading.Lock()
_lib = None


class TtmError(RuntimeError):
    """Raised for a non-zero status of the C ABI; `.code` holds the status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def _declare(L):
    sig = [C.c_uint, C.c_uint, C.c_void_p, _SZ, _SZ, _SZ, C.c_void_p, _SZ, _SZ, C.c_void_p, _SZ, _SZ,
           C.c_void_p]
    for name in ("tlibttm_ttm_f32", "tlibttm_ttm_f64"):
        f = getattr(L, name)
        f.restype = C.c_int
        f.argtypes = sig
    L.tlibttm_ttm_ex.restype = C.c_int
    L.tlibttm_ttm_ex.argtypes = [C.c_int, C.c_int] + sig
    L.tlibttm_ttm_f32_bf16x3_noalloc.restype = C.c_int
    L.tlibttm_ttm_f32_bf16x3_noalloc.argtypes = sig
    L.tlibttm_last_error.restype = C.c_char_p
    L.tlibttm_last_kernel.restype = C.c_char_p
    L.tlibttm_set_precision.restype = C.c_int
    L.tlibttm_set_precision.argtypes = [C.c_int]
    L.tlibttm_get_precision.restype = C.c_int
    L.tlibttm_launch_count.restype = C.c_ulonglong
    L.tlibttm_launch_count.argtypes = [C.c_int]
    L.tlibttm_synchronize.restype = C.c_int
    L.tlibttm_synchronize.argtypes = [C.c_void_p]
    L.tlibttm_release_buffers.restype = C.c_int
    L.tlibttm_k_order_layout.restype = C.c_int
    L.tlibttm_k_order_layout.argtypes = [_SZ, C.c_size_t, C.c_size_t]
    L.tlibttm_inverse_mode.restype = C.c_size_t
    L.tlibttm_inverse_mode.argtypes = [_SZ, C.c_size_t, C.c_size_t]
    L.tlibttm_strides.restype = C.c_int
    L.tlibttm_strides.argtypes = [_SZ, C.c_size_t, _SZ, _SZ]
    L.tlibttm_inject.restype = C.c_int
    L.tlibttm_inject.argtypes = [C.c_int, C.c_longlong]


def lib():
    """The loaded library (built on first use if its sources are present)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                try:
                    from . import build as _build
                    _build.build()
                except Exception as e:  # noqa: BLE001 - surface the build failure loudly
                    raise ImportError(f"libtlibttm_cuda.so is missing and could not be built: {e}") from e
            try:
                L = C.CDLL(LIB_PATH)
            except OSError as e:
                raise ImportError(f"cannot load {LIB_PATH}: {e}") from e
            _declare(L)
            _lib = L
    return _lib


def sz(v):
    """A C size_t[] holding the integers of v."""
    v = [int(x) for x in v]
    return (C.c_size_t * max(len(v), 1))(*v)


def check(rc: int):
    if rc != OK:
        raise TtmError(rc, lib().tlibttm_last_error().decode())


def ttm_raw(dtype: int, precision: int, q: int, p: int, a_ptr: int, na, wa, pia, b_ptr: int, nb, pib,
            c_ptr: int, nc, wc, stream: int = 0):
    """One call of tlibttm_ttm_ex with raw addresses (host or device) and host metadata."""
    L = lib()
    rc = L.tlibttm_ttm_ex(dtype, precision, q, p, C.c_void_p(a_ptr), sz(na), sz(wa), sz(pia),
                          C.c_void_p(b_ptr), sz(nb), sz(pib) if pib is not None else None,
                          C.c_void_p(c_ptr), sz(nc), sz(wc), C.c_void_p(stream))
    check(rc)


def last_kernel() -> str:
    return lib().tlibttm_last_kernel().decode()


def launch_count(reset: bool = False) -> int:
    return int(lib().tlibttm_launch_count(1 if reset else 0))


def set_precision(name_or_id) -> int:
    pid = PRECISIONS[name_or_id] if isinstance(name_or_id, str) else int(name_or_id)
    return int(lib().tlibttm_set_precision(pid))


def get_precision() -> int:
    return int(lib().tlibttm_get_precision())


def k_order_layout(p: int, k: int):
    buf = (C.c_size_t * p)()
    check(lib().tlibttm_k_order_layout(buf, p, k))
    return list(buf)


def inverse_mode(layout, mode: int) -> int:
    r = int(lib().tlibttm_inverse_mode(sz(layout), len(layout), mode))
    if r == 0:
        raise RuntimeError(lib().tlibttm_last_error().decode())
    return r


def strides(shape, layout):
    out = (C.c_size_t * len(shape))()
    check(lib().tlibttm_strides(sz(shape), len(shape), sz(layout), out))
    return list(out)


def inject(what: int, arg: int = 0) -> None:
    """Host-side fault injection for failure-detection tests (tlibttm_inject)."""
    check(lib().tlibttm_inject(int(what), int(arg)))
