"""CPU checkers for the mode-q tensor-times-matrix product.

TEST INFRASTRUCTURE ONLY. ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` import this package, always as
the checker or as the timed CPU baseline, never as the thing measured on the
GPU and never from the product package ``ttm_b200``.

Two checkers live here:

* ``Oracle`` — ctypes binding of ``oracle/ttm_oracle.c``, a plain-C
  restatement of the reference algorithm (long-double / double accumulation).
* ``Reference`` — ctypes binding of ``oracle/_ref/libtlibttm_ref.so``, the
  reference tlib::ttm headers themselves compiled against OpenBLAS by
  ``oracle/Makefile``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libttm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtlibttm_ref.so")

_SZ = C.POINTER(C.c_size_t)

# Policy ids exported by oracle/ref_shim.cpp, in its enum order.
REF_POLICIES = [
    "combined", "sequential/slice/none", "sequential/subtensor/none",
    "parallel_blas/slice/none", "parallel_blas/subtensor/none",
    "parallel_blas/slice/all", "parallel_blas/subtensor/all",
    "parallel_loop/slice/outer", "parallel_loop/slice/all",
    "parallel_loop/subtensor/all", "parallel_loop_blas/slice/all",
    "parallel_loop_blas/subtensor/all", "parallel_taskloop/slice/none",
    "parallel_taskloop/subtensor/none", "parallel_task/slice/none",
    "parallel_task/subtensor/none",
]


EXAMPLES_DIR = os.path.join(HERE, "_ref", "examples")


def build(ref: bool = True, ref_root: str | None = None) -> None:
    """Build the checkers with oracle/Makefile.

    With ``ref``, also the reference build and its example programs, from the reference checkout
    ``ref_root`` (default: the environment variable TLIBTTM_REF_ROOT); without one, prebuilt
    copies under oracle/_ref are kept."""
    targets = ["oracle", "ref", "examples"] if ref else ["oracle"]
    root = ref_root if ref_root is not None else os.environ.get("TLIBTTM_REF_ROOT", "")
    subprocess.run(["make", "-s", "-C", HERE] + targets + ([f"REF_ROOT={root}"] if root else []), check=True)


def _sz(v):
    arr = (C.c_size_t * max(len(v), 1))(*[int(x) for x in v])
    return arr


def _ptr(x):
    return x.ctypes.data_as(C.c_void_p) if x is not None else None


def dense_strides(n, pi):
    """Dense strides of shape n under one-based layout pi (no vector special case)."""
    p = len(n)
    w = [1] * p
    for r in range(1, p):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


class Oracle:
    """The C restatement (oracle/ttm_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        self.lib = C.CDLL(path)
        L = self.lib
        for name in ("oracle_ttm_f32", "oracle_ttm_f64"):
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = [C.c_uint, C.c_uint, C.c_void_p, _SZ, _SZ, _SZ, C.c_void_p, _SZ, _SZ,
                          C.c_void_p, _SZ, _SZ]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_case.restype = C.c_int
        L.oracle_case.argtypes = [C.c_uint, C.c_size_t, _SZ]
        L.oracle_fibres.restype = C.c_int
        L.oracle_fibres.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_void_p, _SZ, _SZ, _SZ,
                                    C.c_void_p, _SZ, _SZ, _SZ, _SZ, _SZ, C.c_size_t, C.c_void_p]

    def ttm(self, q, a_flat, na, wa, pia, b_flat, nb, pib, c_flat, nc, wc):
        """Low-level call on flat numpy buffers; raises RuntimeError with the reference text."""
        f = self.lib.oracle_ttm_f64 if a_flat.dtype == np.float64 else self.lib.oracle_ttm_f32
        p = len(na)
        rc = f(q, p, _ptr(a_flat), _sz(na), _sz(wa), _sz(pia), _ptr(b_flat), _sz(nb),
               _sz(pib) if pib is not None else None, _ptr(c_flat), _sz(nc), _sz(wc))
        if rc:
            raise RuntimeError(self.lib.oracle_last_error().decode())

    def case(self, p, q, pi):
        return self.lib.oracle_case(p, q, _sz(pi))

    def fibres(self, q, a_flat, na, wa, pia, b_flat, nb, pib, wc, fk, fi):
        fk = np.ascontiguousarray(fk, dtype=np.uint64)
        fi = np.ascontiguousarray(fi, dtype=np.uint64)
        out = np.empty((len(fk), nb[0]), dtype=np.float64)
        dt = 1 if a_flat.dtype == np.float64 else 0
        self.lib.oracle_fibres(dt, q, len(na), _ptr(a_flat), _sz(na), _sz(wa), _sz(pia),
                               _ptr(b_flat), _sz(nb), _sz(pib), _sz(wc),
                               fk.ctypes.data_as(_SZ), fi.ctypes.data_as(_SZ), len(fk),
                               _ptr(out))
        return out


class Reference:
    """The reference tlib::ttm compiled with OpenBLAS (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            build(ref=True)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        for name in ("tlibref_ttm_f32", "tlibref_ttm_f64"):
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_void_p, _SZ, _SZ, _SZ, C.c_void_p,
                          _SZ, _SZ, C.c_void_p, _SZ, _SZ, C.c_char_p, C.c_size_t]
        L.tlibref_cores.restype = C.c_uint
        L.tlibref_compute_k_order_layout.argtypes = [_SZ, C.c_size_t, C.c_size_t]
        L.tlibref_is_valid_layout.argtypes = [_SZ, C.c_size_t]
        L.tlibref_inverse_mode.argtypes = [_SZ, C.c_size_t, C.c_size_t, _SZ]
        L.tlibref_compute_strides.argtypes = [_SZ, C.c_size_t, _SZ, _SZ]
        L.tlibref_is_valid_strides.argtypes = [_SZ, C.c_size_t, _SZ]
        L.tlibref_shape_kind.argtypes = [_SZ, C.c_size_t]
        L.tlibref_is_case.argtypes = [C.c_uint, C.c_uint, C.c_size_t, _SZ]

    @property
    def cores(self) -> int:
        return int(self.lib.tlibref_cores())

    def ttm(self, q, a_flat, na, wa, pia, b_flat, nb, pib, c_flat, nc, wc, policy=0):
        f = self.lib.tlibref_ttm_f64 if a_flat.dtype == np.float64 else self.lib.tlibref_ttm_f32
        err = C.create_string_buffer(512)
        rc = f(policy, q, len(na), _ptr(a_flat), _sz(na), _sz(wa), _sz(pia), _ptr(b_flat),
               _sz(nb), _sz(pib), _ptr(c_flat), _sz(nc), _sz(wc), err, 512)
        if rc:
            raise RuntimeError(err.value.decode())

    # reference helpers (include/tlib/detail/{layout,shape,strides,cases}.h)
    def k_order_layout(self, p, k):
        v = (C.c_size_t * p)()
        if self.lib.tlibref_compute_k_order_layout(v, p, k) < 0:
            raise RuntimeError("compute_k_order_layout threw")
        return list(v)

    def is_valid_layout(self, pi):
        return bool(self.lib.tlibref_is_valid_layout(_sz(pi), len(pi)))

    def inverse_mode(self, pi, mode):
        out = (C.c_size_t * 1)()
        if self.lib.tlibref_inverse_mode(_sz(pi), len(pi), mode, out) < 0:
            raise RuntimeError("inverse_mode threw")
        return int(out[0])

    def strides(self, n, pi):
        out = (C.c_size_t * len(n))()
        if self.lib.tlibref_compute_strides(_sz(n), len(n), _sz(pi), out) < 0:
            raise RuntimeError("compute_strides threw")
        return list(out)

    def is_valid_strides(self, pi, w):
        r = self.lib.tlibref_is_valid_strides(_sz(pi), len(pi), _sz(w))
        if r < 0:
            raise RuntimeError("is_valid_strides threw")
        return bool(r)

    def shape_kind(self, n):
        return int(self.lib.tlibref_shape_kind(_sz(n), len(n)))

    def is_case(self, case_nr, p, q, pi):
        return bool(self.lib.tlibref_is_case(case_nr, p, q, _sz(pi)))
