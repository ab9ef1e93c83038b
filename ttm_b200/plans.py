"""Plans over the C ABI: many TTMs prepared once and run many times.

* ``BatchPlan``  — independent TTMs in one persistent grouped launch (device work queue);
* ``ChainPlan``  — a Tucker chain ``A x_{r1} B_1 x_{r2} B_2 ...`` with intermediates kept on the GPU;
* both can run as a captured CUDA graph (``run_graph``).

Operands are torch CUDA tensors (device memory is required); the plans keep references to them,
so running a plan again reads the tensors' current contents.
"""
from __future__ import annotations

import ctypes as C

from . import _lib

try:
    import torch
except Exception:  # noqa: BLE001
    torch = None


class _Problem(C.Structure):
    _fields_ = [("q", C.c_uint), ("p", C.c_uint),
                ("a", C.c_void_p), ("na", C.POINTER(C.c_size_t)), ("wa", C.POINTER(C.c_size_t)),
                ("pia", C.POINTER(C.c_size_t)),
                ("b", C.c_void_p), ("nb", C.POINTER(C.c_size_t)), ("pib", C.POINTER(C.c_size_t)),
                ("c", C.c_void_p), ("nc", C.POINTER(C.c_size_t)), ("wc", C.POINTER(C.c_size_t))]


def _declare(L):
    if getattr(L, "_plans_declared", False):
        return
    L.tlibttm_plan_batched.restype = C.c_int
    L.tlibttm_plan_batched.argtypes = [C.c_int, C.c_int, C.c_size_t, C.POINTER(_Problem), C.POINTER(C.c_void_p)]
    L.tlibttm_plan_batched_ex.restype = C.c_int
    L.tlibttm_plan_batched_ex.argtypes = [C.c_int, C.c_int, C.c_size_t, C.POINTER(_Problem), C.c_uint,
                                          C.POINTER(C.c_void_p)]
    L.tlibttm_plan_chain.restype = C.c_int
    L.tlibttm_plan_chain.argtypes = [C.c_int, C.c_int, C.c_uint, C.c_void_p, C.POINTER(C.c_size_t),
                                     C.POINTER(C.c_size_t), C.c_uint, C.POINTER(C.c_uint),
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                     C.c_void_p, C.POINTER(C.c_void_p)]
    for name in ("tlibttm_plan_run", "tlibttm_plan_run_graph"):
        f = getattr(L, name)
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.c_void_p]
    L.tlibttm_plan_launches.restype = C.c_int
    L.tlibttm_plan_launches.argtypes = [C.c_void_p]
    L.tlibttm_plan_destroy.restype = C.c_int
    L.tlibttm_plan_destroy.argtypes = [C.c_void_p]
    L._plans_declared = True


def _dense_strides(shape, pi):
    w = [1] * len(shape)
    for r in range(1, len(shape)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * shape[pi[r - 1] - 1]
    return w


def _dtype(t) -> int:
    return _lib.F32 if t.dtype == torch.float32 else _lib.F64


class _Plan:
    def __init__(self):
        self._h = C.c_void_p()
        self._keep = []

    @property
    def launches(self) -> int:
        return int(_lib.lib().tlibttm_plan_launches(self._h))

    def run(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().tlibttm_plan_run(self._h, C.c_void_p(s)))

    def run_graph(self, stream=None):
        """Replays the plan as one CUDA graph (captured on the first call)."""
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().tlibttm_plan_run_graph(self._h, C.c_void_p(s)))

    def close(self):
        if self._h:
            _lib.lib().tlibttm_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


class BatchPlan(_Plan):
    """Independent TTMs C_i = A_i x_{q_i} B_i; each entry (q, A, B, C, pia) with C preallocated.

    A_i and C_i are dense torch CUDA tensors in memory order with layout ``pia`` (one-based,
    fastest mode first; their shapes are the mode extents in mode order); B_i has shape (m, n_q)
    and is read row-major (or column-major when ``b_cm``). ``few_launches``: small-m problems of
    any size share the grouped small-m launch (fewer launches per run; for eager launching rather
    than graph replay)."""

    FEW_LAUNCHES = 1

    def __init__(self, problems, precision="default", few_launches=False):
        super().__init__()
        L = _lib.lib()
        _declare(L)
        arr = (_Problem * len(problems))()
        dt = None
        for i, pr in enumerate(problems):
            q, A, B, Cc, na, pia = pr["q"], pr["A"], pr["B"], pr["C"], pr["na"], pr["pia"]
            m, nq = pr["m"], na[q - 1]
            nc = list(na)
            nc[q - 1] = m
            meta = [_lib.sz(na), _lib.sz(_dense_strides(na, pia)), _lib.sz(pia), _lib.sz([m, nq]),
                    _lib.sz([1, 2] if pr.get("b_cm", False) else [2, 1]), _lib.sz(nc),
                    _lib.sz(_dense_strides(nc, pia))]
            self._keep.append((A, B, Cc, meta))
            arr[i] = _Problem(q, len(na), A.data_ptr(), meta[0], meta[1], meta[2], B.data_ptr(), meta[3], meta[4],
                              Cc.data_ptr(), meta[5], meta[6])
            dt = _dtype(A)
        self._keep.append(arr)
        _lib.check(L.tlibttm_plan_batched_ex(dt if dt is not None else _lib.F32,
                                             _lib.PRECISIONS.get(precision, precision)
                                             if isinstance(precision, str) else int(precision), len(problems), arr,
                                             self.FEW_LAUNCHES if few_launches else 0, C.byref(self._h)))


class ChainPlan(_Plan):
    """C = A x_{modes[0]} Bs[0] x_{modes[1]} Bs[1] ... (Tucker projection, ttmpy.ttms).

    A: dense torch CUDA tensor with mode extents ``na`` and layout ``pia``; Bs[s] of shape
    (m_s, current extent of mode modes[s]), row-major; C preallocated with the final extents."""

    def __init__(self, A, na, pia, modes, Bs, C_out, precision="default"):
        super().__init__()
        L = _lib.lib()
        _declare(L)
        n = len(modes)
        if len(Bs) != n:
            raise ValueError("ChainPlan: one matrix per mode is required.")
        ext = list(na)
        for r, b in zip(modes, Bs):
            if not 1 <= r <= len(na) or b.dim() != 2 or int(b.shape[1]) != ext[r - 1]:
                raise ValueError(f"ChainPlan: matrix for mode {r} must have {ext[r - 1] if 1 <= r <= len(na) else '?'} "
                                 "columns (the current extent of that mode).")
            ext[r - 1] = int(b.shape[0])
        if C_out.numel() != int(__import__("math").prod(ext)) or A.numel() != int(__import__("math").prod(na)):
            raise ValueError("ChainPlan: A or C does not have the element count its extents imply.")
        mods = (C.c_uint * n)(*modes)
        bptr = (C.c_void_p * n)(*[b.data_ptr() for b in Bs])
        ms = _lib.sz([b.shape[0] for b in Bs])
        pibs = _lib.sz([x for _ in Bs for x in (2, 1)])
        self._keep.extend([A, list(Bs), C_out, mods, bptr, ms, pibs, _lib.sz(na), _lib.sz(pia)])
        _lib.check(L.tlibttm_plan_chain(_dtype(A), _lib.PRECISIONS.get(precision, precision)
                                        if isinstance(precision, str) else int(precision), len(na), A.data_ptr(),
                                        self._keep[-2], self._keep[-1], n, mods, bptr, ms, pibs, C_out.data_ptr(),
                                        C.byref(self._h)))
