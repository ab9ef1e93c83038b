"""Drop-in for the reference's Python binding ``ttmpy`` (ttmpy/src/wrapped_ttm.cpp).

    from ttm_b200 import ttmpy as tp
    C = tp.ttm(q, A, B)                 # mode-q product, q one-based
    D = tp.ttms(q, A, Bs, "forward")    # multiply every mode except q

Both functions run on the GPU through the C ABI (include/tlibttm.h); there is
no CPU fallback. Inputs may be numpy arrays (results come back as numpy
arrays, the call blocks) or device arrays: torch CUDA tensors, or any object
that exposes ``__cuda_array_interface__`` (versions 0-3: CuPy, Numba, ...) or
the DLPack protocol (``__dlpack__``). Device arrays are used in place, with
no copy and no host round trip; results are torch CUDA tensors produced on
the current torch stream (they expose both protocols in turn, so CuPy and
others take them without a copy), or the caller's own array given as ``out``.

Same contract as the reference binding, plus four widenings:

* float32 as well as float64 (the reference binds only double,
  wrapped_ttm.cpp:229-230). Other dtypes are converted to float64, as
  pybind11's ``array_t<double>`` does.
* A's layout pi is read from its strides (a C-ordered array gives the
  last-order layout the reference hard-codes, wrapped_ttm.cpp:45), so
  transposed or permuted views are computed correctly without a copy; C gets
  A's layout, as in the reference (wrapped_ttm.cpp:57-66).
* B's own memory order is honoured (row- or column-major); the reference
  assumes row-major (wrapped_ttm.cpp:46).
* device arrays in place (above): the reference binds numpy only and copies
  every result into a new numpy array (wrapped_ttm.cpp:57-66).

Error behaviour follows the reference: its own checks raise ValueError with
the same texts (wrapped_ttm.cpp:37-53, 90-127); checks of tlib::ttm raise
RuntimeError with tlib's texts (include/tlib/ttm.h:65-90).
"""
from __future__ import annotations

import numpy as np

from . import _lib

try:  # torch is optional for numpy callers
    import torch
except Exception:  # noqa: BLE001
    torch = None


def _is_torch(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor)


def _cai_layout(iface):
    """(pointer, shape, element strides, numpy dtype) of a ``__cuda_array_interface__`` dict.

    Strides None means C order (the interface's convention); byte strides must be whole
    elements. Masked arrays are rejected.
    """
    if iface.get("mask") is not None:
        raise ValueError("ttmpy: masked device arrays are not supported.")
    shape = tuple(int(x) for x in iface["shape"])
    dt = np.dtype(iface["typestr"])
    ptr = int(iface["data"][0]) if iface.get("data") is not None else 0
    st = iface.get("strides")
    if st is None:
        strides, acc = [], 1
        for n in reversed(shape):
            strides.append(acc)
            acc *= n
        strides = tuple(reversed(strides))
    else:
        if any(int(b) % dt.itemsize for b in st):
            raise ValueError("ttmpy: device array strides must be whole elements.")
        strides = tuple(int(b) // dt.itemsize for b in st)
    return ptr, shape, strides, dt


def _device_view(x):
    """A torch tensor over the memory of ``x`` (no copy) when ``x`` is a device array given
    through ``__cuda_array_interface__`` or DLPack; None for numpy arrays, torch tensors and
    anything else.

    A ``stream`` entry of the CUDA array interface (version 3) is honoured: the current torch
    stream waits for the producer's stream before any library work reads the memory. DLPack
    producers order their own work, given the consumer's stream by ``torch.from_dlpack``.
    """
    if torch is None or _is_torch(x) or isinstance(x, np.ndarray):
        return None
    iface = getattr(x, "__cuda_array_interface__", None)
    if iface is not None:
        _cai_layout(iface)
        t = torch.as_tensor(x, device="cuda")
        stream = iface.get("stream")
        if stream is not None and int(stream) != 0:
            ev = torch.cuda.Event()
            ev.record(torch.cuda.ExternalStream(int(stream), device=t.device))
            torch.cuda.current_stream(t.device).wait_event(ev)
        return t
    if hasattr(x, "__dlpack__"):
        return torch.from_dlpack(x)
    return None


def _layout_from_strides(shape, strides):
    """One-based layout pi listing modes from smallest to largest stride (ties: higher mode first)."""
    p = len(shape)
    order = sorted(range(p), key=lambda r: (strides[r], -r))
    return [r + 1 for r in order]


def _dense_strides(shape, pi):
    w = [1] * len(shape)
    for r in range(1, len(shape)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * shape[pi[r - 1] - 1]
    return w


def _dtype_id(dt) -> int:
    return _lib.F32 if dt in (np.float32, getattr(torch, "float32", None)) else _lib.F64


def _prec(precision) -> int:
    if isinstance(precision, str):
        return _lib.PRECISIONS[precision]
    return int(precision)


def _check_q_p(q, p, fn):
    if p == 0:
        if fn == "ttm":
            raise ValueError("Error calling ttmpy::ttm: first input should be a tensor with order greater than zero.")
        raise ValueError("Error calling ttmpy::ttms: input tensor order should be greater than zero.")


def _out_error(nc, wc, dt):
    return ValueError(f"ttmpy: out must be an array of shape {tuple(nc)} and dtype {dt} laid out like A "
                      f"(strides {tuple(wc)} in elements).")


def _ttm_numpy(q, A, B, precision, out=None):
    if precision == "tuned":
        precision = "plain"
    dB = B if _is_torch(B) else _device_view(B)
    if dB is not None:
        B = dB.detach().cpu().numpy()
    A = np.asarray(A)
    p = A.ndim
    _check_q_p(q, p, "ttm")
    if q == 0 or q > p:
        raise ValueError("Error calling ttmpy::ttm: contraction mode should be greater than zero and at most equal to p.")
    if A.dtype not in (np.float32, np.float64):
        A = A.astype(np.float64)
    B = np.asarray(B)
    if B.ndim != 2:
        raise ValueError("Error calling ttmpy::ttm: second input should be a mtrix with order equal to 2.")
    if B.dtype != A.dtype:
        B = B.astype(A.dtype)
    if any(s < 0 for s in A.strides) or any(s % A.itemsize for s in A.strides):
        A = np.ascontiguousarray(A)
    if B.flags.c_contiguous:
        pib = [2, 1]
    elif B.flags.f_contiguous:
        pib = [1, 2]
    else:
        B = np.ascontiguousarray(B)
        pib = [2, 1]
    na = list(A.shape)
    wa = [s // A.itemsize for s in A.strides]
    pia = _layout_from_strides(na, wa)
    nb = list(B.shape)
    nc = list(na)
    nc[q - 1] = nb[0]
    wc = _dense_strides(nc, pia)
    if out is None:
        C = np.lib.stride_tricks.as_strided(np.empty(int(np.prod(nc)), dtype=A.dtype), shape=nc,
                                            strides=[w * A.itemsize for w in wc])
    else:
        C = out
        if (not isinstance(C, np.ndarray) or C.dtype != A.dtype or list(C.shape) != nc
                or [st // C.itemsize for st in C.strides] != wc or not C.flags.writeable):
            raise _out_error(nc, wc, A.dtype)
    _lib.ttm_raw(_dtype_id(A.dtype.type), _prec(precision), q, p, A.ctypes.data, na, wa, pia,
                 B.ctypes.data, nb, pib, C.ctypes.data, nc, wc, 0)
    return C


def _ttm_torch(q, A, B, precision, out=None):
    B_in = B
    p = A.dim()
    _check_q_p(q, p, "ttm")
    if q == 0 or q > p:
        raise ValueError("Error calling ttmpy::ttm: contraction mode should be greater than zero and at most equal to p.")
    if A.dtype not in (torch.float32, torch.float64):
        A = A.to(torch.float64)
    if not _is_torch(B):
        B = _device_view(B)
        if B is None:
            B = torch.as_tensor(np.asarray(B_in), device=A.device)
    if B.dim() != 2:
        raise ValueError("Error calling ttmpy::ttm: second input should be a mtrix with order equal to 2.")
    B = B.to(device=A.device, dtype=A.dtype)
    if any(s < 0 for s in A.stride()):
        A = A.contiguous()
    if B.is_contiguous():
        pib = [2, 1]
    elif B.t().is_contiguous():
        pib = [1, 2]
    else:
        B = B.contiguous()
        pib = [2, 1]
    na = list(A.shape)
    wa = list(A.stride())
    pia = _layout_from_strides(na, wa)
    nb = list(B.shape)
    nc = list(na)
    nc[q - 1] = nb[0]
    wc = _dense_strides(nc, pia)
    if out is None:
        C = torch.empty_strided(nc, wc, dtype=A.dtype, device=A.device)
    else:
        C = out if _is_torch(out) else _device_view(out)
        if (C is None or C.dtype != A.dtype or C.device != A.device or list(C.shape) != nc
                or list(C.stride()) != wc):
            raise _out_error(nc, wc, str(A.dtype).replace("torch.", ""))
    stream = torch.cuda.current_stream(A.device).cuda_stream if A.is_cuda else 0
    if precision == "tuned" and A.is_cuda and _dense_strides(na, pia) == wa:
        # the learned schedule selector picks among the exact kernels (float32 may also take bf16x3)
        from . import selector
        pr = dict(p=p, na=na, q=q, pia=pia, m=nb[0])
        allowed = set(range(1, selector.NS + 1)) if A.dtype == torch.float32 else set(selector.EXACT)
        with torch.cuda.device(A.device):
            sched, _ = selector.default_selector(A.device).choose(pr, allowed, _dtype_id(A.dtype))
            _lib.check(selector.lib().tlibttm_ttm_sched(_dtype_id(A.dtype), sched, q, p, A.data_ptr(), _lib.sz(na),
                                                        _lib.sz(wa), _lib.sz(pia), B.data_ptr(), _lib.sz(nb),
                                                        _lib.sz(pib), C.data_ptr(), _lib.sz(nc), _lib.sz(wc), stream))
        return C
    if precision == "tuned":
        precision = "auto" if A.dtype == torch.float32 else "plain"
    if A.is_cuda:
        with torch.cuda.device(A.device):
            _lib.ttm_raw(_dtype_id(A.dtype), _prec(precision), q, p, A.data_ptr(), na, wa, pia,
                         B.data_ptr(), nb, pib, C.data_ptr(), nc, wc, stream)
    else:
        _lib.ttm_raw(_dtype_id(A.dtype), _prec(precision), q, p, A.data_ptr(), na, wa, pia,
                     B.data_ptr(), nb, pib, C.data_ptr(), nc, wc, 0)
    return C


def ttm(q, A, B, precision="default", out=None):
    """Mode-q tensor-times-matrix product C = A x_q B (reference wrapped_ttm.cpp:23-76).

    C(i1..j..ip) = sum_{iq} A(i1..iq..ip) * B(j, iq); q is one-based.
    ``precision`` selects the arithmetic ("default", "plain", "bf16x3",
    "auto", or "tuned"); "default" is the library-wide setting (plain unless
    changed). "tuned" lets the learned schedule selector pick the kernel for
    device tensors (FP32-accurate for float32, exact for float64).

    ``out`` (optional) receives C in place and is returned: for device inputs a torch CUDA
    tensor or any device array (CUDA array interface, DLPack) on A's device, for numpy inputs a
    writeable numpy array; either way with C's shape, A's dtype and A's layout (the strides of
    a dense array whose modes are ordered as A's). Anything else raises ValueError.
    """
    q = int(q)
    dA = _device_view(A)
    if dA is not None:
        A = dA
    if _is_torch(A):
        C = _ttm_torch(q, A, B, precision, out)
    else:
        C = _ttm_numpy(q, A, B, precision, out)
    return C if out is None else out


def _ttms_check(q, A, Bs, order):
    if order not in ("optimal", "backward", "forward"):
        raise ValueError("Error calling ttmpy::ttms: multiplication order should be either 'optimal', 'backward' or 'forward'.")
    p = A.dim() if _is_torch(A) else np.asarray(A).ndim
    if p == 0:
        raise ValueError("Error calling ttmpy::ttms: input tensor order should be greater than zero.")
    if len(Bs) != p - 1:
        raise ValueError("Error calling ttmpy::ttms: number of input matrices is not equal to the tensor order - 1.")
    if q == 0 or q > p:
        raise ValueError("Error calling ttmpy::ttms: non-contraction mode should be greater than zero and at most equal to p.")
    if not all((b.dim() if _is_torch(b) else np.asarray(b).ndim) == 2 for b in Bs):
        raise ValueError("Error calling ttmpy::ttms: some of the input matrices are not matrices.")
    na = list(A.shape)
    nbs = [tuple(b.shape) for b in Bs]
    # Same comparisons as wrapped_ttm.cpp:120-121. Like the reference, the
    # matrix of mode q+1 is not compared here; a mismatch there surfaces as
    # tlib's RuntimeError from the contraction itself.
    ok1 = all(nbs[r][1] == na[r] for r in range(q - 1))
    ok2 = all(nbs[r][1] == na[r + 1] for r in range(q, p - 1))
    if not (ok1 and ok2):
        raise ValueError("Error calling ttmpy::ttms: vector dimension is not compatible with the dimension of a tensor mode.")
    return p


def _ttms_sequence(q, p, Bs, order):
    """(mode, matrix index) pairs in the reference's multiplication order (wrapped_ttm.cpp:132-218)."""
    def bidx(r):  # matrix of mode r (one-based, r != q)
        return r - 1 if r < q else r - 2

    modes = [r for r in range(1, p + 1) if r != q]
    if order == "forward":
        seq = modes
    elif order == "backward":
        seq = modes[::-1]
    else:
        # ascending 1/n_k - 1/m_k for B_k of shape (m_k, n_k): shrinking products first
        def key(r):
            m_k, n_k = Bs[bidx(r)].shape
            return 1.0 / float(n_k) - 1.0 / float(m_k)
        seq = sorted(modes, key=key)
    return [(r, bidx(r)) for r in seq]


def ttms(q, A, Bs, order="forward", precision="default"):
    """Multiply A by Bs[k] on every mode except q (reference wrapped_ttm.cpp:81-222).

    ``order`` is "forward" (ascending modes), "backward" (descending) or
    "optimal" (ascending 1/n_k - 1/m_k, i.e. the most shrinking factors first).
    The whole chain runs as one plan (include/tlibttm.h, tlibttm_plan_chain):
    numpy inputs are moved to the GPU once, intermediates stay in device
    buffers the plan owns, and only the final tensor returns to the host.
    Device arrays (torch, CUDA array interface, DLPack) are read in place and
    the result is a torch CUDA tensor.
    """
    q = int(q)
    dA = _device_view(A)
    if dA is not None:
        A = dA
    views = [_device_view(b) for b in Bs]
    Bs = [b if v is None else v for b, v in zip(Bs, views)]
    p = _ttms_check(q, A, Bs, order)
    seq = _ttms_sequence(q, p, Bs, order)
    if torch is None or not torch.cuda.is_available():
        c = A
        for r, k in seq:
            c = ttm(r, c, Bs[k], precision)
        return c
    from .plans import ChainPlan
    host = not _is_torch(A)
    if host:
        A = np.asarray(A)
        if A.dtype not in (np.float32, np.float64):
            A = A.astype(np.float64)
        dev = torch.device("cuda", torch.cuda.current_device())
        tA = torch.from_numpy(np.ascontiguousarray(A)).to(dev)
    else:
        tA = A.contiguous()
        if tA.dtype not in (torch.float32, torch.float64):
            tA = tA.to(torch.float64)
        dev = tA.device
    dt = tA.dtype
    # C-ordered tensor: mode r has extent shape[r-1]; layout is last-order (p, ..., 1).
    na = list(tA.shape)
    pia = list(range(p, 0, -1))
    bs = []
    ext = list(na)
    for r, k in seq:
        b = Bs[k]
        if int(b.shape[1]) != ext[r - 1]:
            # what tlib::ttm raises for this contraction (include/tlib/ttm.h:80)
            raise RuntimeError("Error in tlib::tensor_times_matrix: contraction dimension of A and B are not equal.")
        b = b.to(device=dev, dtype=dt) if _is_torch(b) else torch.from_numpy(np.asarray(b)).to(device=dev, dtype=dt)
        bs.append(b.contiguous())
        ext[r - 1] = int(b.shape[0])
    out = torch.empty(ext, device=dev, dtype=dt)
    with torch.cuda.device(dev):
        plan = ChainPlan(tA.reshape(-1), na, pia, [r for r, _ in seq], bs, out.reshape(-1), precision=precision)
        plan.run()
        torch.cuda.current_stream(dev).synchronize()
        plan.close()
    return out.cpu().numpy() if host else out
