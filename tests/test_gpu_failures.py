"""Failure detection without a GPU fault (host-side injection through tlibttm_inject).

* A bounded wait that runs out: the bf16x3 kernel's first pipeline stage is never filled (the
  single-SM kernel's B stage; the pair kernel's first A stage in the even CTA) and every mbarrier
  wait is bounded at 1 ms, so the waits on that stage expire. The kernel's blocks
  stop, drain their own copies, free tensor memory and raise the device status word;
  tlibttm_synchronize reports TLIBTTM_ERR_DEVICE once (the word is read and cleared), and the
  next call on the same context succeeds with correct results. The same for the allocation-free
  entry point, whose status word is its own.
* A failed device allocation: the n-th allocation of the library fails; the call returns
  TLIBTTM_ERR_ALLOC and the next one succeeds.
* Explicit 8-bit requests that the 8-bit paths cannot run are rejected, not downgraded.
"""
import ctypes as C

import numpy as np
import pytest

import known_answer as ka
from ttm_b200 import _lib

pytestmark = pytest.mark.gpu

SHORT_WAIT_NS = 1_000_000   # 1 ms


@pytest.fixture(autouse=True)
def _clear_injections():
    yield
    _lib.inject(_lib.INJECT_NONE)


def _problem(dev, na, pia, q, m, seed=0, dtype=None):
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=dev).manual_seed(seed)
    nq = na[q - 1]
    nc = list(na)
    nc[q - 1] = m
    a = torch.randn(int(np.prod(na)), device=dev, generator=g, dtype=dtype)
    b = torch.randn(m * nq, device=dev, generator=g, dtype=dtype)
    c = torch.full((int(np.prod(nc)),), float("nan"), device=dev, dtype=dtype)
    md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2], nc=nc,
              wc=ka.dense_strides(nc, pia))
    return a, b, c, md


def _args(q, a, b, c, md, stream):
    return [q, len(md["na"]), C.c_void_p(a), _lib.sz(md["na"]), _lib.sz(md["wa"]), _lib.sz(md["pia"]),
            C.c_void_p(b), _lib.sz(md["nb"]), _lib.sz(md["pib"]), C.c_void_p(c), _lib.sz(md["nc"]),
            _lib.sz(md["wc"]), C.c_void_p(stream)]


def _want(a, b, md, q):
    """FP64 result on the device (torch), for the recovery check."""
    import torch
    na, m = md["na"], md["nb"][0]
    p = len(na)
    A = a.double().view(*reversed(na))          # first-order layout: torch dims are modes p..1
    B = b.double().view(na[q - 1], m).t()       # column-major (m, n_q)
    axis = p - q
    return torch.movedim(torch.tensordot(A, B, dims=([axis], [1])), -1, axis).reshape(-1)


@pytest.mark.parametrize("entry", ["ex", "noalloc"])
@pytest.mark.parametrize("m", [64, 256])   # the single-SM kernel, and the pair kernel (clusters of two)
def test_bounded_wait_runs_out_and_is_reported_once(cuda, entry, m):
    import torch
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    q, pia = 2, [1, 2, 3]
    a, b, c, md = _problem(cuda, [256, 64, 40], pia, q, m)

    def call():
        args = _args(q, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream)
        if entry == "ex":
            return L.tlibttm_ttm_ex(_lib.F32, _lib.PREC_BF16X3, *args)
        return L.tlibttm_ttm_f32_bf16x3_noalloc(*args)

    assert call() == 0, L.tlibttm_last_error()            # set-up outside the injected launch
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0
    _lib.inject(_lib.INJECT_WAIT_NS, SHORT_WAIT_NS)
    _lib.inject(_lib.INJECT_SKIP_B_STAGE, 1)
    assert call() == 0, L.tlibttm_last_error()            # the launch itself succeeds
    assert _lib.last_kernel() == ("tc_bf16x3" if m <= 128 else "tc_bf16x3_pair")
    rc = L.tlibttm_synchronize(C.c_void_p(stream))
    assert rc == _lib.ERR_DEVICE, (rc, L.tlibttm_last_error())
    assert b"bounded wait" in L.tlibttm_last_error()
    # read and cleared: reported once, and the context stays usable
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0
    _lib.inject(_lib.INJECT_NONE)
    c.fill_(float("nan"))
    assert call() == 0, L.tlibttm_last_error()
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0
    got, want = c.double(), _want(a, b, md, q)
    assert float(torch.linalg.norm(got - want) / torch.linalg.norm(want)) <= 1e-5


def test_failed_allocation_returns_err_alloc(cuda):
    import torch
    L = _lib.lib()
    L.tlibttm_release_buffers()
    q, pia = 2, [1, 2, 3]
    # host operands: the call stages them in device buffers it allocates
    na, m = [64, 48, 40], 40
    a_h = np.random.default_rng(0).standard_normal(int(np.prod(na))).astype(np.float64)
    b_h = np.random.default_rng(1).standard_normal(m * na[q - 1]).astype(np.float64)
    nc = [64, m, 40]
    c_h = np.zeros(int(np.prod(nc)))
    md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, na[q - 1]], pib=[1, 2], nc=nc,
              wc=ka.dense_strides(nc, pia))
    args = _args(q, a_h.ctypes.data, b_h.ctypes.data, c_h.ctypes.data, md, 0)
    _lib.inject(_lib.INJECT_FAIL_ALLOC, 1)
    rc = L.tlibttm_ttm_ex(_lib.F64, _lib.PREC_PLAIN, *args)
    assert rc == _lib.ERR_ALLOC, (rc, L.tlibttm_last_error())
    assert L.tlibttm_ttm_ex(_lib.F64, _lib.PREC_PLAIN, *args) == 0, L.tlibttm_last_error()
    want = np.einsum("kli,jl->kji", a_h.reshape(40, 48, 64), b_h.reshape(48, m).T).reshape(-1)
    assert np.linalg.norm(c_h - want) <= 1e-13 * np.linalg.norm(want)
    # device operands on the bf16x3 path: its pre-split B image is the allocation that fails
    stream = torch.cuda.current_stream().cuda_stream
    a, b, c, md = _problem(cuda, [256, 64, 40], pia, q, 64)
    args = _args(q, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream)
    _lib.inject(_lib.INJECT_FAIL_ALLOC, 1)
    rc = L.tlibttm_ttm_ex(_lib.F32, _lib.PREC_BF16X3, *args)
    assert rc == _lib.ERR_ALLOC, (rc, L.tlibttm_last_error())
    assert L.tlibttm_ttm_ex(_lib.F32, _lib.PREC_BF16X3, *args) == 0, L.tlibttm_last_error()
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0


def test_explicit_8bit_requests_are_not_downgraded(cuda):
    import torch
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # ozaki keeps int32 digit sums exact only up to n_q = 16384
    a, b, c, md = _problem(cuda, [20000, 32], [1, 2], 1, 24, dtype=torch.float64)
    rc = L.tlibttm_ttm_ex(_lib.F64, _lib.PREC_OZAKI, *_args(1, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream))
    assert rc == _lib.ERR_UNSUPPORTED and b"16384" in L.tlibttm_last_error()
    # fp8 takes float operands only
    rc = L.tlibttm_ttm_ex(_lib.F64, _lib.PREC_FP8, *_args(1, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream))
    assert rc == _lib.ERR_UNSUPPORTED
