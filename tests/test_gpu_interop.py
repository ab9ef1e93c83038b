"""Zero-copy device arrays in ttmpy: objects exposing ``__cuda_array_interface__`` or DLPack are
read in place (no copy: the library gets the producer's own pointer), ``out`` receives C in the
caller's memory, and results equal the torch-tensor path bit for bit and the C oracle within
the exact-path bound (FP32 2e-6, FP64 1e-13 relative Frobenius)."""
import numpy as np
import pytest

from ttm_b200 import _lib, ttmpy

pytestmark = pytest.mark.gpu

TOL = {np.float32: 2e-6, np.float64: 1e-13}


class CAIArray:
    """A foreign device array seen only through the CUDA array interface (as CuPy or Numba
    expose it); `stream` adds the version-3 producer stream."""

    def __init__(self, t, stream=None):
        self._t = t
        self._stream = stream

    @property
    def __cuda_array_interface__(self):
        d = dict(self._t.__cuda_array_interface__)
        if self._stream is not None:
            d["version"] = 3
            d["stream"] = self._stream
        return d


class DLArray:
    """A foreign device array seen only through DLPack."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, stream=None, **kw):
        return self._t.__dlpack__(stream=stream, **kw)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


def _oracle(oracle_c, q, tA, tB):
    """C of A x_q B through the C oracle, as numpy: tA is a dense torch tensor under some layout
    (a permuted view of contiguous memory), tB a row-major matrix."""
    import known_answer as ka
    na = list(tA.shape)
    wa = list(tA.stride())
    pia = ttmpy._layout_from_strides(na, wa)
    n = int(np.prod(na))
    flat_a = tA.as_strided((n,), (1,), tA.storage_offset()).cpu().numpy()
    b = tB.contiguous().cpu().numpy()
    nc = list(na)
    nc[q - 1] = b.shape[0]
    wc = ka.dense_strides(nc, pia)
    want = np.zeros(int(np.prod(nc)), dtype=flat_a.dtype)
    oracle_c.ttm(q, flat_a, na, wa, pia, b.reshape(-1), list(b.shape), [2, 1], want, nc, wc)
    return np.lib.stride_tricks.as_strided(want, shape=nc, strides=[w * want.itemsize for w in wc])


def _rel(got, want):
    g = np.asarray(got, dtype=np.float64)
    return np.linalg.norm(g - want) / np.linalg.norm(want)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("wrap", [CAIArray, DLArray])
def test_device_arrays_in_place(cuda, oracle_c, wrap, dtype):
    import torch
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    g = torch.Generator(device=cuda).manual_seed(3)
    base = torch.randn(7, 40, 33, 6, device=cuda, dtype=tdt, generator=g)
    tA = base.permute(2, 0, 3, 1)                    # strided view: a permuted layout, no copy
    for q, m in ((1, 24), (2, 5), (4, 130)):
        tB = torch.randn(m, tA.shape[q - 1], device=cuda, dtype=tdt, generator=g)
        A, B = wrap(tA), wrap(tB)
        assert ttmpy._device_view(A).data_ptr() == tA.data_ptr()      # no copy of A
        assert ttmpy._device_view(B).data_ptr() == tB.data_ptr()
        C = ttmpy.ttm(q, A, B)
        assert isinstance(C, torch.Tensor) and C.is_cuda and C.dtype == tdt
        assert torch.equal(C, ttmpy.ttm(q, tA, tB))                  # the torch path's exact bits
        want = _oracle(oracle_c, q, tA, tB)
        assert _rel(C.cpu().numpy(), want) <= TOL[dtype]


@pytest.mark.parametrize("wrap", [CAIArray, DLArray, lambda t: t])
def test_out_receives_c_in_caller_memory(cuda, oracle_c, wrap):
    import torch
    g = torch.Generator(device=cuda).manual_seed(4)
    tA = torch.randn(30, 20, 50, device=cuda, generator=g)
    tB = torch.randn(17, 20, device=cuda, generator=g)
    buf = torch.full((30, 17, 50), float("nan"), device=cuda)
    out = wrap(buf)
    ptr = buf.data_ptr()
    r = ttmpy.ttm(2, wrap(tA), wrap(tB), out=out)
    assert r is out
    torch.cuda.synchronize()
    assert buf.data_ptr() == ptr and not torch.isnan(buf).any()
    assert torch.equal(buf, ttmpy.ttm(2, tA, tB))
    # a C-ordered A gives last-order C: an out with first-order strides is refused
    bad = torch.empty((50, 17, 30), device=cuda).permute(2, 1, 0)
    with pytest.raises(ValueError, match="out must be an array of shape"):
        ttmpy.ttm(2, tA, tB, out=wrap(bad))


def test_producer_stream_is_waited_for(cuda):
    """Version-3 `stream`: A is written on a side stream and handed over without a host sync; the
    product, enqueued on the current stream, must see the finished data."""
    import torch
    side = torch.cuda.Stream()
    src = torch.randn(64, 512, 256, device=cuda)
    tB = torch.randn(8, 512, device=cuda)
    want = ttmpy.ttm(2, src, tB)
    for _ in range(3):
        tA = torch.empty_like(src)
        with torch.cuda.stream(side):
            tA.mul_(0).add_(src)          # the producer's work, queued behind nothing on the current stream
            tA.copy_(src)
        C = ttmpy.ttm(2, CAIArray(tA, stream=side.cuda_stream), tB)
        torch.cuda.synchronize()
        assert torch.equal(C, want)


def test_half_precision_device_input_is_widened_like_the_reference(cuda):
    """The reference binds float64 only and converts other inputs (wrapped_ttm.cpp:229-230);
    a float16 device array is converted to float64 on the device."""
    import torch
    tA = torch.arange(24, device=cuda, dtype=torch.float16).reshape(3, 2, 4)
    tB = torch.arange(10, device=cuda, dtype=torch.float16).reshape(5, 2)
    C = ttmpy.ttm(2, CAIArray(tA), CAIArray(tB))
    assert C.dtype == torch.float64
    want = np.einsum("ijk,xj->ixk", tA.double().cpu().numpy(), tB.double().cpu().numpy())
    assert np.array_equal(C.cpu().numpy(), want)


def test_ttms_on_device_arrays(cuda):
    import torch
    A = torch.arange(3 * 2 * 4 * 5, device=cuda, dtype=torch.float64).reshape(3, 2, 4, 5)
    Bs = [torch.arange(2 * 6, device=cuda, dtype=torch.float64).reshape(6, 2),
          torch.arange(4 * 7, device=cuda, dtype=torch.float64).reshape(7, 4),
          torch.arange(5 * 9, device=cuda, dtype=torch.float64).reshape(9, 5)]
    D = np.einsum("ijkl,yj->iykl", A.cpu().numpy(), Bs[0].cpu().numpy())
    D = np.einsum("ijkl,yk->ijyl", D, Bs[1].cpu().numpy())
    D = np.einsum("ijkl,yl->ijky", D, Bs[2].cpu().numpy())
    for wrap in (CAIArray, DLArray):
        for order in ("forward", "backward", "optimal"):
            got = ttmpy.ttms(1, wrap(A), [wrap(b) for b in Bs], order)
            assert np.array_equal(got.cpu().numpy(), D)


def test_numpy_out(cuda):
    A = np.random.default_rng(5).standard_normal((6, 5, 4))
    B = np.random.default_rng(6).standard_normal((3, 5))
    out = np.full((6, 3, 4), np.nan)
    r = ttmpy.ttm(2, A, B, out=out)
    assert r is out and np.allclose(out, np.einsum("ijk,xj->ixk", A, B), rtol=1e-12, atol=1e-12)
    assert _lib.last_kernel() != ""
