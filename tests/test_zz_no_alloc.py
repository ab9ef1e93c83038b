"""The allocation-free bf16x3 entry point, tlibttm_ttm_f32_bf16x3_noalloc.

Some callers cannot let a library allocate device memory: an application whose
own allocator has already reserved the GPU's memory, a latency-bound loop that
must not risk the implicit device synchronisation of cudaMalloc/cudaFree, or a
process under a fixed memory budget. This entry point runs the same split-BF16
tensor-core kernels as the bf16x3 precision of tlibttm_ttm_ex, with its scratch
(the bf16 image of B, at most 1 MiB, and a status word) in arrays that live in
the library for the life of the process.

The file is named to be collected last, so that a run stopping at the first
failure has already run every other test. It passes alone in a fresh process
and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import known_answer as ka
from ttm_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-5   # the bf16x3 tolerance used throughout the GPU tests


def _problem(dev, na, pia, q, m, b_cm, seed):
    import torch
    g = torch.Generator(device=dev).manual_seed(seed)
    nq = na[q - 1]
    nc = list(na)
    nc[q - 1] = m
    a = torch.randn(int(np.prod(na)), device=dev, generator=g)
    b = torch.randn(m * nq, device=dev, generator=g)
    md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2] if b_cm else [2, 1], nc=nc,
              wc=ka.dense_strides(nc, pia))
    return a, b, md


def _call(fn_name, q, a_ptr, b_ptr, c_ptr, md, stream, extra=()):
    L = _lib.lib()
    fn = getattr(L, fn_name)
    args = list(extra) + [q, len(md["na"]), C.c_void_p(a_ptr), _lib.sz(md["na"]), _lib.sz(md["wa"]),
                          _lib.sz(md["pia"]), C.c_void_p(b_ptr), _lib.sz(md["nb"]), _lib.sz(md["pib"]),
                          C.c_void_p(c_ptr), _lib.sz(md["nc"]), _lib.sz(md["wc"]), C.c_void_p(stream)]
    return fn(*args)


def test_noalloc_matches_existing_entry_point_twice(cuda):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    # Two calls in a row; the second B is smaller, so stale bytes left in the shared image by the
    # first call would show up in its result if any were read.
    for na, pia, q, m, b_cm, seed in (([256, 64, 40], [1, 2, 3], 2, 256, True, 1),
                                      ([96, 33, 300], [1, 2, 3], 1, 48, False, 2)):
        a, b, md = _problem(cuda, na, pia, q, m, b_cm, seed)
        c_old = torch.full((int(np.prod(md["nc"])),), float("nan"), device=cuda)
        c_new = torch.full_like(c_old, float("nan"))
        rc = _call("tlibttm_ttm_ex", q, a.data_ptr(), b.data_ptr(), c_old.data_ptr(), md, stream,
                   extra=(_lib.F32, _lib.PREC_BF16X3))
        assert rc == 0, L.tlibttm_last_error()
        rc = _call("tlibttm_ttm_f32_bf16x3_noalloc", q, a.data_ptr(), b.data_ptr(), c_new.data_ptr(), md, stream)
        assert rc == 0, L.tlibttm_last_error()
        assert _lib.last_kernel().startswith("tc_bf16x3")
        assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0, L.tlibttm_last_error()
        x = c_new.double().cpu().numpy()
        y = c_old.double().cpu().numpy()
        assert np.all(np.isfinite(x))
        err = np.linalg.norm(x - y) / np.linalg.norm(y)
        assert err <= TOL, (na, q, m, err)


def test_noalloc_matches_the_oracle(cuda, oracle_c):
    """Against the C oracle (FP64 accumulation of the float inputs), not only against the other
    entry point of the same kernel; m = 272 > 256 takes two 256-column blocks of B (a 1 MiB image,
    exactly the limit)."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    for na, pia, q, m, b_cm, seed in (([64, 48, 40], [2, 1, 3], 1, 40, True, 4),
                                      ([40, 512, 24], [1, 2, 3], 2, 272, False, 5)):
        a, b, md = _problem(cuda, na, pia, q, m, b_cm, seed)
        c = torch.full((int(np.prod(md["nc"])),), float("nan"), device=cuda)
        rc = _call("tlibttm_ttm_f32_bf16x3_noalloc", q, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream)
        assert rc == 0, L.tlibttm_last_error()
        assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0, L.tlibttm_last_error()
        ha, hb = a.cpu().numpy(), b.cpu().numpy()
        want = np.zeros(int(np.prod(md["nc"])), dtype=np.float32)
        oracle_c.ttm(q, ha, md["na"], md["wa"], md["pia"], hb, md["nb"], md["pib"], want, md["nc"], md["wc"])
        got = c.double().cpu().numpy()
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= TOL, (na, q, m, err)


def _pool_used_high(dev_index):
    """High watermark of the device's default stream-ordered pool (cudaMallocAsync), through the
    CUDA runtime that torch loaded."""
    rt = C.CDLL("libcudart.so.12")
    pool = C.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(C.byref(pool), C.c_int(dev_index)) == 0
    val = C.c_uint64(0)
    assert rt.cudaMemPoolGetAttribute(pool, C.c_int(8), C.byref(val)) == 0   # cudaMemPoolAttrUsedMemHigh
    return rt, pool, val.value


def test_noalloc_allocates_nothing(cuda):
    """The pool's high watermark is reset, the entry point runs twice, and the watermark has not
    moved; the allocating bf16x3 path then moves it, which shows that the check sees allocations."""
    import torch
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # m = 64: the single-SM kernel, whose B image the allocating entry point takes from the pool
    a, b, md = _problem(cuda, [256, 64, 40], [1, 2, 3], 2, 64, True, 6)
    c = torch.empty(int(np.prod(md["nc"])), device=cuda)
    # first call on this device (its one-time symbol lookup) outside the measured window
    assert _call("tlibttm_ttm_f32_bf16x3_noalloc", 2, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream) == 0
    torch.cuda.synchronize()
    rt, pool, _ = _pool_used_high(cuda.index or 0)
    assert rt.cudaMemPoolSetAttribute(pool, C.c_int(8), C.byref(C.c_uint64(0))) == 0   # reset to current use
    _, _, before = _pool_used_high(cuda.index or 0)
    for _ in range(2):
        rc = _call("tlibttm_ttm_f32_bf16x3_noalloc", 2, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream)
        assert rc == 0, L.tlibttm_last_error()
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0
    _, _, after = _pool_used_high(cuda.index or 0)
    assert after == before
    rc = _call("tlibttm_ttm_ex", 2, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream,
               extra=(_lib.F32, _lib.PREC_BF16X3))
    assert rc == 0, L.tlibttm_last_error()
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0
    _, _, grown = _pool_used_high(cuda.index or 0)
    assert grown > before


def test_noalloc_rejects_what_it_cannot_hold(cuda):
    import torch
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # m = 256, n_q = 2048: a 2 MiB B image, over the 1 MiB the entry point holds.
    a, b, md = _problem(cuda, [2048, 64], [1, 2], 1, 256, True, 3)
    c = torch.empty(256 * 64, device=cuda)
    rc = _call("tlibttm_ttm_f32_bf16x3_noalloc", 1, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream)
    assert rc == _lib.ERR_ARG
    assert "at most 1048576 bytes" in L.tlibttm_last_error().decode()
    # m = 272 > 256 pads B to two 256-column blocks: with n_q = 544 the image is 1,114,112 bytes
    a, b, md = _problem(cuda, [544, 40], [1, 2], 1, 272, True, 7)
    c = torch.empty(272 * 40, device=cuda)
    rc = _call("tlibttm_ttm_f32_bf16x3_noalloc", 1, a.data_ptr(), b.data_ptr(), c.data_ptr(), md, stream)
    assert rc == _lib.ERR_ARG
    assert "1114112-byte" in L.tlibttm_last_error().decode()
    # host operands would need staging buffers
    na, pia, q, m = [64, 32, 8], [1, 2, 3], 2, 32
    ha = np.zeros(64 * 32 * 8, dtype=np.float32)
    hb = np.zeros(m * 32, dtype=np.float32)
    hc = np.zeros(64 * m * 8, dtype=np.float32)
    md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, 32], pib=[1, 2], nc=[64, m, 8],
              wc=ka.dense_strides([64, m, 8], pia))
    rc = _call("tlibttm_ttm_f32_bf16x3_noalloc", q, ha.ctypes.data, hb.ctypes.data, hc.ctypes.data, md, stream)
    assert rc == _lib.ERR_ARG
    assert "device memory" in L.tlibttm_last_error().decode()
    assert L.tlibttm_synchronize(C.c_void_p(stream)) == 0
