"""Shapes whose output tiles cannot fill the GPU: a split l (K) range.

* `bvec`: few output rows (outer * inner <= 8) with 16 < m <= 256 and a long l range, e.g. the
  order-1 product c = B a (reference include/tlib/detail/mtm.h:171-177, 212-218): B is streamed
  by the whole GPU, each block's partial sums go to a workspace and a second kernel adds them in
  a fixed block order.
  The same kernels take small m (m <= 16) with few rows, where the column and row kernels would
  run one or two blocks.
* the SIMT slice-GEMM with its K loop split over blocks (few row x column tiles, long l range),
  partial tiles added in a fixed order.

Both are exact FMA in the I/O type (bound: FP32 2e-6 and FP64 1e-13 relative Frobenius error
against the C oracle, the bounds of the other exact-path tests), deterministic (two runs give
identical bits), and at full size (n = 2^26) exact on integer data.
"""
import numpy as np
import pytest

import known_answer as ka
from ttm_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = {np.float32: 2e-6, np.float64: 1e-13}


def _run(dev, na, pia, q, m, b_cm, dtype, precision=_lib.PREC_DEFAULT, a=None, b=None, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    nq = na[q - 1]
    nc = list(na)
    nc[q - 1] = m
    wa, wc = ka.dense_strides(na, pia), ka.dense_strides(nc, pia)
    if a is None:
        a = rng.standard_normal(int(np.prod(na))).astype(dtype)
    if b is None:
        b = rng.standard_normal(m * nq).astype(dtype)
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    tc = torch.full((int(np.prod(nc)),), float("nan"), device=dev, dtype=ta.dtype)
    pib = [1, 2] if b_cm else [2, 1]
    _lib.ttm_raw(_lib.F32 if dtype == np.float32 else _lib.F64, precision, q, len(na), ta.data_ptr(), na, wa, pia,
                 tb.data_ptr(), [m, nq], pib, tc.data_ptr(), nc, wc, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    md = dict(na=na, wa=wa, pia=pia, nb=[m, nq], pib=pib, nc=nc, wc=wc)
    return a, b, tc.cpu().numpy(), md, _lib.last_kernel()


def _check(oracle_c, q, a, b, got, md):
    want = np.zeros(int(np.prod(md["nc"])), dtype=a.dtype)
    oracle_c.ttm(q, a, md["na"], md["wa"], md["pia"], b, md["nb"], md["pib"], want, md["nc"], md["wc"])
    return np.linalg.norm(got.astype(np.float64) - want) / np.linalg.norm(want.astype(np.float64))


BVEC_CASES = [
    # (na, pia, q, m, b_cm)          notes
    ([1 << 18], [1], 1, 64, True),   # order 1: c = B a
    ([1 << 18], [1], 1, 200, False), # order 1, row-major B, m not a multiple of 64
    ([5000], [1], 1, 17, True),      # l range not a multiple of the chunk, m just above the small-m kernels
    ([4, 1 << 16], [1, 2], 2, 96, True),   # order 2, four rows (inner 4)
    ([1 << 16, 8], [1, 2], 1, 33, False),  # order 2, eight rows (outer 8), row-major B
    ([3, 8192, 2], [1, 2, 3], 2, 130, True),  # six rows (inner 3 x outer 2)
]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("case", BVEC_CASES)
def test_bvec_against_oracle(cuda, oracle_c, case, dtype):
    na, pia, q, m, b_cm = case
    a, b, got, md, kern = _run(cuda, na, pia, q, m, b_cm, dtype)
    assert kern == "bvec", kern
    err = _check(oracle_c, q, a, b, got, md)
    assert err <= TOL[dtype], (case, err)
    # deterministic: the same bits again, and under the FP32-accurate precision (bvec is exact)
    _, _, again, _, _ = _run(cuda, na, pia, q, m, b_cm, dtype, a=a, b=b)
    assert np.array_equal(got, again)
    if dtype == np.float32:
        _, _, auto, _, kern = _run(cuda, na, pia, q, m, b_cm, dtype, precision=_lib.PREC_AUTO, a=a, b=b)
        assert kern == "bvec" and np.array_equal(got, auto)


SMALL_M_FEW_ROWS = [
    # (na, pia, q, m, b_cm)           m <= 16, outer * inner <= 8 rows, n_q >= 4096
    ([1 << 16, 2], [2, 1], 1, 8, True),    # two rows 2 apart (inner 2): not 16-byte aligned
    ([5001, 3], [1, 2], 1, 5, False),      # three contiguous fibres of odd length, row-major B
    ([4097], [1], 1, 1, True),             # order 1, m = 1: one dot product
    ([7, 8192], [1, 2], 2, 16, True),      # seven rows (inner 7)
    ([1 << 15, 8], [1, 2], 1, 3, True),    # eight aligned fibres, A below the TMA kernel's size
    # more than eight rows: row tiles of eight along the grid
    ([63, 16411], [1, 2], 2, 8, True),     # 63 strided rows (a partial last tile)
    ([2049, 1023], [1, 2], 1, 16, False),  # 1023 contiguous fibres, row-major B
    ([5, 7, 17000], [1, 2, 3], 3, 1, True),  # 35 rows over two modes, m = 1
    ([9, 1100, 11], [2, 1, 3], 2, 4, False),  # q = pi_1 with outer 99 rows, row-major B
]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("case", SMALL_M_FEW_ROWS)
def test_small_m_few_rows_take_the_l_split(cuda, oracle_c, case, dtype):
    """Small m with few output rows and a long l range: the column and row kernels would run one
    or a few blocks over the whole range, so the l range is split over the GPU (the bvec kernels,
    row tiles of eight beyond eight rows, and their fixed-order reduction), exact and
    deterministic."""
    na, pia, q, m, b_cm = case
    n0 = _lib.launch_count()
    a, b, got, md, kern = _run(cuda, na, pia, q, m, b_cm, dtype)
    assert kern == "bvec", kern
    assert _lib.launch_count() - n0 == 2
    err = _check(oracle_c, q, a, b, got, md)
    assert err <= TOL[dtype], (case, err)
    _, _, again, _, _ = _run(cuda, na, pia, q, m, b_cm, dtype, a=a, b=b)
    assert np.array_equal(got, again)


SPLIT_CASES = [
    # (na, pia, q, m, b_cm, dtype)        the row x column tiles are too few for the GPU
    ([128, 16384], [1, 2], 2, 256, True, np.float32),    # two 128 x 128 tiles, l range 16384
    ([128, 16384], [1, 2], 2, 256, False, np.float32),
    ([16384, 100], [1, 2], 1, 40, True, np.float32),     # contiguous fibres (q = pi_1), 100 rows
    ([64, 8192, 3], [1, 2, 3], 2, 100, False, np.float64),   # double: 64 x 64 tiles, 192 rows
    ([40, 9000], [1, 2], 2, 300, True, np.float64),
]


@pytest.mark.parametrize("case", SPLIT_CASES)
def test_split_k_simt_gemm_against_oracle(cuda, oracle_c, case):
    na, pia, q, m, b_cm, dtype = case
    n0 = _lib.launch_count()
    a, b, got, md, kern = _run(cuda, na, pia, q, m, b_cm, dtype, precision=_lib.PREC_PLAIN)
    assert kern == "simt_gemm", kern
    assert _lib.launch_count() - n0 == 2      # the split GEMM and the fixed-order reduction
    err = _check(oracle_c, q, a, b, got, md)
    assert err <= TOL[dtype], (case, err)
    _, _, again, _, _ = _run(cuda, na, pia, q, m, b_cm, dtype, precision=_lib.PREC_PLAIN, a=a, b=b)
    assert np.array_equal(got, again)


def test_split_k_replaces_a_single_block_tensor_core_launch(cuda, oracle_c):
    """Under auto, a shape whose bf16x3 tiles would fill a handful of SMs runs the split-K SIMT
    GEMM instead (exact, and faster for such shapes)."""
    a, b, got, md, kern = _run(cuda, [128, 16384], [1, 2], 2, 64, True, np.float32, precision=_lib.PREC_AUTO)
    assert kern == "simt_gemm", kern
    assert _check(oracle_c, 2, a, b, got, md) <= TOL[np.float32]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_order_one_full_size_known_answer(cuda, dtype):
    """c = B a with n = 2^26 and m = 64 (B holds 2^32 elements): integer entries and a with eight
    non-zeros make every output an exact integer, so the result must match bit for bit."""
    import torch
    n, m = 1 << 26, 64
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(n, 8, replace=False))
    coef = rng.integers(-5, 6, 8)
    g = torch.Generator(device=cuda).manual_seed(2)
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    B = torch.randint(-8, 9, (n, m), device=cuda, generator=g).to(tdt)      # [l][j]: column-major (m, n)
    a = torch.zeros(n, device=cuda, dtype=tdt)
    a[torch.from_numpy(idx).to(cuda)] = torch.from_numpy(coef.astype(dtype)).to(cuda)
    c = torch.full((m,), float("nan"), device=cuda, dtype=tdt)
    _lib.ttm_raw(_lib.F32 if dtype == np.float32 else _lib.F64, _lib.PREC_DEFAULT, 1, 1, a.data_ptr(), [n], [1], [1],
                 B.data_ptr(), [m, n], [1, 2], c.data_ptr(), [m], [1], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _lib.last_kernel() == "bvec"
    cols = B[torch.from_numpy(idx).to(cuda)].double().cpu().numpy()     # the 8 columns of B used
    want = (coef.astype(np.float64)[:, None] * cols).sum(0)
    assert np.array_equal(c.double().cpu().numpy(), want)
