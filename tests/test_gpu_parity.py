"""Parity of the CUDA path with the oracle, through the C ABI, on a CUDA device.

Tolerances: plain FP64 within 1e-13 and plain FP32 within 2e-6 relative
Frobenius error of each case against the reference's own outputs / the oracle
(the required bound for plain FP32 is 1e-5); exact-integer known answers
within 4 ULP as in the reference's unit test.
"""
import os

import numpy as np
import pytest

from cases import golden_cases, make_inputs
import known_answer as ka
from ttm_b200 import _lib
from ttm_b200 import ttmpy as tp

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_outputs.npz")


def relerr(x, ref):
    ref = np.asarray(ref, dtype=np.float64)
    d = np.linalg.norm(np.asarray(x, dtype=np.float64) - ref)
    return d / max(np.linalg.norm(ref), 1e-300)


def abi_host(q, a, md, b, precision=_lib.PREC_PLAIN):
    c = np.full(int(np.prod(md["nc"])), np.nan, dtype=a.dtype)
    dt = _lib.F32 if a.dtype == np.float32 else _lib.F64
    _lib.ttm_raw(dt, precision, q, len(md["na"]), a.ctypes.data, md["na"], md["wa"], md["pia"], b.ctypes.data,
                 md["nb"], md["pib"], c.ctypes.data, md["nc"], md["wc"])
    return c


def abi_device(q, a, md, b, dev, precision=_lib.PREC_PLAIN):
    import torch
    ta = torch.from_numpy(a).to(dev)
    tb = torch.from_numpy(b).to(dev)
    tc = torch.full((int(np.prod(md["nc"])),), float("nan"), dtype=ta.dtype, device=dev)
    dt = _lib.F32 if a.dtype == np.float32 else _lib.F64
    _lib.ttm_raw(dt, precision, q, len(md["na"]), ta.data_ptr(), md["na"], md["wa"], md["pia"], tb.data_ptr(),
                 md["nb"], md["pib"], tc.data_ptr(), md["nc"], md["wc"], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return tc.cpu().numpy()


def test_golden_fixtures_host_pointers(cuda):
    gold = np.load(GOLDEN)
    for case in golden_cases():
        a, b, md = make_inputs(case)
        c = abi_host(case["q"], a, md, b)
        tol = 1e-13 if case["dtype"] == "f64" else 2e-6
        assert relerr(c, gold[f"c{case['id']}"]) <= tol, case


def test_golden_fixtures_device_pointers(cuda):
    gold = np.load(GOLDEN)
    for case in golden_cases()[::3]:
        a, b, md = make_inputs(case)
        c = abi_device(case["q"], a, md, b, cuda)
        tol = 1e-13 if case["dtype"] == "f64" else 2e-6
        assert relerr(c, gold[f"c{case['id']}"]) <= tol, case


@pytest.mark.parametrize("rank", [2, 3, 4])
def test_known_answers(cuda, rank):
    """test/src/gtest_tlib_ttm.cpp:137-259 restated: all shapes in {2,4,8}^p, all layouts, all q, both B layouts."""
    for na in ka.shapes(rank):
        for pia in ka.layouts(rank):
            for q in range(1, rank + 1):
                nq = na[q - 1]
                m = 2 * nq
                a = ka.init_a(na, pia, q)
                nc = list(na)
                nc[q - 1] = m
                md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], nc=nc,
                          wc=ka.dense_strides(nc, pia))
                want = ka.expected_c(na, pia, q, m)
                b = np.ones(m * nq)
                for pib in ([2, 1], [1, 2]):
                    md["pib"] = pib
                    c = abi_host(q, a, md, b)
                    assert ka.ulp_close(c, want), (na, pia, q, pib)


def _random_problem(rng, p, total_log2, dtype):
    # random split of total_log2 bits over p extents, each >= 2
    bits = np.ones(p, dtype=int)
    for _ in range(total_log2 - p):
        bits[rng.integers(0, p)] += 1
    return [int(2 ** x) for x in bits]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_layout_mode_sweep_vs_oracle(cuda, oracle_c, dtype):
    """A reduced-size instance of the layout/mode sweep: p in 3..6, all q, first/last/random layouts,
    m in {1, 8, 64, 512}, N(0,1) entries, against the C oracle."""
    rng = np.random.default_rng(11)
    worst = 0.0
    for p in (3, 4, 5, 6):
        na = _random_problem(rng, p, 16, dtype)
        lays = [list(range(1, p + 1)), list(range(p, 0, -1)), [int(x) + 1 for x in rng.permutation(p)]]
        for pia in lays:
            for q in range(1, p + 1):
                for m in (1, 8, 64, 512):
                    nq = na[q - 1]
                    nc = list(na)
                    nc[q - 1] = m
                    md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq],
                              pib=[1, 2] if (m + q) % 2 else [2, 1], nc=nc, wc=ka.dense_strides(nc, pia))
                    a = rng.standard_normal(int(np.prod(na))).astype(dtype)
                    b = rng.standard_normal(m * nq).astype(dtype)
                    c = abi_host(q, a, md, b)
                    ref = np.zeros(int(np.prod(nc)), dtype=dtype)
                    oracle_c.ttm(q, a, md["na"], md["wa"], pia, b, md["nb"], md["pib"], ref, nc, md["wc"])
                    worst = max(worst, relerr(c, ref))
    assert worst <= (1e-13 if dtype == np.float64 else 2e-6), worst


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stream_cols_box_shapes(cuda, oracle_c, dtype):
    """The TMA-fed small-m kernel packs KB = P / IB slices into one box when inner is small, folds
    a large inner into (i mod IB, i / IB) boxes when there are few slices, and splits the l range
    (partial tiles added by the last unit) when tiles are few or B is large. Cover each box mode,
    partial boxes in i, k and l, B restaged per unit, every m bucket and both B layouts; shapes
    the kernel declines (mostly out-of-range fill) must take another kernel."""
    import torch
    from ttm_b200.selector import lib
    rng = np.random.default_rng(21)
    shapes = [(4, 300, 5, 1), (4, 1000, 70, 16), (8, 257, 33, 8), (12, 700, 16, 3), (36, 120, 9, 2),
              (64, 37, 33, 8), (64, 130, 1000, 1), (100, 256, 16, 4), (128, 37, 33, 8), (260, 256, 5, 1),
              (256, 4, 3000, 16), (512, 2, 1000, 1), (4096, 1, 37, 8), (1536, 2, 9, 2), (65536, 1, 3, 1),
              (8192, 3, 20, 4), (96, 1, 50, 16), (4, 3, 16, 3),
              (64, 200, 1, 4), (4, 1000, 2, 8), (128, 40, 3, 16)]       # n_q below one box of l
    if dtype == np.float64:
        shapes += [(2, 512, 7, 2), (6, 256, 9, 8)]
    dt = _lib.F32 if dtype == np.float32 else _lib.F64
    taken = []
    for n, (inner, outer, nq, m) in enumerate(shapes):
        na = [inner, nq, outer]
        nc = [inner, m, outer]
        pia = [1, 2, 3]
        md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2] if n % 2 else [2, 1],
                  nc=nc, wc=ka.dense_strides(nc, pia))
        a = rng.standard_normal(int(np.prod(na))).astype(dtype)
        b = rng.standard_normal(m * nq).astype(dtype)
        ta, tb = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
        tc = torch.full((int(np.prod(nc)),), float("nan"), dtype=ta.dtype, device=cuda)
        rc = lib().tlibttm_ttm_sched(dt, 6, 2, 3, ta.data_ptr(), _lib.sz(na), _lib.sz(md["wa"]), _lib.sz(pia),
                                     tb.data_ptr(), _lib.sz(md["nb"]), _lib.sz(md["pib"]), tc.data_ptr(), _lib.sz(nc),
                                     _lib.sz(md["wc"]), None)
        valid = lib().tlibttm_schedule_valid(dt, 6, 2, 3, _lib.sz(na), _lib.sz(pia), m)
        assert rc == (0 if valid else _lib.ERR_UNSUPPORTED), (inner, outer, nq, m, rc)
        if not valid:
            continue
        assert _lib.last_kernel() == "stream_cols"
        taken.append((inner, outer))
        c = tc.cpu().numpy()
        ref = np.zeros(int(np.prod(nc)), dtype=dtype)
        oracle_c.ttm(2, a, na, md["wa"], pia, b, md["nb"], md["pib"], ref, nc, md["wc"])
        assert relerr(c, ref) <= (1e-14 if dtype == np.float64 else 2e-6), (inner, outer, nq, m)
    # the folded boxes, the restaged B and the narrow-row boxes were all exercised
    for want in ((4096, 1), (65536, 1), (512, 2), (256, 4), (4, 1000), (64, 200), (128, 40)):
        assert want in taken, want
    assert (96, 1) not in taken and (4, 3) not in taken


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stream_cols_two_ctas_per_sm(cuda, oracle_c, dtype):
    """Column mode with at least as many tiles as SMs and m <= 8 runs the 96-register build two
    CTAs per SM with 48 KB rings; cover it with one unit per tile and with the l range split three
    (float) or two (double) ways (128 x 1280 slices, n_q 256, m 2), several units per CTA, and the
    m buckets 1, 4 and 8."""
    import torch
    from ttm_b200.selector import lib
    rng = np.random.default_rng(22)
    shapes = [(256, 1024, 8, 8), (64, 4096, 20, 3), (128, 1280, 256, 2), (512, 384, 40, 8), (256, 640, 64, 1)]
    dt = _lib.F32 if dtype == np.float32 else _lib.F64
    for n, (inner, outer, nq, m) in enumerate(shapes):
        na = [inner, nq, outer]
        nc = [inner, m, outer]
        pia = [1, 2, 3]
        md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2] if n % 2 else [2, 1],
                  nc=nc, wc=ka.dense_strides(nc, pia))
        a = rng.standard_normal(int(np.prod(na))).astype(dtype)
        b = rng.standard_normal(m * nq).astype(dtype)
        ta, tb = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
        tc = torch.full((int(np.prod(nc)),), float("nan"), dtype=ta.dtype, device=cuda)
        rc = lib().tlibttm_ttm_sched(dt, 6, 2, 3, ta.data_ptr(), _lib.sz(na), _lib.sz(md["wa"]), _lib.sz(pia),
                                     tb.data_ptr(), _lib.sz(md["nb"]), _lib.sz(md["pib"]), tc.data_ptr(), _lib.sz(nc),
                                     _lib.sz(md["wc"]), None)
        assert rc == 0 and _lib.last_kernel() == "stream_cols", (inner, outer, nq, m, rc)
        c = tc.cpu().numpy()
        ref = np.zeros(int(np.prod(nc)), dtype=dtype)
        oracle_c.ttm(2, a, na, md["wa"], pia, b, md["nb"], md["pib"], ref, nc, md["wc"])
        assert relerr(c, ref) <= (1e-14 if dtype == np.float64 else 2e-6), (inner, outer, nq, m)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stream_rows_contiguous_fibres(cuda, oracle_c, dtype):
    """The TMA-fed small-m kernel in row mode (q = pi_1, contiguous fibres) through schedule 6:
    partial l chunks, row counts off the 512-row tile (second box partly or wholly past the end), few tiles (l split with partial tiles added
    by the last unit), a B restaged per unit, every m bucket; fibres that are too short or not
    16-byte aligned are declined."""
    import torch
    from ttm_b200.selector import lib
    rng = np.random.default_rng(41)
    dt = _lib.F32 if dtype == np.float32 else _lib.F64
    cases = [(20, 1000, 1), (256, 3000, 8), (64, 257, 16), (1000, 50, 3), (4096, 10, 2), (68, 70000, 4),
             (3000, 7, 16), (16, 513, 5), (16, 100000, 8)]
    if dtype == np.float64:
        cases += [(18, 600, 5)]
    declined = [(4, 1000, 1), (18, 100, 2)] if dtype == np.float32 else [(2, 1000, 1), (9, 100, 2)]
    for n, (nq, outer, m) in enumerate(cases + declined):
        na, pia, nc = [nq, outer], [1, 2], [m, outer]
        md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2] if n % 2 else [2, 1],
                  nc=nc, wc=ka.dense_strides(nc, pia))
        a = rng.standard_normal(nq * outer).astype(dtype)
        b = rng.standard_normal(m * nq).astype(dtype)
        ta, tb = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
        tc = torch.full((m * outer,), float("nan"), dtype=ta.dtype, device=cuda)
        rc = lib().tlibttm_ttm_sched(dt, 6, 1, 2, ta.data_ptr(), _lib.sz(na), _lib.sz(md["wa"]), _lib.sz(pia),
                                     tb.data_ptr(), _lib.sz(md["nb"]), _lib.sz(md["pib"]), tc.data_ptr(), _lib.sz(nc),
                                     _lib.sz(md["wc"]), None)
        if (nq, outer, m) in declined:
            assert rc == _lib.ERR_UNSUPPORTED, (nq, outer, m)
            continue
        assert rc == 0 and _lib.last_kernel() == "stream_rows", (nq, outer, m, rc)
        ref = np.zeros(m * outer, dtype=dtype)
        oracle_c.ttm(1, a, na, md["wa"], pia, b, md["nb"], md["pib"], ref, nc, md["wc"])
        assert relerr(tc.cpu().numpy(), ref) <= (1e-14 if dtype == np.float64 else 2e-6), (nq, outer, m)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_short_contiguous_fibres(cuda, oracle_c, dtype):
    """q = pi_1 with n_q <= 16: rows of A are short and contiguous (the span and flat-tile row
    kernels); row counts that are not multiples of a span or a warp's tile, n_q = 1, every m bucket,
    both B layouts."""
    rng = np.random.default_rng(31)
    # n_q in {1, 2, 4, 8, 16}: the span kernel (tail spans, m below its bucket, vector and scalar
    # stores); other lengths: the flat-tile kernel
    # (12, 20001, 16) and (16, 3001, 9): staged outputs whose double build needs more than 48 KB of
    # shared memory (the launch opts in)
    for n, (nq, outer, m) in enumerate(((1, 5000, 1), (2, 70001, 8), (3, 4099, 3), (5, 12345, 16), (16, 33333, 2),
                                        (16, 31, 5), (7, 100000, 1), (4, 9999, 4), (8, 777, 16), (4, 100003, 1),
                                        (8, 5001, 3), (1, 333, 16), (12, 20001, 16), (16, 3001, 9))):
        na = [nq, outer]
        pia = [1, 2]
        nc = [m, outer]
        md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2] if n % 2 else [2, 1],
                  nc=nc, wc=ka.dense_strides(nc, pia))
        a = rng.standard_normal(nq * outer).astype(dtype)
        b = rng.standard_normal(m * nq).astype(dtype)
        c = abi_device(1, a, md, b, cuda)
        assert _lib.last_kernel() == "rowdot"
        ref = np.zeros(m * outer, dtype=dtype)
        oracle_c.ttm(1, a, na, md["wa"], pia, b, md["nb"], md["pib"], ref, nc, md["wc"])
        assert relerr(c, ref) <= (1e-14 if dtype == np.float64 else 2e-6), (nq, outer, m)


def test_kernel_selection_and_strided(cuda):
    rng = np.random.default_rng(3)
    # rowdot: q = pi_1 (inner == 1), small m
    cases = [([64, 32, 16], [1, 2, 3], 1, 4, "rowdot"),
             ([64, 32, 16], [1, 2, 3], 2, 8, "colvec"),
             ([256, 64, 512], [1, 2, 3], 2, 8, "stream_cols"),
             ([256, 64, 512], [1, 2, 3], 1, 4, "stream_rows"),
             ([257, 64, 512], [1, 2, 3], 2, 8, "colvec"),
             ([64, 32, 16], [1, 2, 3], 2, 40, "simt_gemm"),
             ([64, 32, 16], [2, 3, 1], 2, 40, "simt_gemm")]
    for na, pia, q, m, kern in cases:
        nq = na[q - 1]
        nc = list(na)
        nc[q - 1] = m
        md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, nq], pib=[1, 2], nc=nc,
                  wc=ka.dense_strides(nc, pia))
        a = rng.standard_normal(int(np.prod(na)))
        b = rng.standard_normal(m * nq)
        # device operands: host ones above 64 MB are staged in pieces, which changes the choice
        c = abi_device(q, a, md, b, cuda)
        assert _lib.last_kernel() == kern
        A = np.lib.stride_tricks.as_strided(a, shape=na, strides=[8 * w for w in md["wa"]])
        Bm = b.reshape(nq, m).T
        want = np.moveaxis(np.tensordot(A, Bm, axes=([q - 1], [1])), -1, q - 1)
        C = np.lib.stride_tricks.as_strided(c, shape=nc, strides=[8 * w for w in md["wc"]])
        assert np.allclose(C, want, rtol=1e-12, atol=1e-12)
    # non-dense (padded) strides take the strided kernel and keep the gaps of C
    na, pia, q, m = [5, 6, 7], [1, 2, 3], 2, 9
    wa = [1, 8, 64]            # mode 1 padded to 8, mode 2 padded to 8
    nc = [5, 9, 7]
    wc = [1, 6, 60]            # mode 1 padded to 6, mode 2 padded to 10
    a = rng.standard_normal(1 + 4 * 1 + 5 * 8 + 6 * 64)
    b = rng.standard_normal(m * 6)
    span_c = 1 + 4 * 1 + 8 * 6 + 6 * 60
    c = np.full(span_c, 7.5)
    _lib.ttm_raw(_lib.F64, _lib.PREC_PLAIN, q, 3, a.ctypes.data, na, wa, pia, b.ctypes.data, [m, 6], [2, 1],
                 c.ctypes.data, nc, wc)
    assert _lib.last_kernel() == "strided"
    A = np.lib.stride_tricks.as_strided(a, shape=na, strides=[8 * w for w in wa])
    want = np.moveaxis(np.tensordot(A, b.reshape(m, 6), axes=([1], [1])), -1, 1)
    C = np.lib.stride_tricks.as_strided(c, shape=nc, strides=[8 * w for w in wc])
    assert np.allclose(C, want, rtol=1e-12, atol=1e-12)
    mask = np.ones(span_c, bool)
    idx = (np.arange(5)[:, None, None] + 6 * np.arange(9)[None, :, None] + 60 * np.arange(7)[None, None, :])
    mask[idx.reshape(-1)] = False
    assert np.all(c[mask] == 7.5)


def test_a256_cube_q2_m128_full_size(cuda, oracle_c):
    """A 256^3 first-order, q=2, B (128, 256) column-major, U[-1,1] from seed 0 (the reference's CPU case)."""
    rng = np.random.default_rng(0)
    na, pia, q, m = [256, 256, 256], [1, 2, 3], 2, 128
    a = rng.uniform(-1, 1, 256 ** 3).astype(np.float32)
    b = rng.uniform(-1, 1, m * 256).astype(np.float32)
    nc = [256, m, 256]
    md = dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, 256], pib=[1, 2], nc=nc,
              wc=ka.dense_strides(nc, pia))
    c = abi_host(q, a, md, b)
    ref = np.zeros(len(c), dtype=np.float32)
    oracle_c.ttm(q, a, na, md["wa"], pia, b, md["nb"], md["pib"], ref, nc, md["wc"])
    assert relerr(c, ref) <= 1e-6


def test_64bit_indexing_sampled_fibres(cuda):
    """More than 2^31 elements (8.7 GB fp32): sampled fibres against float64 dot products."""
    import torch
    na = [256, 256, 256, 130]
    q, m = 2, 64
    g = torch.Generator(device=cuda).manual_seed(5)
    A = torch.randn(130, 256, 256, 256, device=cuda, generator=g)   # memory order (mode4, mode3, mode2, mode1)
    B = torch.randn(256, m, device=cuda, generator=g)               # column-major (m, nq): element (j,l) at j + l*m
    C = torch.empty(130, 256, m, 256, device=cuda)
    pia = [1, 2, 3, 4]
    wa = ka.dense_strides(na, pia)
    nc = [256, m, 256, 130]
    wc = ka.dense_strides(nc, pia)
    _lib.ttm_raw(_lib.F32, _lib.PREC_PLAIN, q, 4, A.data_ptr(), na, wa, pia, B.data_ptr(), [m, 256], [1, 2],
                 C.data_ptr(), nc, wc, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    rng = np.random.default_rng(1)
    Bh = B.double().cpu().numpy()          # [l][j]
    for _ in range(40):
        i4, i3, i1 = int(rng.integers(130)), int(rng.integers(256)), int(rng.integers(256))
        fib = A[i4, i3, :, i1].double().cpu().numpy()
        want = fib @ Bh
        got = C[i4, i3, :, i1].double().cpu().numpy()
        assert relerr(got, want) <= 2e-6
    del A, C
    torch.cuda.empty_cache()


def test_ttmpy_reference_cases(cuda):
    """ttmpy/tests/test.py restated: exact equality with einsum on arange inputs."""
    A = np.arange(3 * 2 * 4, dtype=np.float64).reshape(3, 2, 4)
    for q, spec, nb in ((1, "ijk,xi->xjk", (5, 3)), (2, "ijk,xj->ixk", (5, 2)), (3, "ijk,xk->ijx", (5, 4))):
        B = np.arange(nb[0] * nb[1], dtype=np.float64).reshape(nb)
        assert np.all(tp.ttm(q, A, B) == np.einsum(spec, A, B))
    A = np.arange(3 * 2 * 4 * 5, dtype=np.float64).reshape(3, 2, 4, 5)
    specs = {1: "ijkl,yi->yjkl", 2: "ijkl,yj->iykl", 3: "ijkl,yk->ijyl", 4: "ijkl,yl->ijky"}
    for q in range(1, 5):
        modes = [r for r in range(1, 5) if r != q]
        Bs = []
        D = A
        for idx, r in enumerate(modes):
            mr = (6, 7, 9)[idx]        # the reference's matrices are (6,.), (7,.), (9,.) in list order
            Br = np.arange(mr * A.shape[r - 1], dtype=np.float64).reshape(mr, A.shape[r - 1])
            Bs.append(Br)
            D = np.einsum(specs[r], D, Br)
        for order in ("forward", "backward", "optimal"):
            C = tp.ttms(q, A, Bs, order)
            assert np.all(C == D), (q, order)


def test_ttmpy_torch_and_permuted_views(cuda):
    import torch
    rng = np.random.default_rng(9)
    A = rng.standard_normal((6, 5, 7))
    B = rng.standard_normal((4, 5))
    want = np.einsum("ijk,xj->ixk", A, B)
    got = tp.ttm(2, torch.from_numpy(A).to(cuda), torch.from_numpy(B).to(cuda))
    assert got.is_cuda and np.allclose(got.cpu().numpy(), want, rtol=1e-12, atol=1e-12)
    # permuted (non C-ordered) numpy view and a column-major B
    At = np.transpose(rng.standard_normal((7, 5, 6)), (2, 1, 0))
    Bf = np.asfortranarray(B)
    assert np.allclose(tp.ttm(2, At, Bf), np.einsum("ijk,xj->ixk", At, Bf), rtol=1e-12, atol=1e-12)
    A32 = A.astype(np.float32)
    assert np.allclose(tp.ttm(2, A32, B.astype(np.float32)), np.einsum("ijk,xj->ixk", A32, B), rtol=1e-5,
                       atol=1e-5)


@pytest.mark.parametrize("dtype,prec", [(np.float32, _lib.PREC_PLAIN), (np.float32, _lib.PREC_BF16X3),
                                        (np.float64, _lib.PREC_PLAIN)])
@pytest.mark.parametrize("q", [1, 2, 3])
def test_pipelined_host_staging(cuda, dtype, prec, q):
    """Large host operands go through the chunked, overlapped copy-in / compute / copy-out path
    (chunks of whole slices when there are many, column blocks of each slice when there are few)."""
    import torch
    na, pia = [256, 256, 320], [1, 2, 3]    # 84 MB fp32; q=1,2: many slices; q=3: one slice, column blocks
    nq = na[q - 1]
    m = 48
    nc = list(na)
    nc[q - 1] = m
    wa, wc = ka.dense_strides(na, pia), ka.dense_strides(nc, pia)
    rng = np.random.default_rng(q)
    a = torch.from_numpy(rng.standard_normal(int(np.prod(na))).astype(dtype)).pin_memory()
    b = rng.standard_normal(m * nq).astype(dtype)
    c = torch.full((int(np.prod(nc)),), float("nan"), dtype=a.dtype).pin_memory()
    if a.numel() * a.element_size() < (64 << 20):
        pytest.skip("below the pipelining threshold")
    dt = _lib.F32 if dtype == np.float32 else _lib.F64
    _lib.ttm_raw(dt, prec, q, 3, a.data_ptr(), na, wa, pia, b.ctypes.data, [m, nq], [1, 2], c.data_ptr(), nc, wc)
    qh = pia.index(q)
    inner = int(np.prod([na[pia[r] - 1] for r in range(qh)]))
    outer = int(np.prod(na)) // (inner * nq)
    A3 = a.numpy().astype(np.float64).reshape(outer, nq, inner)
    want = np.matmul(b.astype(np.float64).reshape(nq, m).T, A3).reshape(-1)
    tol = 1e-5 if prec == _lib.PREC_BF16X3 else (2e-6 if dtype == np.float32 else 1e-13)
    assert relerr(c.numpy(), want) <= tol


UNALIGNED_COLUMN_CASES = [
    # (na, pia, q, m): strided rows not on 16-byte boundaries (the column kernel's cp.async ring)
    ([99, 3001, 7], [1, 2, 3], 2, 5),     # 693 rows: the l range split over the warps of a block
    ([99, 3001, 7], [1, 2, 3], 2, 16),
    ([301, 20, 600], [1, 2, 3], 2, 3),    # 180600 rows: one row per lane, no split
    ([3, 513, 37], [2, 1, 3], 3, 9),      # inner 1539 over two modes, n_q not a multiple of 8
]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("case", UNALIGNED_COLUMN_CASES)
def test_unaligned_column_kernel(cuda, oracle_c, case, dtype):
    """Rows of i that are not 16-byte aligned take the column kernel whose threads stream their
    rows through a shared-memory ring of asynchronous copies; exact FMA against the C oracle."""
    import torch
    na, pia, q, m = case
    rng = np.random.default_rng(7)
    nq = na[q - 1]
    nc = list(na)
    nc[q - 1] = m
    wa, wc = ka.dense_strides(na, pia), ka.dense_strides(nc, pia)
    a = rng.standard_normal(int(np.prod(na))).astype(dtype)
    b = rng.standard_normal(m * nq).astype(dtype)
    ta, tb = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    tc = torch.full((int(np.prod(nc)),), float("nan"), device=cuda, dtype=ta.dtype)
    _lib.ttm_raw(_lib.F32 if dtype == np.float32 else _lib.F64, _lib.PREC_DEFAULT, q, len(na), ta.data_ptr(), na, wa,
                 pia, tb.data_ptr(), [m, nq], [1, 2], tc.data_ptr(), nc, wc, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _lib.last_kernel() == "colvec", _lib.last_kernel()
    ref = np.zeros(int(np.prod(nc)), dtype=dtype)
    oracle_c.ttm(q, a, na, wa, pia, b, [m, nq], [1, 2], ref, nc, wc)
    assert relerr(tc.cpu().numpy(), ref) <= (1e-13 if dtype == np.float64 else 2e-6)
