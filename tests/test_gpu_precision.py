"""The 8-bit tensor-core paths through the C ABI on a CUDA device.

ozaki (double): within 1e-12 relative Frobenius error of the FP64 oracle (the required bound),
on N(0,1) data and on magnitudes log-uniform over [1e-4, 1e4]; exact on small integers.
fp8 (float): within 1e-4 of the same product with the operands rounded as the path rounds them
(tests/emulation.py), so the check is on the kernels, not on e4m3's own error; that error is
reported separately against the exact product.
"""
import numpy as np
import pytest

import known_answer as ka
from emulation import fp8_ttm
from ttm_b200 import _lib

pytestmark = pytest.mark.gpu

# (na, pia, q, m, pib): strided fibres, permuted layouts, q = pi_1 (rows are slices k),
# several l chunks, n_q = 1, m across N tiles (fp8 256 columns, ozaki 64)
CASES = [([64, 48, 40], [1, 2, 3], 2, 64, [1, 2]),
         ([64, 48, 40], [3, 1, 2], 1, 100, [2, 1]),
         ([300, 33, 7], [1, 2, 3], 1, 17, [1, 2]),
         ([20, 30, 40, 6], [1, 2, 3, 4], 3, 256, [2, 1]),
         ([16, 1000, 8], [1, 2, 3], 2, 40, [1, 2]),
         ([5, 1, 7], [1, 2, 3], 2, 20, [1, 2]),
         ([33, 65, 3, 9], [4, 2, 1, 3], 2, 300, [2, 1])]


def relerr(x, ref):
    ref = np.asarray(ref, dtype=np.float64)
    return np.linalg.norm(np.asarray(x, dtype=np.float64) - ref) / max(np.linalg.norm(ref), 1e-300)


def md_of(na, pia, q, m, pib):
    nc = list(na)
    nc[q - 1] = m
    return dict(na=na, wa=ka.dense_strides(na, pia), pia=pia, nb=[m, na[q - 1]], pib=pib, nc=nc,
                wc=ka.dense_strides(nc, pia))


def run_device(q, a, md, b, prec, dev):
    import torch
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    tc = torch.full((int(np.prod(md["nc"])),), float("nan"), dtype=ta.dtype, device=dev)
    dt = _lib.F32 if a.dtype == np.float32 else _lib.F64
    _lib.ttm_raw(dt, prec, q, len(md["na"]), ta.data_ptr(), md["na"], md["wa"], md["pia"], tb.data_ptr(),
                 md["nb"], md["pib"], tc.data_ptr(), md["nc"], md["wc"], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return tc.cpu().numpy()


def logical(flat, n, w):
    return np.lib.stride_tricks.as_strided(flat, shape=n, strides=[flat.itemsize * x for x in w])


def b_matrix(b, md):
    m, nq = md["nb"]
    return b.reshape(nq, m).T if md["pib"][0] == 1 else b.reshape(m, nq)


def draw(rng, n, dist, dtype):
    if dist == "normal":
        return rng.standard_normal(n).astype(dtype)
    if dist == "loguniform":
        return (rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-4, 4, n)).astype(dtype)
    return rng.integers(-8, 9, n).astype(dtype)


@pytest.mark.parametrize("dist", ["normal", "loguniform", "integers"])
def test_ozaki_vs_fp64_oracle(cuda, oracle_c, dist):
    rng = np.random.default_rng(5)
    for na, pia, q, m, pib in CASES:
        md = md_of(na, pia, q, m, pib)
        a = draw(rng, int(np.prod(na)), dist, np.float64)
        b = draw(rng, m * na[q - 1], dist, np.float64)
        c = run_device(q, a, md, b, _lib.PREC_OZAKI, cuda)
        assert _lib.last_kernel() == "tc_ozaki"
        ref = np.zeros(int(np.prod(md["nc"])))
        oracle_c.ttm(q, a, na, md["wa"], pia, b, md["nb"], pib, ref, md["nc"], md["wc"])
        if dist == "integers":
            assert np.array_equal(c, ref), (na, q, m)      # every digit product and sum is exact
        else:
            assert relerr(c, ref) <= 1e-12, (na, q, m, relerr(c, ref))


@pytest.mark.parametrize("dist", ["normal", "loguniform", "integers"])
def test_fp8_vs_emulated_rounding(cuda, dist):
    rng = np.random.default_rng(6)
    for na, pia, q, m, pib in CASES:
        md = md_of(na, pia, q, m, pib)
        a = draw(rng, int(np.prod(na)), dist, np.float32)
        b = draw(rng, m * na[q - 1], dist, np.float32)
        c = run_device(q, a, md, b, _lib.PREC_FP8, cuda)
        assert _lib.last_kernel() in ("tc_fp8", "tc_fp8_pair")
        A = logical(a, na, md["wa"])
        want = fp8_ttm(q, A, b_matrix(b, md))
        C = logical(c, md["nc"], md["wc"])
        if dist == "integers":
            assert np.array_equal(C, want), (na, q, m)      # |x| <= 8 is exact in e4m3
        else:
            assert relerr(C, want) <= 1e-4, (na, q, m, relerr(C, want))
            exact = np.moveaxis(np.tensordot(A.astype(np.float64), b_matrix(b, md).astype(np.float64),
                                             axes=([q - 1], [1])), -1, q - 1)
            assert 1e-4 < relerr(C, exact) < 0.1, (na, q, m, relerr(C, exact))


def test_small_m_and_out_of_range_take_the_exact_kernels(cuda):
    """m <= 16 runs the bandwidth kernels whatever the precision; fp8 on double and ozaki on
    float are refused."""
    rng = np.random.default_rng(7)
    md = md_of([64, 48, 40], [1, 2, 3], 2, 8, [1, 2])
    a = rng.standard_normal(64 * 48 * 40)
    b = rng.standard_normal(8 * 48)
    run_device(2, a, md, b, _lib.PREC_OZAKI, cuda)
    assert _lib.last_kernel() in ("colvec", "stream_cols")
    md = md_of([64, 48, 40], [1, 2, 3], 2, 32, [1, 2])
    b = rng.standard_normal(32 * 48)
    with pytest.raises(_lib.TtmError):
        run_device(2, a, md, b, _lib.PREC_FP8, cuda)
    with pytest.raises(_lib.TtmError):
        run_device(2, a.astype(np.float32), md, b.astype(np.float32), _lib.PREC_OZAKI, cuda)


def test_precision_study_small(cuda):
    """The study driver on a small instance: every path reports errors against the FP64 kernel
    in the expected order of accuracy."""
    from ttm_b200.precision import study
    res = study(size=32, m=40, reps=1, log=lambda s: None)
    assert len(res["cases"]) == 8
    for case in res["cases"]:
        p = case["paths"]
        assert p["fp64_native"]["kernel"] == "simt_gemm"
        assert p["ozaki"]["rms_rel"] <= 1e-12
        assert p["plain_fp32"]["rms_rel"] <= 1e-5 and p["bf16x3"]["rms_rel"] <= 1e-5
        assert p["bf16x3"]["kernel"].startswith("tc_bf16x3") and p["fp8"]["kernel"] == "tc_fp8"
        assert 1e-4 < p["fp8"]["rms_rel"] < 0.1
        assert p["ozaki"]["max_rel"] <= p["plain_fp32"]["max_rel"] <= p["fp8"]["max_rel"]


# (na, pia, q, m, pib): shapes of the one-launch fp8 kernel on SM pairs (128 < m <= 256,
# n_q <= 256, rows of >= 128 i or contiguous fibres): one and several 64-l stages, n_q not a
# multiple of 32 or 64, partial tiles, both B layouts
PAIR8_CASES = [([256, 40, 6], [1, 2, 3], 2, 200, [1, 2]),
               ([200, 96, 3], [1, 2, 3], 2, 256, [2, 1]),
               ([132, 256, 2], [1, 2, 3], 2, 130, [1, 2]),
               ([64, 200, 50], [2, 1, 3], 2, 160, [2, 1]),
               ([48, 36, 100], [2, 1, 3], 2, 256, [1, 2]),
               ([128, 64, 256], [3, 1, 2], 1, 250, [2, 1])]


@pytest.mark.parametrize("dist", ["normal", "loguniform", "integers"])
def test_fp8_pair_kernel_vs_emulated_rounding(cuda, dist):
    """The one-launch fp8 kernel (fibre scales found from the tile in shared memory) rounds every
    operand exactly as the separate path does: integers come out exact, other data within the
    FP32 accumulation of the emulated product; all-zero fibres (exponent 0) included."""
    rng = np.random.default_rng(16)
    for n, (na, pia, q, m, pib) in enumerate(PAIR8_CASES):
        md = md_of(na, pia, q, m, pib)
        a = draw(rng, int(np.prod(na)), dist, np.float32)
        b = draw(rng, m * na[q - 1], dist, np.float32)
        A = logical(a, na, md["wa"])
        if n == 0:
            np.moveaxis(A, q - 1, -1)[3, :, :] = 0.0      # a run of all-zero fibres
        c = run_device(q, a, md, b, _lib.PREC_FP8, cuda)
        assert _lib.last_kernel() == "tc_fp8_pair", (na, q, m)
        want = fp8_ttm(q, A, b_matrix(b, md))
        C = logical(c, md["nc"], md["wc"])
        if dist == "integers":
            assert np.array_equal(C, want), (na, q, m)
        else:
            assert relerr(C, want) <= 1e-5, (na, q, m, relerr(C, want))
