"""bf16x3 tensor-core path (tcgen05): FP32-accurate results from BF16 products.

Bar: relative Frobenius error <= 1e-5 against the FP64-accumulated oracle on
N(0,1) data (the required accuracy of the split-BF16 path), over both
tile geometries (i-contiguous slices and q = pi_1), partial tiles in every
dimension, m above and below one MMA N tile, and both B layouts.
"""
import numpy as np
import pytest

import known_answer as ka
from ttm_b200 import _lib

pytestmark = pytest.mark.gpu


def run(dev, na, pia, q, m, b_cm, dist="normal", seed=0, precision=_lib.PREC_BF16X3, schedule=None, c_off=0):
    """One bf16x3 contraction through the C ABI (by precision, or by a named schedule) against an
    FP64 reference; `c_off` shifts C by that many floats off its 16-byte alignment."""
    import ctypes as C
    import torch
    rng = np.random.default_rng(seed)
    nq = na[q - 1]
    nc = list(na)
    nc[q - 1] = m
    wa, wc = ka.dense_strides(na, pia), ka.dense_strides(nc, pia)
    N = int(np.prod(na))
    if dist == "normal":
        a = rng.standard_normal(N)
        b = rng.standard_normal(m * nq)
    else:   # |x| log-uniform on [1e-4, 1e4], random sign
        a = np.exp(rng.uniform(np.log(1e-4), np.log(1e4), N)) * rng.choice([-1, 1], N)
        b = np.exp(rng.uniform(np.log(1e-4), np.log(1e4), m * nq)) * rng.choice([-1, 1], m * nq)
    a = a.astype(np.float32)
    b = b.astype(np.float32)
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    tbuf = torch.full((int(np.prod(nc)) + c_off,), float("nan"), device=dev)
    tc = tbuf[c_off:]
    pib = [1, 2] if b_cm else [2, 1]
    stream = torch.cuda.current_stream().cuda_stream
    if schedule is None:
        _lib.ttm_raw(_lib.F32, precision, q, len(na), ta.data_ptr(), na, wa, pia, tb.data_ptr(), [m, nq], pib,
                     tc.data_ptr(), nc, wc, stream)
    else:
        from ttm_b200.selector import lib as sched_lib
        _lib.check(sched_lib().tlibttm_ttm_sched(_lib.F32, schedule, q, len(na), C.c_void_p(ta.data_ptr()),
                                                 _lib.sz(na), _lib.sz(wa), _lib.sz(pia), C.c_void_p(tb.data_ptr()),
                                                 _lib.sz([m, nq]), _lib.sz(pib), C.c_void_p(tc.data_ptr()),
                                                 _lib.sz(nc), _lib.sz(wc), C.c_void_p(stream)))
    assert _lib.lib().tlibttm_synchronize(None) == 0, _lib.lib().tlibttm_last_error()
    kern = _lib.last_kernel()
    got = tc.cpu().numpy().astype(np.float64)
    # FP64 reference on the dense slice view
    qh = pia.index(q)
    inner = int(np.prod([na[pia[r] - 1] for r in range(qh)]))
    outer = N // (inner * nq)
    A3 = a.astype(np.float64).reshape(outer, nq, inner)
    Bm = b.astype(np.float64).reshape(nq, m).T if b_cm else b.astype(np.float64).reshape(m, nq)
    want = np.einsum("kli,jl->kji", A3, Bm).reshape(-1)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    return err, kern


CASES = [
    # (na, pia, q, m, b_cm)      geometry notes
    ([256, 64, 40], [1, 2, 3], 2, 256, True),     # i-contiguous, inner 256, full N tile
    ([256, 64, 40], [1, 2, 3], 2, 256, False),    # row-major B
    ([200, 50, 12], [1, 2, 3], 2, 100, True),     # partial M tile (inner 200), partial K chunk (nq 50), N 112
    ([36, 70, 9], [1, 2, 3], 2, 17, False),       # inner 36 < 128, m just above the bandwidth kernels
    ([64, 48, 33], [1, 2, 3], 3, 300, True),      # q = pi_p (outer 1), m > 256: two j blocks
    ([96, 33, 300], [1, 2, 3], 1, 64, True),      # q = pi_1: K-major tiles, partial K chunk (96 = 3 x 32)
    ([132, 20, 70], [1, 3, 2], 1, 48, False),     # q = pi_1, partial M tile (outer 1400), nq 132
    ([40, 30, 20, 12], [2, 4, 1, 3], 1, 32, True),  # inner 30*12=360 under a permuted layout
    # rows not 16-byte aligned for TMA: the converter warps load A themselves
    ([33, 40, 7], [1, 2, 3], 2, 64, True),        # inner 33 (odd), partial M tile
    ([135, 19, 11], [1, 2, 3], 2, 40, False),     # inner 135, nq 19, partial K chunk
    ([37, 20, 30], [1, 2, 3], 1, 48, True),       # q = pi_1 with nq 37 (K-major tiles)
    ([21, 17, 300], [1, 3, 2], 1, 20, False),     # q = pi_1, nq 21, outer 5100
    # inner <= 64: several slices share a 128-row tile (folded), last tile partly past the end
    ([32, 40, 7], [1, 2, 3], 2, 32, True),        # inner 32: 4 slices per tile, 7 slices
    ([64, 50, 9], [1, 2, 3], 2, 48, False),       # inner 64: 2 slices per tile
    ([20, 33, 5], [1, 2, 3], 2, 40, True),        # inner 20 (unaligned: converters load), 32-row slots
    ([48, 16, 11], [1, 2, 3], 2, 300, False),     # inner 48 in 64-row slots, two j blocks
]


@pytest.mark.parametrize("case", CASES)
def test_bf16x3_accuracy(cuda, case):
    na, pia, q, m, b_cm = case
    err, kern = run(cuda, na, pia, q, m, b_cm)
    assert kern.startswith("tc_bf16x3"), kern
    assert err <= 1e-5, (case, err)


def test_bf16x3_log_uniform(cuda):
    err, kern = run(cuda, [256, 64, 40], [1, 2, 3], 2, 256, True, dist="loguniform", seed=4)
    assert kern.startswith("tc_bf16x3")
    assert err <= 1e-5, err


# The pair kernel (two SMs per MMA, B resident in tensor memory): 128 < m <= 256, n_q <= 256,
# rows of 128 consecutive i (inner >= 128) or contiguous fibres (q = pi_1, n_q % 4 == 0).
PAIR_CASES = [
    # (na, pia, q, m, b_cm, c_off)   geometry notes
    ([256, 64, 40], [1, 2, 3], 2, 256, True, 0),      # two tiles per slice, full M
    ([256, 64, 40], [1, 2, 3], 2, 256, False, 0),     # row-major B
    ([200, 50, 12], [1, 2, 3], 2, 129, True, 0),      # partial tile (inner 200), l padding, one row in the odd CTA
    ([136, 17, 9], [1, 2, 3], 2, 200, False, 0),      # 8-row last tile, n_q 17: one stage, half padding
    ([128, 256, 6], [1, 2, 3], 2, 256, True, 0),      # n_q 256: eight stages, B fills 256 columns
    ([64, 48, 33], [1, 2, 3], 3, 192, True, 0),       # q = pi_p: one slice, inner 3072
    ([40, 30, 20, 12], [2, 4, 1, 3], 1, 144, True, 0),  # inner 30*12 = 360 under a permuted layout
    ([256, 64, 40], [1, 2, 3], 2, 160, True, 1),      # C off its 16-byte alignment: scalar stores
    ([96, 33, 300], [1, 2, 3], 1, 160, True, 0),      # contiguous fibres, partial last tile (outer 9900)
    ([132, 20, 70], [1, 3, 2], 1, 256, False, 0),     # contiguous fibres, n_q 132: nine sub-blocks
    ([256, 40, 30], [1, 2, 3], 1, 131, True, 0),      # contiguous fibres, n_q 256
    ([20, 64, 50], [1, 2, 3], 1, 250, False, 2),      # contiguous fibres, n_q 20, C unaligned
]


@pytest.mark.parametrize("case", PAIR_CASES)
def test_bf16x3_pair_kernel(cuda, case):
    na, pia, q, m, b_cm, c_off = case
    err, kern = run(cuda, na, pia, q, m, b_cm, c_off=c_off)
    assert kern == "tc_bf16x3_pair", kern
    assert err <= 1e-5, (case, err)


def test_bf16x3_pair_and_single_sm_kernels_agree(cuda):
    """The same problems through the pair kernel's schedule (7) and the single-SM kernel's (5)."""
    for na, pia, q, m in (([256, 64, 40], [1, 2, 3], 2, 256), ([96, 33, 300], [1, 2, 3], 1, 176)):
        e_pair, k_pair = run(cuda, na, pia, q, m, True, seed=5, schedule=7)
        e_one, k_one = run(cuda, na, pia, q, m, True, seed=5, schedule=5)
        assert (k_pair, k_one) == ("tc_bf16x3_pair", "tc_bf16x3")
        assert e_pair <= 1e-5 and e_one <= 1e-5, (e_pair, e_one)
        assert abs(e_pair - e_one) <= 2e-6


def test_bf16x3_pair_log_uniform(cuda):
    err, kern = run(cuda, [256, 64, 40], [1, 2, 3], 2, 256, True, dist="loguniform", seed=6)
    assert kern == "tc_bf16x3_pair"
    assert err <= 1e-5, err


def test_bf16x3_repeatable_and_device_status_clear(cuda):
    e1, _ = run(cuda, [256, 64, 40], [1, 2, 3], 2, 64, True, seed=3)
    e2, _ = run(cuda, [256, 64, 40], [1, 2, 3], 2, 64, True, seed=3)
    assert e1 == e2
    assert _lib.lib().tlibttm_synchronize(None) == 0
