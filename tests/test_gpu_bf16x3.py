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


def run(dev, na, pia, q, m, b_cm, dist="normal", seed=0, precision=_lib.PREC_BF16X3):
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
    tc = torch.full((int(np.prod(nc)),), float("nan"), device=dev)
    pib = [1, 2] if b_cm else [2, 1]
    _lib.ttm_raw(_lib.F32, precision, q, len(na), ta.data_ptr(), na, wa, pia, tb.data_ptr(), [m, nq], pib,
                 tc.data_ptr(), nc, wc, torch.cuda.current_stream().cuda_stream)
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
    assert kern == "tc_bf16x3", kern
    assert err <= 1e-5, (case, err)


def test_bf16x3_log_uniform(cuda):
    err, kern = run(cuda, [256, 64, 40], [1, 2, 3], 2, 256, True, dist="loguniform", seed=4)
    assert kern == "tc_bf16x3"
    assert err <= 1e-5, err


def test_bf16x3_repeatable_and_device_status_clear(cuda):
    e1, _ = run(cuda, [256, 64, 40], [1, 2, 3], 2, 64, True, seed=3)
    e2, _ = run(cuda, [256, 64, 40], [1, 2, 3], 2, 64, True, seed=3)
    assert e1 == e2
    assert _lib.lib().tlibttm_synchronize(None) == 0
