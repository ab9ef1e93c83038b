"""ttmpy argument errors (reference ttmpy/src/wrapped_ttm.cpp:37-127): ValueError with the same texts."""
import numpy as np
import pytest

from ttm_b200 import ttmpy as tp


def test_ttm_errors():
    A = np.zeros((3, 2, 4))
    with pytest.raises(ValueError, match="first input should be a tensor with order greater than zero"):
        tp.ttm(1, np.float64(1.0), np.zeros((2, 2)))
    with pytest.raises(ValueError, match="contraction mode should be greater than zero and at most equal to p"):
        tp.ttm(0, A, np.zeros((5, 3)))
    with pytest.raises(ValueError, match="contraction mode should be greater than zero and at most equal to p"):
        tp.ttm(4, A, np.zeros((5, 3)))
    with pytest.raises(ValueError, match="second input should be a mtrix with order equal to 2"):
        tp.ttm(1, A, np.zeros(3))
    with pytest.raises(RuntimeError, match="contraction dimension of A and B are not equal"):
        tp.ttm(1, A, np.zeros((5, 4)))


def test_ttms_errors():
    A = np.zeros((3, 2, 4, 5))
    Bs = [np.zeros((6, 2)), np.zeros((7, 4)), np.zeros((9, 5))]
    with pytest.raises(ValueError, match="multiplication order should be either"):
        tp.ttms(1, A, Bs, "sideways")
    with pytest.raises(ValueError, match="number of input matrices is not equal to the tensor order - 1"):
        tp.ttms(1, A, Bs[:2])
    with pytest.raises(ValueError, match="non-contraction mode should be greater than zero"):
        tp.ttms(5, A, Bs)
    with pytest.raises(ValueError, match="some of the input matrices are not matrices"):
        tp.ttms(1, A, [np.zeros(2), Bs[1], Bs[2]])
    with pytest.raises(ValueError, match="vector dimension is not compatible"):
        tp.ttms(1, A, [Bs[0], Bs[1], np.zeros((9, 4))])


def test_ttms_sequences():
    from ttm_b200.ttmpy import _ttms_sequence
    Bs = [np.zeros((6, 3)), np.zeros((7, 2)), np.zeros((9, 4))]
    assert [r for r, _ in _ttms_sequence(2, 4, Bs, "forward")] == [1, 3, 4]
    assert [r for r, _ in _ttms_sequence(2, 4, Bs, "backward")] == [4, 3, 1]
    # 1/n - 1/m: mode1 1/3-1/6=.167, mode3 1/2-1/7=.357, mode4 1/4-1/9=.139
    assert [r for r, _ in _ttms_sequence(2, 4, Bs, "optimal")] == [4, 1, 3]


def test_ttms_mode_q_plus_1_mismatch_is_runtime_error():
    """The reference does not compare the matrix of mode q+1 in its own checks; the mismatch
    surfaces from tlib::ttm as RuntimeError (needs no GPU: rejected before any launch)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("the chain runs on the GPU")
    A = np.zeros((3, 2, 4, 5))
    with pytest.raises(RuntimeError, match="contraction dimension of A and B are not equal"):
        tp.ttms(1, A, [np.zeros((6, 3)), np.zeros((7, 4)), np.zeros((9, 5))])
