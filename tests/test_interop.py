"""Host-side logic of ttmpy's device-array interop (no GPU needed): reading the CUDA array
interface, and the checks on ``out`` that run before any library call."""
import numpy as np
import pytest

from ttm_b200 import ttmpy


def test_cuda_array_interface_c_order_and_byte_strides():
    ptr, shape, st, dt = ttmpy._cai_layout({"shape": (3, 4, 5), "typestr": "<f4", "data": (4096, False),
                                            "version": 2})
    assert (ptr, shape, st, dt) == (4096, (3, 4, 5), (20, 5, 1), np.dtype(np.float32))
    # Fortran order given as byte strides
    _, _, st, dt = ttmpy._cai_layout({"shape": (3, 4), "typestr": "<f8", "data": (8, False),
                                      "strides": (8, 24), "version": 3, "stream": 1})
    assert st == (1, 3) and dt == np.dtype(np.float64)
    # the layout read from those strides is the first-order one
    assert ttmpy._layout_from_strides([3, 4], [1, 3]) == [1, 2]


def test_cuda_array_interface_rejections():
    with pytest.raises(ValueError, match="masked"):
        ttmpy._cai_layout({"shape": (2,), "typestr": "<f4", "data": (0, False), "mask": object(), "version": 2})
    with pytest.raises(ValueError, match="whole elements"):
        ttmpy._cai_layout({"shape": (2, 2), "typestr": "<f4", "data": (0, False), "strides": (6, 4), "version": 2})


def test_host_objects_are_not_device_views():
    assert ttmpy._device_view(np.zeros((2, 2))) is None
    assert ttmpy._device_view([[1.0, 2.0]]) is None
    assert ttmpy._device_view(3.0) is None


@pytest.mark.parametrize("bad", [
    np.zeros((4, 5, 6)),                          # wrong shape (C is 4 x 7 x 6)
    np.zeros((4, 7, 6), dtype=np.float32),        # wrong dtype
    np.zeros((6, 7, 4)).transpose(2, 1, 0),       # right shape, other layout
    [[0.0]],                                      # not an array
])
def test_numpy_out_must_match_c(bad):
    A = np.ones((4, 5, 6))
    B = np.ones((7, 5))
    with pytest.raises(ValueError, match="out must be an array of shape"):
        ttmpy.ttm(2, A, B, out=bad)
