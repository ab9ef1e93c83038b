"""CPU emulation of the fp8 path's arithmetic (test infrastructure only).

The fp8 path scales every mode-q fibre of A and every row of B by a power of two 2^(8-e), where
max|x| = f 2^e with f in [0.5, 1), rounds the scaled values to e4m3 (round to nearest even,
saturating at +-448) and accumulates exact products in FP32. This module rebuilds those
rounded operands in float64 so that the GPU result can be compared with the same product
computed exactly: the only remaining difference is the FP32 accumulation.
"""
import numpy as np


def fibre_exponents(x):
    """e with max|x| = f 2^e, f in [0.5, 1), over the last axis (0 for all-zero fibres)."""
    mx = np.abs(x).max(axis=-1)
    _, e = np.frexp(mx)
    return np.where(mx > 0, e, 0)


def e4m3_round(x):
    """Round float64 values to the nearest e4m3 value (ties to even), saturating at +-448."""
    x = np.asarray(x, dtype=np.float64)
    ax = np.abs(x)
    _, E = np.frexp(np.where(ax > 0, ax, 1.0))
    e = np.maximum(E - 1, -6)                 # binade exponent; subnormals share the 2^-6 binade
    step = np.ldexp(1.0, e - 3)               # 3 fraction bits
    q = np.round(x / step) * step             # numpy rounds half to even
    return np.clip(q, -448.0, 448.0)


def fp8_operand(x):
    """The fp8 image of x, scaled back: per fibre (last axis) 2^(e-8) * e4m3(x * 2^(8-e))."""
    e = fibre_exponents(x)[..., None]
    return np.ldexp(e4m3_round(np.ldexp(x.astype(np.float64), 8 - e)), e - 8)


def fp8_ttm(q, A, B):
    """C = A x_q B with both operands rounded as the fp8 path rounds them (A: numpy array in its
    logical shape, B: (m, n_q)); exact float64 accumulation."""
    Aq = fp8_operand(np.moveaxis(A, q - 1, -1))
    Be = fp8_operand(B)
    return np.moveaxis(np.tensordot(Aq, Be, axes=([-1], [1])), -1, q - 1)
