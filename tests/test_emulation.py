"""The fp8 emulation used by the precision tests (CPU only)."""
import numpy as np

from emulation import e4m3_round, fibre_exponents, fp8_operand


def test_e4m3_values():
    x = np.array([1.0, 0.3, 448.0, 460.0, 1000.0, -17.0, 2.0 ** -9, 2.0 ** -10, 3 * 2.0 ** -11, 0.0, 15.5, 240.0])
    want = np.array([1.0, 0.3125, 448.0, 448.0, 448.0, -16.0, 2.0 ** -9, 0.0, 2.0 ** -9, 0.0, 16.0, 240.0])
    assert np.array_equal(e4m3_round(x), want)


def test_e4m3_grid_is_fixed():
    # every e4m3 value rounds to itself: 3 fraction bits per binade, subnormals step 2^-9
    vals = [0.0] + [m * 2.0 ** -9 for m in range(1, 8)]
    vals += [(1 + f / 8) * 2.0 ** e for e in range(-6, 9) for f in range(8) if (1 + f / 8) * 2.0 ** e <= 448]
    v = np.array(vals + [-x for x in vals])
    assert np.array_equal(e4m3_round(v), v)


def test_fibre_scaling():
    x = np.array([[3.0, -0.5, 0.0], [0.0, 0.0, 0.0], [1e-30, 2e-30, -4e-30]])
    assert list(fibre_exponents(x)) == [2, 0, int(np.frexp(4e-30)[1])]
    y = fp8_operand(x)
    assert y[0, 0] == 3.0 and y[0, 1] == -0.5 and np.all(y[1] == 0)
    assert np.allclose(y[2], x[2], rtol=2 ** -4)
