"""Known-answer construction of the reference's unit test, restated.

test/src/gtest_tlib_ttm.cpp:26-55 (ttm_init) fills A so that every mode-q
fibre holds consecutive integers, counting along mode q first and then along
the other modes in layout order; B is all ones of shape (2*n_q, n_q)
(:187-188). Every C element is then the closed-form sum of its fibre
(refc, :82-87), compared within 4 ULP (:92-134). Shapes: every extent in
{2,4,8} (generate_shapes(2,3), test/include/gtest_aux.h:248-283), all p!
layouts (generate_permutations, :285-299), all q, B row- and column-major.
"""
import itertools

import numpy as np


def shapes(rank, init=2, steps=3):
    ext = [init * (2 ** s) for s in range(steps)]
    return [list(t) for t in itertools.product(ext, repeat=rank)]


def layouts(rank):
    return [list(t) for t in itertools.permutations(range(1, rank + 1))]


def dense_strides(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


def geometry(na, pia, q):
    qh = pia.index(q)
    inner = int(np.prod([na[pia[r] - 1] for r in range(qh)])) if qh else 1
    outer = int(np.prod([na[pia[r] - 1] for r in range(qh + 1, len(na))])) if qh + 1 < len(na) else 1
    return inner, outer


def init_a(na, pia, q, dtype=np.float64):
    """Flat A (memory order): A[k][l][i] = 1 + l + nq*(i + inner*k)."""
    nq = na[q - 1]
    inner, outer = geometry(na, pia, q)
    k = np.arange(outer).reshape(outer, 1, 1)
    l = np.arange(nq).reshape(1, nq, 1)
    i = np.arange(inner).reshape(1, 1, inner)
    return (1 + l + nq * (i + inner * k)).astype(dtype).reshape(-1)


def expected_c(na, pia, q, m, dtype=np.float64):
    """Flat C (memory order) for B = ones(m, nq): every j equals the fibre sum."""
    nq = na[q - 1]
    inner, outer = geometry(na, pia, q)
    k = np.arange(outer).reshape(outer, 1, 1)
    i = np.arange(inner).reshape(1, 1, inner)
    first = 1 + nq * (i + inner * k)
    s = (2 * first + nq - 1) * nq // 2
    return np.broadcast_to(s, (outer, m, inner)).astype(dtype).reshape(-1)


def ulp_close(x, y, ulps=4):
    """gtest AlmostEquals analogue: |x - y| within `ulps` units in the last place of the larger magnitude."""
    x = np.asarray(x)
    y = np.asarray(y)
    tol = ulps * np.spacing(np.maximum(np.abs(x), np.abs(y)).astype(x.dtype))
    return bool(np.all(np.abs(x - y) <= tol))
