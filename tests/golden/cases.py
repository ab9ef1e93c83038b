"""Seeded parity cases shared by the golden-fixture generator and the tests.

Each case is a dict: id, dtype ("f32"/"f64"), q (one-based), na, pia
(one-based layout), m, pib ((1,2) column-major / (2,1) row-major B), seed.
Inputs are regenerated from the seed by `make_inputs`, so fixtures only store
outputs. Extents include 1s (the reference's vector/scalar stride special
case) and m spans both sides of the small-m bandwidth kernels.
"""
import itertools

import numpy as np


def _shapes(p, rng):
    fixed = {1: [(5,), (1,)], 2: [(3, 4), (1, 5)], 3: [(3, 4, 2), (2, 1, 3)], 4: [(2, 3, 2, 3), (3, 1, 2, 2)],
             5: [(2, 2, 3, 2, 2)]}
    return fixed[p]


def golden_cases():
    rng = np.random.default_rng(20240601)
    cases = []
    cid = 0
    for p in range(1, 6):
        perms = list(itertools.permutations(range(1, p + 1)))
        if len(perms) > 6:
            sel = rng.choice(len(perms), size=6, replace=False)
            perms = [perms[i] for i in sorted(sel)]
        for na in _shapes(p, rng):
            for pia in perms:
                for q in range(1, p + 1):
                    for m in (1, 3, 17):
                        for pib in ((1, 2), (2, 1)):
                            for dt in ("f32", "f64"):
                                # thin the sweep for p >= 4 to keep fixtures small
                                if p >= 4 and (cid % 3):
                                    cid += 1
                                    continue
                                cases.append(dict(id=cid, dtype=dt, q=q, na=list(na), pia=list(pia), m=m,
                                                  pib=list(pib), seed=1000 + cid))
                                cid += 1
    return cases


def dense_strides(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


def make_inputs(case):
    """Flat A (memory order) and flat B for a case, plus metadata."""
    rng = np.random.default_rng(case["seed"])
    dt = np.float32 if case["dtype"] == "f32" else np.float64
    na = case["na"]
    q = case["q"]
    nq = na[q - 1]
    m = case["m"]
    nc = list(na)
    nc[q - 1] = m
    a = rng.standard_normal(int(np.prod(na))).astype(dt)
    b = rng.standard_normal(m * nq).astype(dt)
    wa = dense_strides(na, case["pia"])
    wc = dense_strides(nc, case["pia"])
    return a, b, dict(na=na, wa=wa, pia=case["pia"], nb=[m, nq], pib=case["pib"], nc=nc, wc=wc)
