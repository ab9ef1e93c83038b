"""Seeded random TTM problems (shapes only), used by the batched benchmark and the schedule tuner.

`random_problem(rng)` draws one problem as in the batched workload: order p uniform on 3..5,
extents log-uniform on [8, 512], contraction mode q uniform, layout a random permutation, m
log-uniform on [1, 256]; A and C are capped at 2^24 elements (the largest extent is halved until
A fits, m is redrawn until C fits).
"""
from __future__ import annotations

import math

import numpy as np

CAP = 1 << 24


def random_problem(rng: np.random.Generator, cap: int = CAP):
    p = int(rng.integers(3, 6))
    na = [int(round(math.exp(rng.uniform(math.log(8), math.log(512))))) for _ in range(p)]
    while math.prod(na) > cap:
        i = int(np.argmax(na))
        na[i] = max(1, na[i] // 2)
    q = int(rng.integers(1, p + 1))
    pia = [int(x) + 1 for x in rng.permutation(p)]
    nq = na[q - 1]
    for _ in range(64):
        m = int(round(math.exp(rng.uniform(0.0, math.log(256)))))
        if math.prod(na) // nq * m <= cap:
            break
    else:
        m = 1
    return dict(p=p, na=na, q=q, pia=pia, m=m)


def problems(count: int, seed: int, cap: int = CAP):
    rng = np.random.default_rng(seed)
    return [random_problem(rng, cap) for _ in range(count)]


def flops(pr) -> float:
    return 2.0 * pr["m"] * math.prod(pr["na"])


def io_bytes(pr, es: int = 4) -> float:
    na = pr["na"]
    nq = na[pr["q"] - 1]
    n_a = math.prod(na)
    return es * (n_a + n_a // nq * pr["m"] + pr["m"] * nq)
