"""Host-side helpers of the measurement and tuning tools (no GPU): the layout/mode sweep's extent
sets and layouts, the seeded problem generator of the batched workload and the selector, and the
selector's input features."""
import math

import numpy as np

from ttm_b200 import selector, sweep, workloads


def test_sweep_extent_sets():
    sets = sweep.extent_sets(0)
    assert len(sets) == 6
    assert sets[:4] == [list(s) for s in sweep.FIXED]
    for na in sets:
        assert math.prod(na) == 1 << 26 and min(na) >= 2 and 3 <= len(na) <= 6
    assert sweep.extent_sets(0) == sets                     # seeded


def test_sweep_layouts():
    for p in range(2, 7):
        for count in (1, 2, 5, 10):
            ls = sweep.layouts(p, count, 7)
            assert len(ls) == min(count, math.factorial(p))
            assert ls[0] == list(range(1, p + 1))
            if len(ls) > 1:
                assert ls[1] == list(range(p, 0, -1))
            assert len({tuple(x) for x in ls}) == len(ls)
            assert all(sorted(x) == list(range(1, p + 1)) for x in ls)


def test_dense_strides_match_layout():
    # the sweep's dense strides: the first mode of the layout is contiguous, each next mode's
    # stride is the previous stride times its extent
    na, pi = [3, 5, 7, 2], [3, 1, 4, 2]
    w = sweep._dense(na, pi)
    assert w[pi[0] - 1] == 1
    for r in range(1, len(na)):
        assert w[pi[r] - 1] == w[pi[r - 1] - 1] * na[pi[r - 1] - 1]


def test_workload_problems():
    a = workloads.problems(300, seed=0)
    assert a == workloads.problems(300, seed=0)           # seeded
    assert a != workloads.problems(300, seed=1)
    for pr in a:
        p, na, q, pia, m = pr["p"], pr["na"], pr["q"], pr["pia"], pr["m"]
        assert 3 <= p <= 5 and len(na) == p and 1 <= q <= p
        assert sorted(pia) == list(range(1, p + 1))
        assert math.prod(na) <= workloads.CAP
        assert math.prod(na) // na[q - 1] * m <= workloads.CAP
        assert 1 <= m <= 256 and min(na) >= 1
        assert workloads.flops(pr) == 2.0 * m * math.prod(na)
        n_a = math.prod(na)
        assert workloads.io_bytes(pr) == 4 * (n_a + n_a // na[q - 1] * m + m * na[q - 1])


def test_selector_features():
    for pr in workloads.problems(200, seed=3):
        f = selector.features(pr)
        assert len(f) == selector.FEATURES
        assert all(np.isfinite(f))
        assert f == selector.features(pr)
        inner, nq, outer = selector.geometry(pr["na"], pr["pia"], pr["q"])
        assert inner * nq * outer == math.prod(pr["na"]) and nq == pr["na"][pr["q"] - 1]
        # the one-hot layout block holds exactly p ones
        assert sum(f[11:47]) == pr["p"]
    assert selector.features(workloads.problems(1, seed=3)[0], dtype_id=1)[48] == 1.0
