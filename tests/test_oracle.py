"""Pins the CPU oracle (oracle/ttm_oracle.c) before it is trusted as the checker.

1. Known answers of the reference's own unit test (test/src/gtest_tlib_ttm.cpp:29-134).
2. Outputs of the reference itself (oracle/_ref), committed as tests/golden/ref_outputs.npz.
3. When the reference build is present, a live cross-check on fresh random cases.
"""
import os

import numpy as np
import pytest

from cases import golden_cases, make_inputs
import known_answer as ka

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_outputs.npz")


@pytest.mark.parametrize("rank", [2, 3, 4])
def test_oracle_known_answers(oracle_c, rank):
    shapes = ka.shapes(rank) if rank < 4 else ka.shapes(rank, steps=2)
    n = 0
    for na in shapes:
        for pia in ka.layouts(rank):
            for q in range(1, rank + 1):
                nq = na[q - 1]
                m = 2 * nq
                a = ka.init_a(na, pia, q)
                nc = list(na)
                nc[q - 1] = m
                wa = ka.dense_strides(na, pia)
                wc = ka.dense_strides(nc, pia)
                b = np.ones(m * nq)
                want = ka.expected_c(na, pia, q, m)
                for pib in ([2, 1], [1, 2]):
                    c = np.zeros(len(want))
                    oracle_c.ttm(q, a, na, wa, pia, b, [m, nq], pib, c, nc, wc)
                    assert ka.ulp_close(c, want), (na, pia, q, pib)
                    n += 1
    assert n > 0


def test_oracle_matches_reference_fixtures(oracle_c):
    gold = np.load(GOLDEN)
    worst = {"f32": 0.0, "f64": 0.0}
    for case in golden_cases():
        a, b, md = make_inputs(case)
        c = np.zeros(int(np.prod(md["nc"])), dtype=a.dtype)
        oracle_c.ttm(case["q"], a, md["na"], md["wa"], md["pia"], b, md["nb"], md["pib"], c, md["nc"], md["wc"])
        ref = gold[f"c{case['id']}"]
        err = np.linalg.norm(c.astype(np.float64) - ref) / max(np.linalg.norm(ref), 1e-300)
        worst[case["dtype"]] = max(worst[case["dtype"]], err)
    # The oracle rounds once from a wider accumulator; OpenBLAS rounds per FMA.
    assert worst["f64"] < 1e-14, worst
    assert worst["f32"] < 1e-6, worst


def test_oracle_case_classifier(oracle_c, reference):
    import itertools
    for p in range(1, 6):
        for pi in itertools.permutations(range(1, p + 1)):
            for q in range(1, p + 1):
                want = [c for c in range(1, 9) if reference.is_case(c, p, q, list(pi))]
                got = oracle_c.case(p, q, list(pi))
                assert want == [got] or (not want and got == 0), (p, pi, q, want, got)


def test_oracle_live_vs_reference(oracle_c, reference):
    rng = np.random.default_rng(7)
    for trial in range(60):
        p = int(rng.integers(1, 6))
        na = [int(x) for x in rng.integers(1, 6, size=p)]
        pia = [int(x) + 1 for x in rng.permutation(p)]
        q = int(rng.integers(1, p + 1))
        m = int(rng.integers(1, 20))
        nq = na[q - 1]
        nc = list(na)
        nc[q - 1] = m
        wa = reference.strides(na, pia)
        wc = reference.strides(nc, pia)
        pib = [1, 2] if trial % 2 else [2, 1]
        for dt in (np.float64, np.float32):
            a = rng.standard_normal(int(np.prod(na))).astype(dt)
            b = rng.standard_normal(m * nq).astype(dt)
            c1 = np.zeros(int(np.prod(nc)), dtype=dt)
            c2 = np.zeros_like(c1)
            oracle_c.ttm(q, a, na, wa, pia, b, [m, nq], pib, c1, nc, wc)
            reference.ttm(q, a, na, wa, pia, b, [m, nq], pib, c2, nc, wc)
            tol = 1e-13 if dt == np.float64 else 2e-6
            assert np.allclose(c1, c2, rtol=tol, atol=tol * 10), (p, na, pia, q, m)


def test_oracle_error_texts_match_reference(oracle_c, reference):
    """Every argument check raises the reference's exact text (include/tlib/ttm.h:65-90)."""
    for args in bad_argument_sets():
        q, p, a, na, wa, pia, b, nb, pib, c, nc, wc = args
        msgs = []
        for impl in (oracle_c, reference):
            with pytest.raises(RuntimeError) as ei:
                impl.ttm(q, a, na, wa, pia, b, nb, pib, c, nc, wc) if p else _call_p0(impl, args)
            msgs.append(str(ei.value))
        assert msgs[0] == msgs[1]


def _call_p0(impl, args):
    q, p, a, na, wa, pia, b, nb, pib, c, nc, wc = args
    impl.ttm(q, a, [], [], [], b, nb, pib, c, [], [])


def bad_argument_sets():
    """(q, p, a, na, wa, pia, b, nb, pib, c, nc, wc) tuples violating one check each, in check order."""
    a = np.zeros(24)
    b = np.zeros(8)
    c = np.zeros(48)
    na, wa, pia = [2, 3, 4], [1, 2, 6], [1, 2, 3]
    nb = [4, 2]
    nc, wc = [4, 3, 4], [1, 4, 12]
    good = [1, 3, a, na, wa, pia, b, nb, [1, 2], c, nc, wc]
    out = []

    def v(i, val):
        g = list(good)
        g[i] = val
        out.append(tuple(g))

    v(0, 0)                       # q == 0
    v(0, 4)                       # q > p
    v(3, [2, 0, 4])               # shape of A invalid (nb[1] still matches na[0])
    v(7, [4, 3])                  # contraction dims differ
    v(7, [5, 2])                  # free dims differ
    v(5, [1, 1, 3])               # layout invalid
    v(4, [6, 2, 1])               # strides of A invalid
    v(11, [12, 4, 1])             # strides of C invalid
    return out
