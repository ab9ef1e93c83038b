"""Batched plans (one persistent grouped launch over a device work queue), Tucker chain plans,
and their CUDA-graph replay, against per-problem FP64 references."""
import numpy as np
import pytest

import known_answer as ka
from ttm_b200 import _lib

pytestmark = pytest.mark.gpu


def _ref(A, na, pia, q, Bm):
    """FP64 reference on the dense slice view; Bm is (m, nq)."""
    qh = pia.index(q)
    inner = int(np.prod([na[pia[r] - 1] for r in range(qh)]))
    nq = na[q - 1]
    outer = int(np.prod(na)) // (inner * nq)
    A3 = A.reshape(outer, nq, inner)
    return np.matmul(Bm, A3).reshape(-1)


def _random_problems(dev, count, dtype, seed):
    import torch
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        p = int(rng.integers(3, 6))
        # extents log-uniform on [8, 512], capped so N_A <= 2^20 here (the plan logic is size independent)
        na = [int(round(np.exp(rng.uniform(np.log(8), np.log(64))))) for _ in range(p)]
        while np.prod(na) > (1 << 20):
            na[int(np.argmax(na))] //= 2
        q = int(rng.integers(1, p + 1))
        pia = [int(x) + 1 for x in rng.permutation(p)]
        m = int(round(np.exp(rng.uniform(0, np.log(256)))))
        nq = na[q - 1]
        A = torch.randn(int(np.prod(na)), device=dev, dtype=dtype)
        B = torch.randn(m, nq, device=dev, dtype=dtype)
        Cc = torch.full((int(np.prod(na)) // nq * m,), float("nan"), device=dev, dtype=dtype)
        out.append(dict(q=q, A=A, B=B, C=Cc, na=na, pia=pia, m=m))
    return out


@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("precision", ["plain", "auto"])
def test_batched_plan_matches_references(cuda, dt, precision):
    import torch
    from ttm_b200.plans import BatchPlan
    dtype = torch.float32 if dt == "f32" else torch.float64
    probs = _random_problems(cuda, 96, dtype, seed=11)
    plan = BatchPlan(probs, precision=precision)
    plan.run()
    torch.cuda.synchronize()
    tol = 2e-6 if dt == "f32" else 1e-13
    if precision == "auto" and dt == "f32":
        tol = 1e-5
    worst = 0.0
    for pr in probs:
        want = _ref(pr["A"].double().cpu().numpy(), pr["na"], pr["pia"], pr["q"], pr["B"].double().cpu().numpy())
        got = pr["C"].double().cpu().numpy()
        worst = max(worst, np.linalg.norm(got - want) / np.linalg.norm(want))
    assert worst <= tol, worst
    # grouped launches (tensor-core, TMA-fed small-m, SIMT) plus the few small-m problems the
    # TMA-fed kernel does not take (unaligned rows) above the single-launch size
    small_misaligned = sum(1 for pr in probs if pr["m"] <= 16 and int(np.prod(pr["na"])) >= 1 << 18)
    assert 1 <= plan.launches <= 16 + small_misaligned
    plan.close()


def test_batched_plan_graph_replay_reads_new_data(cuda):
    import torch
    from ttm_b200.plans import BatchPlan
    probs = _random_problems(cuda, 40, torch.float32, seed=5)
    plan = BatchPlan(probs, precision="plain")
    plan.run_graph()
    torch.cuda.synchronize()
    first = [pr["C"].clone() for pr in probs]
    for pr in probs:                      # new inputs in the same buffers
        pr["A"].mul_(-2.0)
    plan.run_graph()                      # replay of the captured graph
    torch.cuda.synchronize()
    for pr, c0 in zip(probs, first):
        assert torch.allclose(pr["C"], -2.0 * c0, rtol=1e-5, atol=1e-5)
    plan.close()


@pytest.mark.parametrize("precision", ["plain", "bf16x3"])
def test_tucker_chain_plan(cuda, precision):
    """A (40,36,32,28) x U_k^T (m_k = 12, 10, 8, 6) on all four modes, in sequence."""
    import torch
    from ttm_b200.plans import ChainPlan
    na, pia = [40, 36, 32, 28], [1, 2, 3, 4]
    ms = [24, 20, 18, 17]
    A = torch.randn(int(np.prod(na)), device=cuda)
    Us = [torch.randn(ms[k], na[k], device=cuda) for k in range(4)]
    C_out = torch.empty(int(np.prod(ms)), device=cuda)
    plan = ChainPlan(A, na, pia, [1, 2, 3, 4], Us, C_out, precision=precision)
    plan.run_graph()
    torch.cuda.synchronize()
    X = A.double().cpu().numpy().reshape(na[::-1])          # first-order memory: index [i4][i3][i2][i1]
    for k, spec in enumerate(["lkji,ai->lkja", "lkja,bj->lkba", "lkba,ck->lcba", "lcba,dl->dcba"]):
        X = np.einsum(spec, X, Us[k].double().cpu().numpy())
    got = C_out.double().cpu().numpy().reshape(ms[::-1])
    err = np.linalg.norm(got - X) / np.linalg.norm(X)
    assert err <= (2e-6 if precision == "plain" else 1e-5), err
    plan.close()


def test_plan_errors_name_the_problem(cuda):
    """A bad problem is rejected at plan creation (nothing is launched) and named in the message."""
    import torch
    from ttm_b200.plans import BatchPlan
    probs = _random_problems(cuda, 3, torch.float32, seed=2)
    probs[1] = dict(probs[1], m=0)        # C would have a zero extent
    with pytest.raises(_lib.TtmError, match="problem 1: Error in tlib::tensor_times_matrix: shape vector of C is not valid"):
        BatchPlan(probs, precision="plain")


# (na, pia, q, m): every geometry and mode of the bf16x3 kernel in one grouped launch
GROUPED_TC_CASES = [
    ([256, 40, 6], [1, 2, 3], 2, 64),      # rows of i, TMA tiles
    ([200, 33, 5], [1, 2, 3], 2, 130),     # rows of i, a partial last tile, N = 144
    ([20, 48, 30], [1, 2, 3], 2, 17),      # inner <= 32: four slices folded into a 128-row tile
    ([50, 20, 30], [1, 2, 3], 2, 256),     # inner <= 64: two slices per tile
    ([130, 24, 7], [1, 2, 3], 2, 40),      # inner % 4 != 0: the converters load A, C stored directly
    ([36, 300, 4], [2, 1, 3], 2, 300),     # contiguous fibres, two j blocks (m > 256)
    ([30, 64, 50], [2, 1, 3], 2, 96),      # contiguous fibres (q = pi_1)
    ([11, 37, 90], [2, 1, 3], 2, 18),      # fibres with n_q % 4 != 0 (converters load), m % 4 != 0
    ([64, 64, 64], [3, 1, 2], 1, 200),     # another layout
]


def test_grouped_bf16x3_launch_matches_single_launches(cuda):
    """Under auto every float problem with m > 16 that the tensor-core path takes joins one grouped
    bf16x3 launch: one operand split for all B plus one persistent launch per geometry (3 here).
    Each result equals the single-SM bf16x3 kernel's (schedule 5) bit for bit, run before and
    after new data are written into the same buffers (graph replay)."""
    import ctypes as C
    import torch
    from ttm_b200.plans import BatchPlan
    from ttm_b200.selector import lib as sched_lib
    g = torch.Generator(device=cuda).manual_seed(7)
    probs = []
    for na, pia, q, m in GROUPED_TC_CASES:
        n = int(np.prod(na))
        probs.append(dict(q=q, na=na, pia=pia, m=m, A=torch.randn(n, device=cuda, generator=g),
                          B=torch.randn(m, na[q - 1], device=cuda, generator=g),
                          C=torch.full((n // na[q - 1] * m,), float("nan"), device=cuda)))
    plan = BatchPlan(probs, precision="auto")
    assert plan.launches == 3

    def single(pr):
        na, pia, q, m = pr["na"], pr["pia"], pr["q"], pr["m"]
        nc = list(na)
        nc[q - 1] = m
        out = torch.full_like(pr["C"], float("nan"))
        _lib.check(sched_lib().tlibttm_ttm_sched(_lib.F32, 5, q, len(na), C.c_void_p(pr["A"].data_ptr()), _lib.sz(na),
                                                 _lib.sz(ka.dense_strides(na, pia)), _lib.sz(pia),
                                                 C.c_void_p(pr["B"].data_ptr()), _lib.sz([m, na[q - 1]]),
                                                 _lib.sz([2, 1]), C.c_void_p(out.data_ptr()), _lib.sz(nc),
                                                 _lib.sz(ka.dense_strides(nc, pia)),
                                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return out

    for rnd in range(2):
        plan.run_graph()
        torch.cuda.synchronize()
        assert _lib.lib().tlibttm_synchronize(None) == 0
        for i, pr in enumerate(probs):
            want = single(pr)
            torch.cuda.synchronize()
            assert torch.equal(pr["C"], want), (rnd, GROUPED_TC_CASES[i])
            ref = _ref(pr["A"].double().cpu().numpy(), pr["na"], pr["pia"], pr["q"], pr["B"].double().cpu().numpy())
            err = np.linalg.norm(pr["C"].double().cpu().numpy() - ref) / np.linalg.norm(ref)
            assert err <= 1e-5, (GROUPED_TC_CASES[i], err)
        for pr in probs:                   # new A and B in the same buffers
            pr["A"].mul_(-0.5)
            pr["B"].add_(1.0)
    plan.close()


# (na, pia, q, m): row mode (contiguous fibres) and column mode with each box shape, every MB build
GROUPED_STREAM_CASES = [
    ([64, 300, 50], [2, 1, 3], 2, 1),      # contiguous fibres (q = pi_1), n_q % 4 == 0
    ([40, 64, 90], [2, 1, 3], 2, 7),       # contiguous fibres, MB 8
    ([36, 128, 60], [2, 1, 3], 2, 16),     # contiguous fibres, MB 16
    ([1024, 30, 20], [1, 2, 3], 2, 2),     # strided fibres, wide rows of i
    ([12, 50, 500], [1, 2, 3], 2, 3),      # inner 12: many slices per box
    ([256, 8, 70], [1, 2, 3], 2, 5),       # short n_q
    ([384, 40, 33], [1, 2, 3], 2, 11),     # MB 16, one CTA per SM
    ([64, 64, 64], [3, 1, 2], 2, 4),       # another layout
    ([20, 90, 64], [1, 3, 2], 3, 9),
]


@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_grouped_small_m_launch(cuda, dt):
    """Every dense problem with m <= 16 that the TMA-fed kernel takes with B staged whole joins one
    grouped launch per (row/column mode, MB build, CTAs per SM) class: here 9 problems in at most 9
    launches, replayed as a graph with new data; exact FMA arithmetic, so each result is within the
    exact-path bound of the FP64 reference (2e-6 float, 1e-13 double)."""
    import torch
    from ttm_b200.plans import BatchPlan
    dtype = torch.float32 if dt == "f32" else torch.float64
    g = torch.Generator(device=cuda).manual_seed(9)
    probs = []
    for na, pia, q, m in GROUPED_STREAM_CASES:
        n = int(np.prod(na))
        probs.append(dict(q=q, na=na, pia=pia, m=m, A=torch.randn(n, device=cuda, dtype=dtype, generator=g),
                          B=torch.randn(m, na[q - 1], device=cuda, dtype=dtype, generator=g),
                          C=torch.full((n // na[q - 1] * m,), float("nan"), device=cuda, dtype=dtype)))
    plan = BatchPlan(probs, precision="plain")
    assert 1 <= plan.launches <= len(GROUPED_STREAM_CASES)
    tol = 2e-6 if dt == "f32" else 1e-13
    for rnd in range(2):
        plan.run_graph()
        torch.cuda.synchronize()
        for i, pr in enumerate(probs):
            ref = _ref(pr["A"].double().cpu().numpy(), pr["na"], pr["pia"], pr["q"], pr["B"].double().cpu().numpy())
            err = np.linalg.norm(pr["C"].double().cpu().numpy() - ref) / np.linalg.norm(ref)
            assert err <= tol, (rnd, GROUPED_STREAM_CASES[i], err)
        for pr in probs:
            pr["A"].mul_(1.5)
            pr["B"].sub_(0.25)
    plan.close()


def test_graph_replay_without_a_stream_waits_for_queued_work(cuda):
    """run_graph() on the default stream replays on a stream the plan owns; that stream must start
    after the work already queued on the default stream (here: the kernels writing new inputs),
    exactly as a launch on the default stream itself would."""
    import torch
    from ttm_b200.plans import BatchPlan
    probs = _random_problems(cuda, 12, torch.float32, seed=21)
    a0 = [pr["A"].clone() for pr in probs]
    plan = BatchPlan(probs, precision="plain")
    plan.run_graph()
    torch.cuda.synchronize()
    c0 = [pr["C"].clone() for pr in probs]
    for rnd in range(3):
        for pr, a in zip(probs, a0):
            pr["A"].zero_()
            for _ in range(16):           # many queued kernels before the replay
                pr["A"].add_(a, alpha=1.0 / 16)
        plan.run_graph()                  # no synchronisation in between
        torch.cuda.synchronize()
        for pr, c in zip(probs, c0):
            assert torch.allclose(pr["C"], c, rtol=1e-5, atol=1e-5), rnd
    plan.close()


FEW_LAUNCH_CASES = [
    # (na, pia, q, m): small-m problems of at least 2^22 elements, rows not 16-byte aligned (by
    # default each takes a launch of its own), and two slice-GEMM ones
    ([129, 130, 251], [1, 2, 3], 3, 5),
    ([129, 130, 251], [1, 2, 3], 2, 9),
    ([131, 257, 125], [1, 2, 3], 1, 7),
    ([125, 131, 257], [2, 1, 3], 3, 16),
    ([64, 48, 40], [1, 2, 3], 2, 40),
    ([48, 64, 40], [3, 1, 2], 1, 24),
]


@pytest.mark.parametrize("precision", ["plain", "auto"])
def test_batched_plan_few_launches(cuda, precision):
    """TLIBTTM_PLAN_FEW_LAUNCHES puts the large small-m problems into the grouped small-m launch:
    fewer launches, the same results within the exact paths' bound."""
    import torch
    from ttm_b200.plans import BatchPlan
    g = torch.Generator(device=cuda).manual_seed(5)
    runs = {}
    for few in (False, True):
        probs = []
        for na, pia, q, m in FEW_LAUNCH_CASES:
            nq = na[q - 1]
            A = torch.randn(int(np.prod(na)), device=cuda, generator=g)
            B = torch.randn(m, nq, device=cuda, generator=g)
            Cc = torch.full((int(np.prod(na)) // nq * m,), float("nan"), device=cuda)
            probs.append(dict(q=q, A=A, B=B, C=Cc, na=na, pia=pia, m=m))
        plan = BatchPlan(probs, precision=precision, few_launches=few)
        plan.run_graph()
        torch.cuda.synchronize()
        worst = 0.0
        for pr in probs:
            want = _ref(pr["A"].double().cpu().numpy(), pr["na"], pr["pia"], pr["q"], pr["B"].double().cpu().numpy())
            got = pr["C"].double().cpu().numpy()
            worst = max(worst, np.linalg.norm(got - want) / np.linalg.norm(want))
        assert worst <= (1e-5 if precision == "auto" else 2e-6), (few, worst)
        runs[few] = plan.launches
        plan.close()
    assert runs[True] < runs[False], runs
    assert runs[True] <= 8, runs
