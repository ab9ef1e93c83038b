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
    assert plan.launches >= 1
    if precision == "plain":
        # small-m problems of at least 2^18 elements run on their own (forked over the plan's
        # worker streams); every other problem shares the one grouped launch
        singles = sum(1 for pr in probs if pr["m"] <= 16 and int(np.prod(pr["na"])) >= 1 << 18)
        grouped = len(probs) - singles
        assert singles > 1 and plan.launches == (1 if grouped else 0) + singles
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
