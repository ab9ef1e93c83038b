"""Learned schedule selector: the MLP's CUDA training kernels against an FP64 CPU restatement of
the same network (gradient check), schedule control through the C ABI, and a small end-to-end
tuning run."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np_forward(Ws, bs, X):
    acts = [X]
    for i, (W, b) in enumerate(zip(Ws, bs)):
        z = acts[-1] @ W.T + b
        acts.append(np.maximum(z, 0) if i < len(Ws) - 1 else z)
    return acts


def _np_grads(Ws, bs, X, T, M):
    acts = _np_forward(Ws, bs, X)
    cnt = max(M.sum(), 1.0)
    d = 2.0 * (acts[-1] - T) * M / cnt
    loss = float(((acts[-1] - T) ** 2 * M).sum() / cnt)
    gW, gb = [None] * len(Ws), [None] * len(Ws)
    for i in range(len(Ws) - 1, -1, -1):
        dz = d if i == len(Ws) - 1 else d * (acts[i + 1] > 0)
        gW[i] = dz.T @ acts[i]
        gb[i] = dz.sum(0)
        d = dz @ Ws[i]
    return loss, gW, gb


def test_mlp_gradients_match_fp64_oracle(cuda):
    import torch
    from ttm_b200.selector import MLP
    rng = np.random.default_rng(0)
    mlp = MLP(n_in=7, n_out=3, hidden=5, seed=3)
    X = rng.standard_normal((9, 7)).astype(np.float32)
    T = rng.standard_normal((9, 3)).astype(np.float32)
    M = (rng.random((9, 3)) > 0.3).astype(np.float32)
    loss, gW, gb = mlp.gradients(torch.tensor(X, device=cuda), torch.tensor(T, device=cuda),
                                 torch.tensor(M, device=cuda))
    Ws = [w.double().cpu().numpy() for w in mlp.W]
    bs = [b.double().cpu().numpy() for b in mlp.b]
    ref_loss, rW, rb = _np_grads(Ws, bs, X.astype(np.float64), T.astype(np.float64), M.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-5 * max(1.0, abs(ref_loss))
    for g, r in zip(gW + gb, rW + rb):
        g = g.double().cpu().numpy()
        assert np.allclose(g, r, rtol=1e-4, atol=1e-6), np.abs(g - r).max()


def test_mlp_gradients_against_finite_differences(cuda):
    """Directional derivative of the loss (FP64 oracle) equals <grad, direction> from the CUDA kernels."""
    import torch
    from ttm_b200.selector import MLP
    rng = np.random.default_rng(1)
    mlp = MLP(n_in=6, n_out=2, hidden=8, seed=1)
    X = rng.standard_normal((16, 6))
    T = rng.standard_normal((16, 2))
    M = np.ones((16, 2))
    _, gW, gb = mlp.gradients(torch.tensor(X, device=cuda, dtype=torch.float32),
                              torch.tensor(T, device=cuda, dtype=torch.float32),
                              torch.tensor(M, device=cuda, dtype=torch.float32))
    Ws = [w.double().cpu().numpy() for w in mlp.W]
    bs = [b.double().cpu().numpy() for b in mlp.b]
    dirs = [rng.standard_normal(w.shape) for w in Ws] + [rng.standard_normal(b.shape) for b in bs]
    eps = 1e-6
    lp = _np_grads([w + eps * d for w, d in zip(Ws, dirs[:4])], [b + eps * d for b, d in zip(bs, dirs[4:])], X, T, M)[0]
    lm = _np_grads([w - eps * d for w, d in zip(Ws, dirs[:4])], [b - eps * d for b, d in zip(bs, dirs[4:])], X, T, M)[0]
    fd = (lp - lm) / (2 * eps)
    an = sum(float((g.double().cpu().numpy() * d).sum()) for g, d in zip(gW + gb, dirs))
    assert abs(fd - an) <= 1e-3 * max(1.0, abs(fd)), (fd, an)


def test_schedules_through_the_c_abi_agree(cuda):
    import torch
    from ttm_b200 import _lib
    from ttm_b200.selector import Autotuner, valid_mask
    pr = dict(p=3, na=[64, 48, 40], q=2, pia=[1, 2, 3], m=8)
    ok = valid_mask(pr)
    # m = 8: neither tensor-core schedule; n_q = 48: no l split, no B streaming
    assert ok == [True, True, True, False, False, True, False, False, False]
    tuner = Autotuner(cap=1 << 20)
    t = tuner.times(pr)
    assert [x is not None for x in t] == ok and all(x > 0 for x in t if x is not None)
    # every valid schedule computes the same product (exact FMA, different orders): compare outputs
    na, pia, q, m = pr["na"], pr["pia"], pr["q"], pr["m"]
    A = torch.randn(math.prod(na), device=cuda)
    B = torch.randn(m * na[q - 1], device=cuda)
    outs = []
    for s in (1, 2, 3, 6):
        Cc = torch.full((math.prod(na) // na[q - 1] * m,), float("nan"), device=cuda)
        from ttm_b200.selector import lib, _dense
        nc = list(na)
        nc[q - 1] = m
        rc = lib().tlibttm_ttm_sched(_lib.F32, s, q, 3, A.data_ptr(), _lib.sz(na), _lib.sz(_dense(na, pia)),
                                     _lib.sz(pia), B.data_ptr(), _lib.sz([m, na[q - 1]]), _lib.sz([1, 2]),
                                     Cc.data_ptr(), _lib.sz(nc), _lib.sz(_dense(nc, pia)), None)
        assert rc == 0
        outs.append(Cc.double().cpu().numpy())
    for o in outs[1:]:
        assert np.allclose(o, outs[0], rtol=1e-5, atol=1e-5)
    # an invalid schedule is refused without running
    rc = lib().tlibttm_ttm_sched(_lib.F32, 4, q, 3, A.data_ptr(), _lib.sz(na), _lib.sz(_dense(na, pia)), _lib.sz(pia),
                                 B.data_ptr(), _lib.sz([m, na[q - 1]]), _lib.sz([1, 2]), Cc.data_ptr(), _lib.sz(nc),
                                 _lib.sz(_dense(nc, pia)), None)
    assert rc == _lib.ERR_UNSUPPORTED


def test_split_schedules_are_tunable(cuda, oracle_c):
    """c = B a with n = 2^16, m = 64 (order 1): the plain slice-GEMM, its l-split form (schedule 8),
    the B-streaming kernel (9) and bf16x3 (5) are all valid; the exact ones agree with the C oracle
    within the FP32 bound and the autotuner times each of them."""
    import torch
    from ttm_b200 import _lib
    from ttm_b200.selector import Autotuner, lib, valid_mask
    pr = dict(p=1, na=[1 << 16], q=1, pia=[1], m=64)
    ok = valid_mask(pr)
    assert [s for s in range(1, 10) if ok[s - 1]] == [1, 5, 8, 9]
    t = Autotuner(cap=1 << 16, b_cap=64 << 16).times(pr)
    assert all((t[s - 1] is not None) == ok[s - 1] for s in range(1, 10))
    n, m = pr["na"][0], pr["m"]
    rng = np.random.default_rng(4)
    a = rng.standard_normal(n).astype(np.float32)
    b = rng.standard_normal(m * n).astype(np.float32)
    want = np.zeros(m, dtype=np.float32)
    oracle_c.ttm(1, a, [n], [1], [1], b, [m, n], [1, 2], want, [m], [1])
    A, B = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    for s in (1, 8, 9):
        Cc = torch.full((m,), float("nan"), device=cuda)
        _lib.check(lib().tlibttm_ttm_sched(_lib.F32, s, 1, 1, A.data_ptr(), _lib.sz([n]), _lib.sz([1]), _lib.sz([1]),
                                           B.data_ptr(), _lib.sz([m, n]), _lib.sz([1, 2]), Cc.data_ptr(), _lib.sz([m]),
                                           _lib.sz([1]), None))
        torch.cuda.synchronize()
        got = Cc.double().cpu().numpy()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 2e-6, s
        assert _lib.last_kernel() == ("bvec" if s == 9 else "simt_gemm"), s


def test_small_tuning_run(cuda):
    """Time a few hundred small problems, train the network on its own kernels, and check that it
    learned (loss falls) and that selection with autotuner fallback is never worse than guessing."""
    from ttm_b200.selector import train_and_evaluate
    losses = []
    model, res = train_and_evaluate(240, 80, steps=800, cap=1 << 20, log=lambda s: losses.append(s))
    steps = [x for x in losses if x.startswith("step")]
    first = float(steps[0].split()[-1])
    last = float(steps[-1].split()[-1])
    assert last < 0.5 * first, (first, last)
    for k in ("exact", "fp32_accurate"):
        r = res[k]
        assert 0.0 <= r["regret_mlp_with_fallback"] <= r["regret_mlp_alone"] + 1e-9
        assert r["regret_mlp_with_fallback"] < 0.5


def test_shipped_selector_gains_over_the_heuristic_on_held_out_problems(cuda):
    """The network shipped in ttm_b200/schedule_model.json, on the 2,000 held-out problems (seed 2,
    float and double, drawn as in training), timed here by the exhaustive autotuner: its time
    regret is within 5 % of the autotuned time with and without the autotuner fallback, below the
    regret of the planner's fixed heuristic (the method without the network), and the fallback
    decides for fewer than a third of the problems."""
    import json
    from ttm_b200 import selector, workloads
    with open(selector.MODEL_PATH) as f:
        shipped = json.load(f)
    model = selector.MLP.from_json(shipped["model"])
    test = selector.with_dtypes(workloads.problems(2000, 2), 2)
    res = selector.evaluate(model, selector.DtypeTuner(), test, margin=shipped["evaluation"]["margin"])
    assert 0.3 < res["f64_share"] < 0.7
    for k in ("exact", "fp32_accurate"):
        r = res[k]
        assert r["regret_mlp_with_fallback"] <= 0.05, (k, r)
        assert r["regret_mlp_alone"] <= 0.05, (k, r)
        assert r["regret_mlp_with_fallback"] < r["regret_heuristic"], (k, r)
        assert r["regret_mlp_alone"] < r["regret_heuristic"], (k, r)
        assert r["fallback_rate"] < 1.0 / 3.0, (k, r)


def test_tuned_precision_uses_the_shipped_model(cuda):
    import torch
    from ttm_b200 import ttmpy as tp
    rng = np.random.default_rng(4)
    for shape, q, m in (((96, 80, 72), 2, 8), ((96, 80, 72), 1, 40), ((64, 48, 40, 20), 3, 3)):
        A = torch.tensor(rng.standard_normal(shape), device=cuda, dtype=torch.float32)
        B = torch.tensor(rng.standard_normal((m, shape[q - 1])), device=cuda, dtype=torch.float32)
        got = tp.ttm(q, A, B, precision="tuned").double().cpu().numpy()
        want = np.moveaxis(np.tensordot(A.double().cpu().numpy(), B.double().cpu().numpy(), axes=([q - 1], [1])), -1,
                           q - 1)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5
