"""Parity at the benchmark configurations' own sizes.

* Layout/mode sweep at 2^26 elements (p = 3..6, every q, first- and last-order layouts,
  m in {1, 8, 64, 512}, float and double; the library's default arithmetic, exact FMA in the I/O
  type), and the same float cases under precision auto (bf16x3 where m > 16). Each case is
  checked on sampled output fibres against the C oracle, run on exactly those fibres (A's fibres
  gathered into an (n_q, S) tensor, contracted on mode 1).
* The batched workload (512 problems drawn as the benchmark draws them, one batched plan,
  CUDA-graph replay), per problem on sampled fibres against the C oracle.
* The Tucker chain A (192,192,192,192) x_k U_k^T, U_k (32, 192), k = 1..4, through the
  multilinear identity sum_j C[j] x1[j1] x2[j2] x3[j3] x4[j4] = sum_i A[i] y1[i1] y2[i2] y3[i3]
  y4[i4] with y_k = U_k^T x_k, for random x_k, the right side in FP64 on the host.

Bounds (relative, over the sampled fibres): exact FP32 FMA 1e-5 root-mean-square (the FP32
target), FP64 1e-12, bf16x3 1e-5.
"""
import math

import numpy as np
import pytest

from ttm_b200 import _lib
from ttm_b200.sweep import extent_sets, layouts, sample_fibres

pytestmark = pytest.mark.gpu

# C larger than this many elements is skipped (float: 64 GB, double: 64 GB).
MAX_C = {"f32": 1 << 34, "f64": 1 << 33}
TOL = {"f32": 1e-5, "f64": 1e-12}


def _dense(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


def _oracle_on_fibres(oracle_c, a_s, b, dtype):
    """The C oracle on the gathered fibres: A' of extents (n_q, S), first-order, q = 1;
    B (m x n_q) column-major. Returns C' as (S, m)."""
    S, nq = a_s.shape
    m = b.shape[0]
    a1 = np.ascontiguousarray(a_s.astype(dtype))            # memory [s][l] = extents (n_q, S) first-order
    b1 = np.ascontiguousarray(b.T.astype(dtype)).reshape(-1)   # [l][j] = column-major (m, n_q)
    c1 = np.zeros(S * m, dtype=dtype)
    oracle_c.ttm(1, a1.reshape(-1), [nq, S], [1, nq], [1, 2], b1, [m, nq], [1, 2], c1, [m, S], [1, m])
    return c1.reshape(S, m)


def _rel(got, want):
    d = np.linalg.norm(got.astype(np.float64) - want.astype(np.float64))
    return d / max(np.linalg.norm(want.astype(np.float64)), 1e-300)


@pytest.mark.parametrize("dname,precision", [("f32", "default"), ("f64", "default"), ("f32", "auto")])
def test_layout_mode_sweep_full_size_vs_oracle(cuda, oracle_c, dname, precision):
    import torch
    dt = _lib.F32 if dname == "f32" else _lib.F64
    tdt = torch.float32 if dname == "f32" else torch.float64
    npdt = np.float32 if dname == "f32" else np.float64
    n = 1 << 26
    gen = torch.Generator(device=cuda).manual_seed(7)
    A = torch.randn(n, device=cuda, dtype=tdt, generator=gen)
    stream = torch.cuda.current_stream().cuda_stream
    worst, cases, kernels = 0.0, 0, set()
    for si, na in enumerate(extent_sets(0)):
        p = len(na)
        for pia in layouts(p, 2, si):                       # first- and last-order
            for q in range(1, p + 1):
                nq = na[q - 1]
                for m in (1, 8, 64, 512):
                    nout = n // nq * m
                    if nout > MAX_C[dname]:
                        continue
                    nc = list(na)
                    nc[q - 1] = m
                    B = torch.randn(m * nq, device=cuda, dtype=tdt, generator=gen)
                    C = torch.full((nout,), float("nan"), device=cuda, dtype=tdt)
                    _lib.ttm_raw(dt, _lib.PRECISIONS[precision], q, p, A.data_ptr(), na, _dense(na, pia), pia,
                                 B.data_ptr(), [m, nq], [1, 2], C.data_ptr(), nc, _dense(nc, pia), stream)
                    kernels.add(_lib.last_kernel())
                    a_s, b, c_s = sample_fibres(A, B, C, na, pia, q, m, 512 if m >= 64 else 2048, gen)
                    want = _oracle_on_fibres(oracle_c, a_s, b, npdt)
                    err = _rel(c_s, want)
                    assert np.all(np.isfinite(c_s)), (na, pia, q, m)
                    assert err <= TOL[dname], (na, pia, q, m, _lib.last_kernel(), err)
                    worst = max(worst, err)
                    cases += 1
                    del B, C
    del A
    torch.cuda.empty_cache()
    assert cases >= 200
    if precision == "auto":
        assert "tc_bf16x3" in kernels
    print(f"{dname} {precision}: {cases} cases, worst rms {worst:.2e}, kernels {sorted(kernels)}")


def test_batched_workload_512_per_problem_vs_oracle(cuda, oracle_c):
    import torch
    from ttm_b200 import workloads
    from ttm_b200.plans import BatchPlan
    probs = workloads.problems(512, seed=0)
    gen = torch.Generator(device=cuda).manual_seed(1)
    entries = []
    for pr in probs:
        na, q, m = pr["na"], pr["q"], pr["m"]
        n_a = math.prod(na)
        A = torch.randn(n_a, device=cuda, generator=gen)
        B = torch.randn(m, na[q - 1], device=cuda, generator=gen)
        Cc = torch.full((n_a // na[q - 1] * m,), float("nan"), device=cuda)
        entries.append(dict(q=q, A=A, B=B, C=Cc, na=na, pia=pr["pia"], m=m))
    plan = BatchPlan(entries, precision="auto")
    plan.run_graph()
    plan.run_graph()       # a replay reads the same buffers again
    torch.cuda.synchronize()
    worst = 0.0
    for e in entries:
        a_s, b, c_s = sample_fibres(e["A"], e["B"].reshape(-1), e["C"], e["na"], e["pia"], e["q"], e["m"], 256, gen,
                                    b_cm=False)
        want = _oracle_on_fibres(oracle_c, a_s, b, np.float32)
        err = _rel(c_s, want)
        assert err <= 1e-5, (e["na"], e["pia"], e["q"], e["m"], err)
        worst = max(worst, err)
    plan.close()
    print(f"batched 512: worst rms {worst:.2e}")


def test_tucker_192_chain_multilinear_identity(cuda):
    import torch
    from ttm_b200.plans import ChainPlan
    S, r = 192, 32
    gen = torch.Generator(device=cuda).manual_seed(3)
    A = torch.randn(S ** 4, device=cuda, generator=gen)
    Us = [torch.randn(r, S, device=cuda, generator=gen) for _ in range(4)]
    Cc = torch.full((r ** 4,), float("nan"), device=cuda)
    chain = ChainPlan(A, [S] * 4, [1, 2, 3, 4], [1, 2, 3, 4], Us, Cc, precision="auto")
    chain.run_graph()
    torch.cuda.synchronize()
    chain.close()
    # the whole chain in FP64 on the device (first-order memory: index [i4][i3][i2][i1])
    X = A.view(S, S, S, S).double()
    for spec, u in zip(["dcba,ja->dcbj", "dcbj,kb->dckj", "dckj,lc->dlkj", "dlkj,md->mlkj"], Us):
        X = torch.einsum(spec, X, u.double())
    err = ((Cc.view(r, r, r, r).double() - X).norm() / X.norm()).item()
    del X
    assert err <= 2e-5, err                                    # four bf16x3 steps of ~4.5e-6 each
    C4 = Cc.double().cpu().numpy().reshape(r, r, r, r)         # first-order: [j4][j3][j2][j1]
    U = [u.double().cpu().numpy() for u in Us]
    rng = np.random.default_rng(5)
    A4 = A.view(S, S, S, S)                                    # [i4][i3][i2][i1]
    sets = [[rng.standard_normal(r) for _ in range(4)] for _ in range(2)]
    lhs = [float(((C4 @ x[0]) @ x[1]) @ x[2] @ x[3]) for x in sets]
    ys = [[U[k].T @ x[k] for k in range(4)] for x in sets]     # y_k = U_k^T x_k (length S)
    rhs = [0.0] * len(sets)
    rhs_abs = [0.0] * len(sets)
    for i4 in range(S):                                        # FP64 on the host, one slice at a time
        sl = A4[i4].double().cpu().numpy()                     # [i3][i2][i1]
        sa = np.abs(sl)
        for t, y in enumerate(ys):
            rhs[t] += y[3][i4] * float(((sl @ y[0]) @ y[1]) @ y[2])
            rhs_abs[t] += abs(y[3][i4]) * float(((sa @ np.abs(y[0])) @ np.abs(y[1])) @ np.abs(y[2]))
    for t in range(len(sets)):
        assert abs(lhs[t] - rhs[t]) <= 1e-5 * rhs_abs[t], (lhs[t], rhs[t], rhs_abs[t])
