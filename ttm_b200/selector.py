"""Schedule autotuner and learned schedule selector.

A *schedule* is one of the planner's kernel choices (include/tlibttm.h, tlibttm_schedule):
SIMT slice-GEMM, the two small-m kernels for strided fibres, the small-m kernel for contiguous
fibres, the TMA-fed small-m kernel, and the two bf16x3 tensor-core kernels (single SMs, and
pairs of SMs with B in tensor memory). The autotuner times every schedule valid for a
problem (CUDA events, median of a few runs) and keeps the results in a timing database. The
selector is a small multilayer perceptron (3 hidden layers of 64, ReLU) that predicts each
schedule's log2 run time from the problem's shape (p, q, log2 extents, layout, m, dtype); it is
trained on the GPU by the library's own CUDA kernels (tlibttm_mlp_*), picks the schedule with
the lowest prediction, and falls back to the autotuner when its top two predictions are closer
than a margin.

    python -m ttm_b200.selector --train 20000 --test 2000 --out ttm_b200/schedule_model.json

Regret on a set of problems = sum of run times of the chosen schedules / sum of the best
measured times - 1.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import _lib, workloads

try:
    import torch
except Exception:  # noqa: BLE001
    torch = None

# ids 1..9 (include/tlibttm.h tlibttm_schedule): kernels, and for the tensor cores two tile shapes
# (128 rows on one SM, 256 on a pair of SMs), and for the SIMT GEMM the split of the l loop
SCHEDULES = ["simt_gemm", "cols", "cols_split", "rows", "tc_bf16x3", "cols_tma", "tc_bf16x3_pair", "simt_split",
             "bvec"]
EXACT = [1, 2, 3, 4, 6, 8, 9]         # schedules that compute with exact FMA in the I/O type
NS = len(SCHEDULES)
FEATURES = 53
HIDDEN = 64
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "schedule_model.json")


def _declare(L):
    if getattr(L, "_sel_declared", False):
        return
    sig = [C.c_uint, C.c_uint, C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
           C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.c_void_p, C.POINTER(C.c_size_t),
           C.POINTER(C.c_size_t), C.c_void_p]
    L.tlibttm_ttm_sched.restype = C.c_int
    L.tlibttm_ttm_sched.argtypes = [C.c_int, C.c_int] + sig
    L.tlibttm_schedule_valid.restype = C.c_int
    L.tlibttm_schedule_valid.argtypes = [C.c_int, C.c_int, C.c_uint, C.c_uint, C.POINTER(C.c_size_t),
                                         C.POINTER(C.c_size_t), C.c_size_t]
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    L.tlibttm_mlp_forward.restype = i
    L.tlibttm_mlp_forward.argtypes = [vp, vp, vp, vp, i, i, i, i, vp]
    L.tlibttm_mlp_backward.restype = i
    L.tlibttm_mlp_backward.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, i, i, i, vp]
    L.tlibttm_mlp_mse_grad.restype = i
    L.tlibttm_mlp_mse_grad.argtypes = [vp, vp, vp, vp, vp, i, f, vp]
    L.tlibttm_mlp_adam.restype = i
    L.tlibttm_mlp_adam.argtypes = [vp, vp, vp, vp, i, f, f, f, f, i, vp]
    L._sel_declared = True


def lib():
    L = _lib.lib()
    _declare(L)
    return L


# ------------------------------------------------------------------------------ features
def geometry(na, pia, q):
    qh = pia.index(q)
    inner = math.prod(na[pia[r] - 1] for r in range(qh))
    outer = math.prod(na[pia[r] - 1] for r in range(qh + 1, len(na)))
    return inner, na[q - 1], outer


def features(pr, dtype_id=_lib.F32):
    """53 numbers: p, q, log2 extents (padded to 6), q-hat, first/last-order flags, one-hot layout
    (6 x 6), log2 m, dtype, and log2 of inner, outer, n_q and N_A (functions of the former)."""
    p, q, na, pia, m = pr["p"], pr["q"], pr["na"], pr["pia"], pr["m"]
    f = [p / 6.0, q / 6.0]
    f += [math.log2(n) / 9.0 for n in na] + [0.0] * (6 - p)
    qh = pia.index(q) + 1
    f += [qh / 6.0, float(pia == list(range(1, p + 1))), float(pia == list(range(p, 0, -1)))]
    onehot = [0.0] * 36
    for r, mode in enumerate(pia):
        onehot[r * 6 + mode - 1] = 1.0
    f += onehot
    f += [math.log2(m) / 8.0, float(dtype_id)]
    inner, nq, outer = geometry(na, pia, q)
    f += [math.log2(inner) / 24.0, math.log2(outer) / 24.0, math.log2(nq) / 9.0, math.log2(math.prod(na)) / 24.0]
    return f


def dtype_of(pr) -> int:
    """The I/O type of a problem (float unless the problem says otherwise)."""
    return int(pr.get("dtype", _lib.F32))


def with_dtypes(probs, seed, f64_share=0.5):
    """Marks about `f64_share` of the problems double (seeded, independent of the shapes)."""
    rng = np.random.default_rng(10_000 + seed)
    return [dict(pr, dtype=_lib.F64 if rng.random() < f64_share else _lib.F32) for pr in probs]


def valid_mask(pr, dtype_id=None):
    dtype_id = dtype_of(pr) if dtype_id is None else dtype_id
    L = lib()
    na, pia = _lib.sz(pr["na"]), _lib.sz(pr["pia"])
    return [bool(L.tlibttm_schedule_valid(dtype_id, s, pr["q"], pr["p"], na, pia, pr["m"])) for s in range(1, NS + 1)]


# ------------------------------------------------------------------------------ autotuner
class Autotuner:
    """Times every valid schedule of a problem on scratch device buffers (inputs are random; run
    time does not depend on values). Results are cached by problem signature. `cap` bounds the
    elements of A and of C, `b_cap` those of B; a larger problem is refused (ValueError) before
    anything runs."""

    def __init__(self, reps=3, cap=workloads.CAP, dtype_id=_lib.F32, b_cap=256 * 512):
        self.reps = reps
        self.dtype_id = dtype_id
        dt = torch.float32 if dtype_id == _lib.F32 else torch.float64
        dev = torch.device("cuda", torch.cuda.current_device())
        self.A = torch.randn(cap, device=dev, dtype=dt)
        self.C = torch.empty(cap, device=dev, dtype=dt)
        self.B = torch.randn(b_cap, device=dev, dtype=dt)
        self.stream = torch.cuda.current_stream(dev)
        self.db = {}

    @staticmethod
    def key(pr):
        return f"{pr['na']}|{pr['pia']}|{pr['q']}|{pr['m']}"

    def _run(self, pr, s, md):
        rc = lib().tlibttm_ttm_sched(self.dtype_id, s, pr["q"], pr["p"], C.c_void_p(self.A.data_ptr()), *md[:3],
                                     C.c_void_p(self.B.data_ptr()), md[3], md[4], C.c_void_p(self.C.data_ptr()),
                                     md[5], md[6], C.c_void_p(self.stream.cuda_stream))
        _lib.check(rc)

    def times(self, pr):
        """Median run time in microseconds per schedule 1..NS (None where invalid)."""
        k = self.key(pr)
        if k in self.db:
            return self.db[k]
        na, pia, q, m = pr["na"], pr["pia"], pr["q"], pr["m"]
        nc = list(na)
        nc[q - 1] = m
        if math.prod(na) > self.A.numel() or math.prod(nc) > self.C.numel() or m * na[q - 1] > self.B.numel():
            raise ValueError(f"problem {na} q={q} m={m} exceeds the tuner's scratch buffers")
        wa = _dense(na, pia)
        wc = _dense(nc, pia)
        md = [_lib.sz(na), _lib.sz(wa), _lib.sz(pia), _lib.sz([m, na[q - 1]]), _lib.sz([1, 2]), _lib.sz(nc),
              _lib.sz(wc)]
        out = []
        for s, ok in zip(range(1, NS + 1), valid_mask(pr, self.dtype_id)):
            if not ok:
                out.append(None)
                continue
            self._run(pr, s, md)
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(self.reps)]
            for e0, e1 in evs:
                e0.record(self.stream)
                self._run(pr, s, md)
                e1.record(self.stream)
            e1.synchronize()
            out.append(float(np.median([e0.elapsed_time(e1) * 1e3 for e0, e1 in evs])))
        self.db[k] = out
        return out


class DtypeTuner:
    """One Autotuner per I/O type; each problem is timed in its own type (`dtype` key)."""

    def __init__(self, reps=3, cap=workloads.CAP):
        self.tuners = {_lib.F32: Autotuner(reps=reps, cap=cap, dtype_id=_lib.F32),
                       _lib.F64: Autotuner(reps=reps, cap=cap, dtype_id=_lib.F64)}

    def times(self, pr):
        return self.tuners[dtype_of(pr)].times(pr)

    def best(self, pr, allowed=None):
        t = self.times(pr)
        cands = [(t[s - 1], s) for s in range(1, NS + 1) if t[s - 1] is not None and (allowed is None or s in allowed)]
        return min(cands)[1]


def _dense(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


# ------------------------------------------------------------------------------ MLP on the library's kernels
class MLP:
    """in -> 64 -> 64 -> 64 -> out, ReLU on the hidden layers; parameters in float32 on the GPU."""

    def __init__(self, n_in=FEATURES, n_out=len(SCHEDULES), hidden=HIDDEN, seed=0, device=None):
        g = torch.Generator().manual_seed(seed)
        dims = [n_in, hidden, hidden, hidden, n_out]
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.W, self.b = [], []
        for i in range(4):
            bound = math.sqrt(6.0 / (dims[i] + dims[i + 1]))
            self.W.append(((torch.rand(dims[i + 1], dims[i], generator=g) * 2 - 1) * bound).to(self.device))
            self.b.append(torch.zeros(dims[i + 1], device=self.device))
        self.dims = dims
        self.mean = torch.zeros(n_out, device=self.device)   # output offset (mean log time)

    def params(self):
        return self.W + self.b

    def forward(self, X, keep=False):
        L = lib()
        s = torch.cuda.current_stream().cuda_stream
        acts = [X.contiguous()]
        for i in range(4):
            y = torch.empty(X.shape[0], self.dims[i + 1], device=self.device)
            _lib.check(L.tlibttm_mlp_forward(acts[-1].data_ptr(), self.W[i].data_ptr(), self.b[i].data_ptr(),
                                             y.data_ptr(), X.shape[0], self.dims[i], self.dims[i + 1],
                                             1 if i < 3 else 0, s))
            acts.append(y)
        return acts if keep else acts[-1] + self.mean

    def gradients(self, X, T, M):
        """Masked-MSE loss and parameter gradients (all from the library's kernels)."""
        L = lib()
        s = torch.cuda.current_stream().cuda_stream
        acts = self.forward(X, keep=True)
        n = X.shape[0]
        y = acts[-1]
        dy = torch.empty_like(y)
        loss = torch.zeros(1, device=self.device)
        cnt = float(max(M.sum().item(), 1.0))
        _lib.check(L.tlibttm_mlp_mse_grad(y.data_ptr(), (T - self.mean).contiguous().data_ptr(), M.data_ptr(),
                                          dy.data_ptr(), loss.data_ptr(), y.numel(), 1.0 / cnt, s))
        gW, gb = [None] * 4, [None] * 4
        d = dy
        for i in range(3, -1, -1):
            dz = torch.empty_like(acts[i + 1])
            dx = torch.empty_like(acts[i]) if i > 0 else None
            gW[i] = torch.empty_like(self.W[i])
            gb[i] = torch.empty_like(self.b[i])
            _lib.check(L.tlibttm_mlp_backward(acts[i].data_ptr(), self.W[i].data_ptr(), acts[i + 1].data_ptr(),
                                              d.data_ptr(), dz.data_ptr(), dx.data_ptr() if dx is not None else None,
                                              gW[i].data_ptr(), gb[i].data_ptr(), n, self.dims[i], self.dims[i + 1],
                                              1 if i < 3 else 0, s))
            d = dx
        return float(loss.item()), gW, gb

    def fit(self, X, T, M, steps=3000, batch=256, lr=2e-3, seed=0, log=None):
        L = lib()
        s = torch.cuda.current_stream().cuda_stream
        # output offset: per-schedule mean of the valid targets
        self.mean = ((T * M).sum(0) / M.sum(0).clamp(min=1)).to(self.device)
        ps = self.params()
        mom = [torch.zeros_like(p) for p in ps]
        vel = [torch.zeros_like(p) for p in ps]
        g = torch.Generator(device=self.device).manual_seed(seed)
        for step in range(1, steps + 1):
            idx = torch.randint(0, X.shape[0], (batch,), device=self.device, generator=g)
            loss, gW, gb = self.gradients(X[idx], T[idx], M[idx])
            for p, gr, m_, v_ in zip(ps, gW + gb, mom, vel):
                _lib.check(L.tlibttm_mlp_adam(p.data_ptr(), gr.data_ptr(), m_.data_ptr(), v_.data_ptr(), p.numel(),
                                              lr, 0.9, 0.999, 1e-8, step, s))
            if log and (step % 500 == 0 or step == 1):
                log(f"step {step} loss {loss:.4f}")
        return self

    def to_json(self):
        return {"dims": self.dims, "W": [w.cpu().tolist() for w in self.W], "b": [b.cpu().tolist() for b in self.b],
                "mean": self.mean.cpu().tolist()}

    @classmethod
    def from_json(cls, d, device=None):
        m = cls(n_in=d["dims"][0], n_out=d["dims"][-1], hidden=d["dims"][1], device=device)
        m.W = [torch.tensor(w, device=m.device) for w in d["W"]]
        m.b = [torch.tensor(b, device=m.device) for b in d["b"]]
        m.mean = torch.tensor(d["mean"], device=m.device)
        return m


# ------------------------------------------------------------------------------ selection
class Selector:
    """Picks a schedule from the MLP's predictions; falls back to the autotuner when the best two
    predictions are within `margin` (log2 units) of each other."""

    def __init__(self, model: MLP, tuner: Autotuner = None, margin=0.15):
        self.model = model
        self.tuner = tuner
        self.margin = margin

    def choose(self, pr, allowed, dtype_id=None):
        dtype_id = dtype_of(pr) if dtype_id is None else dtype_id
        ok = valid_mask(pr, dtype_id)
        valid = [s for s in range(1, NS + 1) if ok[s - 1] and s in allowed]
        # a model trained before a schedule existed never proposes it; the autotuner times them all
        cands = [s for s in valid if s <= self.model.dims[-1]]
        if not valid:
            raise ValueError("no allowed schedule can run this problem")
        if len(valid) == 1:
            return valid[0], False
        if len(cands) < len(valid) and self.tuner is not None and len(cands) <= 1:
            return self.tuner.best(pr, allowed=set(valid)), True
        if len(cands) == 1:
            return cands[0], False
        X = torch.tensor([features(pr, dtype_id)], device=self.model.device)
        pred = self.model.forward(X)[0].tolist()
        ranked = sorted(cands, key=lambda s: pred[s - 1])
        if self.tuner is not None and pred[ranked[1] - 1] - pred[ranked[0] - 1] < self.margin:
            return self.tuner.best(pr, allowed=set(valid)), True
        return ranked[0], False


def dataset(tuner, probs, log=None):
    X, T, M = [], [], []
    for n, pr in enumerate(probs):
        if log and n and n % 2000 == 0:
            log(f"timed {n} problems")
        t = tuner.times(pr)
        X.append(features(pr, dtype_of(pr)))
        T.append([math.log2(x) if x is not None else 0.0 for x in t])
        M.append([1.0 if x is not None else 0.0 for x in t])
    dev = torch.device("cuda", torch.cuda.current_device())
    return (torch.tensor(X, device=dev), torch.tensor(T, device=dev), torch.tensor(M, device=dev))


def regret(tuner, probs, choose, allowed):
    """sum(t_chosen) / sum(t_best) - 1 over problems, and the geometric mean of the ratios."""
    tot_c = tot_b = 0.0
    logs = []
    for pr in probs:
        t = tuner.times(pr)
        best = min(t[s - 1] for s in allowed if t[s - 1] is not None)
        s = choose(pr)
        tc = t[s - 1]
        tot_c += tc
        tot_b += best
        logs.append(math.log(tc / best))
    return tot_c / tot_b - 1.0, math.exp(sum(logs) / len(logs)) - 1.0


def train_and_evaluate(n_train, n_test, steps=3000, seed_train=1, seed_test=2, margin=0.15, log=print,
                       cap=workloads.CAP):
    t0 = time.time()
    tuner = DtypeTuner(cap=cap)
    train = with_dtypes(workloads.problems(n_train, seed_train, cap=cap), seed_train)
    test = with_dtypes(workloads.problems(n_test, seed_test, cap=cap), seed_test)
    X, T, M = dataset(tuner, train, log=log)
    log(f"timed {n_train} training problems in {time.time() - t0:.0f} s")
    model = MLP().fit(X, T, M, steps=steps, log=log)
    out = {"n_train": n_train, "n_test": n_test, "steps": steps, "margin": margin}
    out.update(evaluate(model, tuner, test, margin=margin))
    out["seconds"] = time.time() - t0
    return model, out


def evaluate(model, tuner, test, margin=0.15):
    """Held-out regret of the network with and without the autotuner fallback, and of the
    planner's fixed heuristic (the method without the network), per schedule set."""
    dataset(tuner, test)
    allowed_sets = {"exact": set(EXACT), "fp32_accurate": set(range(1, NS + 1))}
    out = {"f64_share": sum(dtype_of(p) == _lib.F64 for p in test) / max(len(test), 1)}
    for name, allowed in allowed_sets.items():
        sel = Selector(model, tuner, margin=margin)
        fallbacks = [0]

        def pick(pr, sel=sel, allowed=allowed):
            s, fb = sel.choose(pr, allowed)
            fallbacks[0] += int(fb)
            return s

        r_mlp = regret(tuner, test, pick, allowed)
        sel_nofb = Selector(model, None)
        r_nofb = regret(tuner, test, lambda pr: sel_nofb.choose(pr, allowed)[0], allowed)
        # the method without the network: the planner's fixed heuristic
        r_heur = regret(tuner, test, lambda pr: _heuristic_in(pr, allowed), allowed)
        out[name] = {"regret_mlp_with_fallback": r_mlp[0], "geomean_regret_mlp_with_fallback": r_mlp[1],
                     "fallback_rate": fallbacks[0] / len(test),
                     "regret_mlp_alone": r_nofb[0], "geomean_regret_mlp_alone": r_nofb[1],
                     "regret_heuristic": r_heur[0], "geomean_regret_heuristic": r_heur[1]}
    return out


def _heuristic_in(pr, allowed):
    """The planner's default choice for a problem (plain for 'exact', auto for 'fp32_accurate')."""
    inner, nq, outer = geometry(pr["na"], pr["pia"], pr["q"])
    es = 4 if dtype_of(pr) == _lib.F32 else 8
    if pr["m"] <= 16:
        if inner == 1:
            big = math.prod(pr["na"]) * es >= 64 << 20
            return 6 if (6 in allowed and big and nq >= 16 and valid_mask(pr)[5]) else 4
        if 6 in allowed and math.prod(pr["na"]) * es >= 64 << 20 and valid_mask(pr)[5]:
            return 6
        rv = 16 // es
        w = rv if inner % rv == 0 else 1
        return 3 if math.ceil(inner * outer / (32 * w)) < 148 * 32 else 2
    ok = valid_mask(pr)
    if 9 in allowed and ok[8]:
        return 9
    if 7 in allowed and ok[6]:
        return 7
    if 5 in allowed and ok[4]:
        return 5
    return 1


_default = {}


def default_selector(device=None):
    """The selector trained and shipped with the library (schedule_model.json), without fallback."""
    key = str(device)
    if key not in _default:
        with open(MODEL_PATH) as f:
            d = json.load(f)
        _default[key] = Selector(MLP.from_json(d["model"], device=device), None)
    return _default[key]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--test", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--margin", type=float, default=0.15)
    ap.add_argument("--out", default=MODEL_PATH)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    model, res = train_and_evaluate(a.train, a.test, steps=a.steps, margin=a.margin,
                                    log=lambda s: print(s, flush=True))
    with open(a.out, "w") as f:
        json.dump(dict(model=model.to_json(), evaluation=res), f)
    print(json.dumps(res))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
