"""Layout/mode sweep: throughput of every case of the 2^26-element sweep on one GPU.

    python -m ttm_b200.sweep [--dtypes f32,f64] [--ms 1,8,64,512] [--layouts 10] [--out sweep.json]
                             [--check [--samples 2048]] [--precision auto]

A has prod(n) = 2^26 elements: the extent sets (512,256,512), (128,64,128,64), (32,32,64,32,32),
(32,16,32,16,16,16) and two seeded random splits of the 26 bits over p = 3..6 modes (every
extent >= 2). Every q is contracted under the first-order layout, the last-order layout and
seeded random permutations, with m in {1, 8, 64, 512}, entries N(0,1), B column-major, FP32 and
FP64, device operands, the library's default arithmetic (exact FMA in the I/O type). Cases whose
C would exceed 64 GB are skipped (listed in the output).

Per case: the kernel the planner chose, time (CUDA events around `reps` back-to-back calls after
one untimed call), GB/s of algorithmic bytes s (N_A + N_C + m n_q) and its fraction of the
measured HBM copy bandwidth, and TFLOP/s (2 m N_A). Inputs exceed L2 (256 MB in FP32), so no
flush is needed.
"""
from __future__ import annotations

import argparse
import json
import math
import os

from . import _lib

FIXED = [(512, 256, 512), (128, 64, 128, 64), (32, 32, 64, 32, 32), (32, 16, 32, 16, 16, 16)]
# Largest C (elements) a case may write: 64 GB in either type, so that A, B and C fit on one
# B200 beside the checker's samples; the cases above it (m = 512 with n_q = 2 in double) are
# listed as skipped.
MAX_C = {"f32": 1 << 34, "f64": 1 << 33}


def _dense(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


def extent_sets(seed=0, random_sets=2):
    """The four fixed extent sets and `random_sets` seeded splits of 26 bits (extents >= 2)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sets = [list(s) for s in FIXED]
    for _ in range(random_sets):
        p = int(rng.integers(3, 7))
        bits = [1] * p
        for _ in range(26 - p):
            bits[int(rng.integers(0, p))] += 1
        sets.append([1 << b for b in bits])
    return sets


def layouts(p, count, seed):
    """First-order, last-order, then distinct seeded random permutations (count in all, at most p!)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    count = min(count, math.factorial(p))
    out = [list(range(1, p + 1)), list(range(p, 0, -1))][:count]
    while len(out) < count:
        pi = [int(x) + 1 for x in rng.permutation(p)]
        if pi not in out:
            out.append(pi)
    return out


def view3(na, pia, q):
    """(outer, n_q, inner) of the slice view of a tensor dense under layout pia."""
    qh = pia.index(q)
    inner = math.prod(na[pia[r] - 1] for r in range(qh))
    outer = math.prod(na[pia[r] - 1] for r in range(qh + 1, len(na)))
    return outer, na[q - 1], inner


def sample_fibres(A, B, C, na, pia, q, m, count, gen, b_cm=True):
    """Gathers `count` random output fibres: A_s (count x n_q) and C_s (count x m) as float64
    numpy arrays, and B as a float64 (m x n_q) array. Each fibre is (k, i) of the slice view:
    A_s[s, l] = A[k][l][i], C_s[s, j] = C[k][j][i]."""
    import torch
    outer, nq, inner = view3(na, pia, q)
    n = outer * inner
    idx = torch.randint(0, n, (min(count, n),), device=A.device, generator=gen) if count < n else \
        torch.arange(n, device=A.device)
    ks, iis = idx // inner, idx % inner
    a_s = A.view(outer, nq, inner)[ks, :, iis].double().cpu().numpy()
    c_s = C.view(outer, m, inner)[ks, :, iis].double().cpu().numpy()
    b = B.double().cpu().numpy()
    b = b.reshape(nq, m).T if b_cm else b.reshape(m, nq)
    return a_s, b, c_s


def fibre_errors(a_s, b, c_s):
    """max|c - r| / max|r| and ||c - r|| / ||r|| over the sampled fibres, r = a_s b^T in FP64."""
    import numpy as np
    r = a_s @ b.T
    d = c_s - r
    rmax = float(np.max(np.abs(r))) or 1.0
    rn = float(np.linalg.norm(r)) or 1.0
    return float(np.max(np.abs(d))) / rmax, float(np.linalg.norm(d)) / rn


def hbm_peak():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def sweep(dtypes=("f32", "f64"), ms=(1, 8, 64, 512), n_layouts=10, reps=10, seed=0, log=print, check=False,
          samples=2048, precision=None):
    """Times every case; with `check`, also compares `samples` sampled output fibres per case with
    FP64 dot products (fields max_rel and rms_rel). `precision` is a key of _lib.PRECISIONS (the
    library default when None)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    peak, kind = hbm_peak()
    out = {"hbm_peak_gbs": peak, "peak_kind": kind, "cases": [], "skipped": []}
    n = 1 << 26
    for dname in dtypes:
        dt = _lib.F32 if dname == "f32" else _lib.F64
        tdt = torch.float32 if dname == "f32" else torch.float64
        es = 4 if dname == "f32" else 8
        gen = torch.Generator(device=dev).manual_seed(seed)
        A = torch.randn(n, device=dev, dtype=tdt, generator=gen)
        for si, na in enumerate(extent_sets(seed)):
            p = len(na)
            for pia in layouts(p, n_layouts, seed + si):
                wa = _dense(na, pia)
                for q in range(1, p + 1):
                    nq = na[q - 1]
                    for m in ms:
                        nout = n // nq * m
                        if nout > MAX_C[dname]:
                            out["skipped"].append({"dtype": dname, "na": na, "pia": pia, "q": q, "m": m})
                            continue
                        nc = list(na)
                        nc[q - 1] = m
                        wc = _dense(nc, pia)
                        B = torch.randn(m * nq, device=dev, dtype=tdt, generator=gen)
                        C = torch.empty(nout, device=dev, dtype=tdt)

                        prec = _lib.PRECISIONS[precision] if precision else _lib.PREC_DEFAULT

                        def run():
                            _lib.ttm_raw(dt, prec, q, p, A.data_ptr(), na, wa, pia, B.data_ptr(),
                                         [m, nq], [1, 2], C.data_ptr(), nc, wc, stream.cuda_stream)

                        run()
                        kernel = _lib.last_kernel()
                        # reps calls back to back between two events: the host's per-call cost is
                        # hidden behind the queued kernels, as in a stream of calls
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        for _ in range(reps):
                            run()
                        e1.record(stream)
                        e1.synchronize()
                        t = e0.elapsed_time(e1) / 1e3 / reps
                        gbs = es * (n + nout + m * nq) / t / 1e9
                        row = {"dtype": dname, "na": na, "pia": pia, "q": q, "m": m, "kernel": kernel,
                               "ms": 1e3 * t, "gbs": gbs, "hbm_frac": gbs / peak, "tflops": 2.0 * m * n / t / 1e12}
                        if check:
                            a_s, b_s, c_s = sample_fibres(A, B, C, na, pia, q, m, samples, gen)
                            row["max_rel"], row["rms_rel"] = fibre_errors(a_s, b_s, c_s)
                        out["cases"].append(row)
                        del B, C
        del A
        torch.cuda.empty_cache()
    out["summary"] = summarize(out["cases"])
    for line in format_summary(out["summary"]):
        log(line)
    return out


def summarize(cases):
    s = {}
    for dname in sorted({c["dtype"] for c in cases}):
        for m in sorted({c["m"] for c in cases}):
            rows = [c for c in cases if c["dtype"] == dname and c["m"] == m]
            if not rows:
                continue
            fr = sorted(c["hbm_frac"] for c in rows)
            tf = sorted(c["tflops"] for c in rows)
            kernels = {}
            for c in rows:
                kernels[c["kernel"]] = kernels.get(c["kernel"], 0) + 1
            s[f"{dname}_m{m}"] = {"cases": len(rows), "hbm_frac_min": fr[0], "hbm_frac_median": fr[len(fr) // 2],
                                  "hbm_frac_max": fr[-1], "at_least_85pct": sum(f >= 0.85 for f in fr) / len(fr),
                                  "tflops_median": tf[len(tf) // 2], "kernels": kernels}
            if all("rms_rel" in c for c in rows):
                s[f"{dname}_m{m}"]["max_rel_worst"] = max(c["max_rel"] for c in rows)
                s[f"{dname}_m{m}"]["rms_rel_worst"] = max(c["rms_rel"] for c in rows)
    return s


def format_summary(s):
    lines = []
    for k, v in s.items():
        lines.append(f"{k:8s} {v['cases']:4d} cases  HBM frac min {v['hbm_frac_min']:.2f} median "
                     f"{v['hbm_frac_median']:.2f} max {v['hbm_frac_max']:.2f}  >=85%: {100 * v['at_least_85pct']:.0f}%"
                     f"  TFLOP/s median {v['tflops_median']:.1f}  {v['kernels']}")
    return lines


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--dtypes", default="f32,f64")
    ap.add_argument("--ms", default="1,8,64,512")
    ap.add_argument("--layouts", type=int, default=10)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--out", default=None)
    ap.add_argument("--check", action="store_true", help="compare sampled fibres with FP64 dot products")
    ap.add_argument("--samples", type=int, default=2048)
    ap.add_argument("--precision", default=None)
    a = ap.parse_args()
    torch.cuda.set_device(0)
    res = sweep(a.dtypes.split(","), [int(x) for x in a.ms.split(",")], a.layouts, a.reps, check=a.check,
                samples=a.samples, precision=a.precision)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)


if __name__ == "__main__":
    main()
