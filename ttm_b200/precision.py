"""Precision study: every arithmetic path of the library against the native FP64 kernel.

    python -m ttm_b200.precision [--size 256] [--m 256] [--out study.json]

A is order 4 with extents (S, S, S, S), first-order layout, contracted on each q = 1..4 with a
column-major B of shape (m, S). Two data sets: entries N(0,1), and magnitudes log-uniform on
[1e-4, 1e4] with random signs. The FP64 input (seeded, on the device) runs through the plain
FP64 kernel (the oracle: exact DFMA) and through the ozaki path; its FP32 copy runs through the
plain FP32, bf16x3 and fp8 paths. For every path and case the study reports

    max_rel = max|c - r| / max|r|        (relative error in the infinity norm)
    rms_rel = ||c - r||_2 / ||r||_2      (relative Frobenius error)

against the oracle r, and the path's TFLOP/s (2 m S^4 per TTM, CUDA events, device operands).
At S = 256 the buffers take about 112 GiB of device memory (A and r in FP64, A in FP32, one
output); errors are reduced in chunks so that no full-size temporary is created.
"""
from __future__ import annotations

import argparse
import json
import math
import time

from . import _lib

PATHS = [("fp64_native", _lib.F64, _lib.PREC_PLAIN), ("ozaki", _lib.F64, _lib.PREC_OZAKI),
         ("plain_fp32", _lib.F32, _lib.PREC_PLAIN), ("bf16x3", _lib.F32, _lib.PREC_BF16X3),
         ("fp8", _lib.F32, _lib.PREC_FP8)]
CHUNK = 1 << 26


def _dense(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


def _fill(t, dist, gen):
    """Fill a float64 device tensor in place, chunk by chunk (no full-size temporaries)."""
    import torch
    for s in range(0, t.numel(), CHUNK):
        x = t[s:s + CHUNK]
        if dist == "normal":
            x.normal_(generator=gen)
        else:
            x.uniform_(-4.0, 4.0, generator=gen).mul_(math.log(10.0)).exp_()
            sign = torch.randint(0, 2, (x.numel(),), device=t.device, generator=gen, dtype=torch.int8)
            x.mul_(sign.to(torch.float64).mul_(2).sub_(1))


def _errors(c, r):
    """(max|c-r| / max|r|, ||c-r|| / ||r||), reduced chunk by chunk in float64."""
    import torch
    dmax = rmax = 0.0
    dss = rss = 0.0
    for s in range(0, r.numel(), CHUNK):
        rr = r[s:s + CHUNK]
        d = c[s:s + CHUNK].to(torch.float64).sub_(rr)
        dmax = max(dmax, float(d.abs().max()))
        rmax = max(rmax, float(rr.abs().max()))
        dss += float(torch.dot(d, d))
        rss += float(torch.dot(rr, rr))
    return dmax / rmax, math.sqrt(dss / rss)


def study(size=256, m=256, qs=(1, 2, 3, 4), dists=("normal", "loguniform"), paths=None, reps=3, seed=0,
          log=print):
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    S = size
    n = S ** 4
    na, pia = [S] * 4, [1, 2, 3, 4]
    wa = _dense(na, pia)
    # the FP64 kernel always runs first: it is the reference of every other path
    paths = [p for p in PATHS if p[0] == "fp64_native" or paths is None or p[0] in paths]
    out = {"size": S, "m": m, "layout": "first-order", "b": "column-major (m, S)", "cases": []}
    gen = torch.Generator(device=dev)
    for dist in dists:
        gen.manual_seed(seed)
        A64 = torch.empty(n, dtype=torch.float64, device=dev)
        _fill(A64, dist, gen)
        A32 = A64.to(torch.float32)
        for q in qs:
            nc = list(na)
            nc[q - 1] = m
            wc = _dense(nc, pia)
            B64 = torch.empty(m * S, dtype=torch.float64, device=dev)
            _fill(B64, dist, gen)
            B32 = B64.to(torch.float32)
            nout = n // S * m
            ref = torch.empty(nout, dtype=torch.float64, device=dev)
            case = {"dist": dist, "q": q, "paths": {}}
            for name, dt, prec in paths:
                a, b = (A64, B64) if dt == _lib.F64 else (A32, B32)
                c = ref if name == "fp64_native" else torch.empty(nout, dtype=a.dtype, device=dev)

                def run():
                    _lib.ttm_raw(dt, prec, q, 4, a.data_ptr(), na, wa, pia, b.data_ptr(), [m, S], [1, 2],
                                 c.data_ptr(), nc, wc, stream.cuda_stream)

                run()
                kernel = _lib.last_kernel()
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record(stream)
                for _ in range(reps):
                    run()
                ev[1].record(stream)
                torch.cuda.synchronize(dev)
                t = ev[0].elapsed_time(ev[1]) / 1e3 / reps
                row = {"kernel": kernel, "ms": 1e3 * t, "tflops": 2.0 * m * n / t / 1e12}
                if name != "fp64_native":
                    row["max_rel"], row["rms_rel"] = _errors(c, ref)
                    del c
                case["paths"][name] = row
                log(f"{dist:10s} q={q} {name:12s} {kernel:10s} {1e3 * t:8.2f} ms {row['tflops']:8.1f} TFLOP/s"
                    + (f"  max_rel {row['max_rel']:.2e}  rms_rel {row['rms_rel']:.2e}" if "max_rel" in row else ""))
            out["cases"].append(case)
            del ref, B64, B32
        del A64, A32
        torch.cuda.empty_cache()
    return out


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--m", type=int, default=256)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--paths", default=None, help="comma-separated subset of " + ",".join(p[0] for p in PATHS))
    ap.add_argument("--qs", default="1,2,3,4")
    ap.add_argument("--dists", default="normal,loguniform")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    torch.cuda.set_device(0)
    t0 = time.time()
    res = study(a.size, a.m, qs=[int(x) for x in a.qs.split(",")], dists=a.dists.split(","),
                paths=a.paths.split(",") if a.paths else None, reps=a.reps)
    res["seconds"] = time.time() - t0
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
