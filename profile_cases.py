"""One TTM case through the C ABI, repeated: the measurement driver the ncu captures under
profiles/ run.

    python profile_cases.py --dtype f32 --precision bf16x3 --na 256,256,256,16 --q 2 \
        --m 256 [--pia 1,2,3,4] [--iters 3] [--schedule 7]
    python profile_cases.py --batched 64 --precision auto [--iters 3]

A (extents `na`, layout `pia`, dense) and B (m x n_q, column-major) are N(0,1) on the device,
C is allocated on the device; the call is made `iters` times on the current stream. Prints the
kernel the planner chose and the mean time per call (CUDA events, after one untimed call).
With --batched N: the first N problems of the batched workload (ttm_b200.workloads, seed 0) as one
batched plan, run eagerly `iters` times after one untimed run.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from ttm_b200 import _lib  # noqa: E402


def _dense(n, pi):
    w = [1] * len(n)
    for r in range(1, len(n)):
        w[pi[r] - 1] = w[pi[r - 1] - 1] * n[pi[r - 1] - 1]
    return w


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--precision", default="plain", choices=sorted(_lib.PRECISIONS))
    ap.add_argument("--na", default=None, help="comma-separated extents")
    ap.add_argument("--pia", default=None, help="comma-separated layout (default first-order)")
    ap.add_argument("--q", type=int, default=None)
    ap.add_argument("--m", type=int, default=None)
    ap.add_argument("--batched", type=int, default=0, help="run the batched plan of the first N workload problems")
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--schedule", type=int, default=None,
                    help="run this tlibttm_schedule id (tlibttm_ttm_sched) instead of the planner's choice")
    a = ap.parse_args()
    if a.batched:
        return batched(a)
    if a.na is None or a.q is None or a.m is None:
        ap.error("--na, --q and --m are required without --batched")
    na = [int(x) for x in a.na.split(",")]
    pia = [int(x) for x in a.pia.split(",")] if a.pia else list(range(1, len(na) + 1))
    q, m = a.q, a.m
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    dt = _lib.F32 if a.dtype == "f32" else _lib.F64
    tdt = torch.float32 if a.dtype == "f32" else torch.float64
    n = math.prod(na)
    nc = list(na)
    nc[q - 1] = m
    g = torch.Generator(device=dev).manual_seed(0)
    A = torch.randn(n, device=dev, dtype=tdt, generator=g)
    B = torch.randn(m * na[q - 1], device=dev, dtype=tdt, generator=g)
    C = torch.empty(n // na[q - 1] * m, device=dev, dtype=tdt)
    stream = torch.cuda.current_stream(dev).cuda_stream
    prec = _lib.PRECISIONS[a.precision]

    def run():
        if a.schedule is None:
            _lib.ttm_raw(dt, prec, q, len(na), A.data_ptr(), na, _dense(na, pia), pia, B.data_ptr(), [m, na[q - 1]],
                         [1, 2], C.data_ptr(), nc, _dense(nc, pia), stream)
            return
        import ctypes as C_
        from ttm_b200.selector import lib as sched_lib
        _lib.check(sched_lib().tlibttm_ttm_sched(dt, a.schedule, q, len(na), C_.c_void_p(A.data_ptr()), _lib.sz(na),
                                                 _lib.sz(_dense(na, pia)), _lib.sz(pia), C_.c_void_p(B.data_ptr()),
                                                 _lib.sz([m, na[q - 1]]), _lib.sz([1, 2]), C_.c_void_p(C.data_ptr()),
                                                 _lib.sz(nc), _lib.sz(_dense(nc, pia)), C_.c_void_p(stream)))

    run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.iters):
        run()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / a.iters
    es = 4 if a.dtype == "f32" else 8
    gb = es * (n + n // na[q - 1] * m + m * na[q - 1]) / 1e9
    print(f"kernel {_lib.last_kernel()}  {t:.3f} ms/call  {gb / (t / 1e3):.0f} GB/s algorithmic  "
          f"{2.0 * m * n / (t / 1e3) / 1e12:.1f} TFLOP/s")


def batched(a):
    import torch
    from ttm_b200 import workloads
    from ttm_b200.plans import BatchPlan
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    tdt = torch.float32 if a.dtype == "f32" else torch.float64
    probs = workloads.problems(a.batched, seed=0)
    g = torch.Generator(device=dev).manual_seed(1)
    entries = []
    for pr in probs:
        na, q, m = pr["na"], pr["q"], pr["m"]
        n = math.prod(na)
        entries.append(dict(q=q, na=na, pia=pr["pia"], m=m, A=torch.randn(n, device=dev, dtype=tdt, generator=g),
                            B=torch.randn(m, na[q - 1], device=dev, dtype=tdt, generator=g),
                            C=torch.empty(n // na[q - 1] * m, device=dev, dtype=tdt)))
    plan = BatchPlan(entries, precision=a.precision)
    plan.run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.iters):
        plan.run()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / a.iters
    gb = sum(workloads.io_bytes(p, 4 if a.dtype == "f32" else 8) for p in probs) / 1e9
    print(f"batched {a.batched} problems, {plan.launches} launches per run  {t:.3f} ms/run  "
          f"{gb / (t / 1e3):.0f} GB/s algorithmic")
    plan.close()


if __name__ == "__main__":
    main()
