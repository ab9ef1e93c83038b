"""Generates tests/golden/ref_outputs.npz from the reference tlib::ttm itself.

Runs the reference headers compiled with OpenBLAS (oracle/_ref, built by
oracle/Makefile from the reference sources) on every case of
tests/golden/cases.py with the `combined` policy that operator* and ttmpy
use, and stores each output C (flat, memory order) under key "c<id>".

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import golden_cases, make_inputs  # noqa: E402
from oracle import Reference  # noqa: E402


def main():
    ref = Reference()
    out = {}
    for case in golden_cases():
        a, b, md = make_inputs(case)
        c = np.zeros(int(np.prod(md["nc"])), dtype=a.dtype)
        ref.ttm(case["q"], a, md["na"], md["wa"], md["pia"], b, md["nb"], md["pib"], c, md["nc"], md["wc"])
        out[f"c{case['id']}"] = c
    path = os.path.join(HERE, "ref_outputs.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {len(out)} reference outputs to {path}")


if __name__ == "__main__":
    main()
