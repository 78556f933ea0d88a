"""Writes the golden fixtures tests/golden/*.npz from the oracle (run from the repository root):

    python tests/golden/make_golden.py

The reference (Julia + Trixi.jl) cannot run on this machine, so these vectors are oracle outputs: they
pin the oracle against regressions and give the GPU tests fixed inputs/outputs; they are not
reference-generated.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "trixilw.jl_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import golden_cases  # noqa: E402
import pyoracle  # noqa: E402
import trixilw  # noqa: E402

if __name__ == "__main__":
    for name in golden_cases.CASES:
        out = golden_cases.run_case(name, pyoracle, trixilw)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})
