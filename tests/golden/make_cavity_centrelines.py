"""Writes tests/golden/cavity_centrelines_re1000.npz from the reference repository's physics data:

    python tests/golden/make_cavity_centrelines.py <TrixiLW.jl checkout>
    (or with TLW_REFERENCE_ROOT=<TrixiLW.jl checkout> in the environment)

The reference ships the tabulated lid-driven-cavity centrelines at Re = 1000 (Ghia, Ghia & Shin 1982) that
its utils/extract_lid_driven_cavity.jl compares its cavity run against: data/lid_driven_cavity_y_vs_u1_r1000.txt
(y, v1 on the line x = 0.5) and data/lid_driven_cavity_x_vs_u2_r1000.txt (x, v2 on the line y = 0.5). They are
copied here as arrays so that the GPU test needs no reference tree.
"""
import os

import numpy as np

import sys

HERE = os.path.dirname(os.path.abspath(__file__))

if __name__ == "__main__":
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TLW_REFERENCE_ROOT")
    if not REF:
        raise SystemExit("give the reference checkout as an argument or in TLW_REFERENCE_ROOT")
    y_u1 = np.loadtxt(os.path.join(REF, "data", "lid_driven_cavity_y_vs_u1_r1000.txt"))
    x_u2 = np.loadtxt(os.path.join(REF, "data", "lid_driven_cavity_x_vs_u2_r1000.txt"))
    np.savez_compressed(os.path.join(HERE, "cavity_centrelines_re1000.npz"), y_u1=y_u1, x_u2=x_u2)
    print(y_u1.shape, x_u2.shape)
