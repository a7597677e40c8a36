"""Generate the golden vectors of tests/golden/ from the reference's own code.

The only part of the reference that runs here is its compiled interpolator
ba_interp2.cpp (oracle/_ref, built by oracle/Makefile from the reference
sources).  This script drives it through its mexFunction, exactly as MATLAB
calls it, on seeded inputs, and stores inputs and outputs:

    python tests/golden/make_golden.py

(needs oracle/_ref/libba_interp2_ref.so, i.e. the reference sources at build
time).  The fixtures are small (< 100 KB).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402


def main():
    rng = np.random.default_rng(20201)
    out = {}
    # image 23 x 17 (MATLAB M=17 rows, N=23 columns), 3 channels
    F = rng.standard_normal((3, 23, 17))
    n = 400
    X = rng.uniform(-2.5, 26.0, n)   # columns, includes clamped borders
    Y = rng.uniform(-2.5, 20.0, n)   # rows
    X[:8] = np.arange(1, 9)          # integer nodes
    Y[:8] = np.arange(1, 9) + 0.5
    for name, dt in (("f64", np.float64), ("f32", np.float32)):
        Fd, Xd, Yd = F.astype(dt), X.astype(dt), Y.astype(dt)
        out[f"F_{name}"] = Fd
        out[f"X_{name}"] = Xd
        out[f"Y_{name}"] = Yd
        out[f"Z_{name}"] = oracle.ref_ba_interp2(Fd, Xd, Yd)
        out[f"Z1_{name}"] = oracle.ref_ba_interp2(Fd[0], Xd, Yd)
    np.savez_compressed(os.path.join(HERE, "ba_interp2_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "ba_interp2_ref.npz"))


if __name__ == "__main__":
    main()
