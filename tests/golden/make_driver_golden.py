"""Generates tests/golden/driver_ic.npz: the initial conditions of every test
case the reference's Driver dispatches (src/driver.cpp:107-141), set by the
reference's own src/testcases.cpp compiled into oracle/_ref/ref_harness_strict
(mode `ic`), on an 8 x 6 x 4 grid over a 2.0 x 1.0 x 0.5 box.  The B200 driver's
--dump-ic output is checked against them bit for bit
(tests/test_driver_cpu.py).  Run from the repository root in a container that
has the reference tree:

    make -C oracle ref && python tests/golden/make_driver_golden.py
"""
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "driver_ic.npz")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness_strict")
CASES = ["sod_x", "sod_y", "sod_z", "case3", "case4", "case6", "case12", "case15", "case17",
         "shear_xy", "shear_3d"]
GRID = dict(nx=8, ny=6, nz=4, Lx=2.0, Ly=1.0, Lz=0.5)


def main():
    blob = {}
    with tempfile.TemporaryDirectory() as d:
        for c in CASES:
            out = os.path.join(d, c + ".bin")
            args = [HARNESS, "ic", f"case={c}", "dim=3", f"out={out}"] + [f"{k}={v}" for k, v in GRID.items()]
            subprocess.run(args, check=True, capture_output=True)
            w = np.fromfile(out).reshape(GRID["nx"] + 6, GRID["ny"] + 6, GRID["nz"] + 6, 5)
            blob[c] = w
    blob["grid"] = np.array([GRID["nx"], GRID["ny"], GRID["nz"], GRID["Lx"], GRID["Ly"], GRID["Lz"]])
    np.savez_compressed(OUT, **blob)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
