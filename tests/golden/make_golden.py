"""Generates the golden fixtures in tests/golden/ from the reference itself.

The reference publishes no test vectors, so these fixtures are outputs of the
UNMODIFIED reference sources compiled single-rank by `make -C oracle ref`
(oracle/_ref/ref_harness_strict, -O2 -fno-fast-math -ffp-contract=off) on
seeded synthetic inputs.  Run from the repository root in a container that has
the reference tree:

    make -C oracle ref && python tests/golden/make_golden.py

Each case stores its parameters, the full halo'd input primitive field and the
interior of the outputs (R for rhs cases; W, U and the dt history for step cases).
"""
import importlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

abi = importlib.import_module("3dnssolver_b200.abi")
wl = importlib.import_module("3dnssolver_b200.workloads")

OUT = os.path.join(ROOT, "tests", "golden", "golden_cases.npz")
P, N = abi.BC_PERIODIC, abi.BC_NEUMANN
SHAPE = (10, 8, 6)

# name, kind, params, seed, smooth, terms/steps
CASES = [
    ("rhs_comp_shu_per_cd2", "rhs", dict(convection=1, weights=0, bc=(P, P, P), diffusion_order=2), 11, True, 3),
    ("rhs_comp_borges_nx_cd4", "rhs", dict(convection=1, weights=1, bc=(N, P, P), diffusion_order=4), 12, False, 3),
    ("rhs_char_shu_per_cd6", "rhs", dict(convection=2, weights=0, bc=(P, P, P), diffusion_order=6), 13, False, 3),
    ("rhs_char_borges_nall_cd2", "rhs", dict(convection=2, weights=1, bc=(N, N, N), diffusion_order=2), 14, False, 3),
    ("rhs_char_shu_nx_cd4", "rhs", dict(convection=2, weights=0, bc=(N, P, P), diffusion_order=4), 15, False, 3),
    ("rhs_conv_only_char_ny", "rhs", dict(convection=2, weights=0, bc=(P, N, P), diffusion_order=2), 16, True, 1),
    ("rhs_diff_only_cd6_ny", "rhs", dict(convection=1, weights=0, bc=(P, N, P), diffusion_order=6), 17, False, 2),
    ("rhs_comp_dim2", "rhs", dict(convection=1, weights=0, bc=(P, P, P), diffusion_order=2, dim=2), 18, False, 3),
    ("step3_comp_per_cd2", "step", dict(convection=1, weights=0, bc=(P, P, P), diffusion_order=2, cfl=0.4), 21, True, 3),
    ("step3_char_nx_cd4", "step", dict(convection=2, weights=0, bc=(N, P, P), diffusion_order=4, cfl=0.3), 22, False, 3),
    ("step2_char_borges_nall_cd6", "step", dict(convection=2, weights=1, bc=(N, N, N), diffusion_order=6, cfl=0.3), 23, True, 2),
]


def params_for(kw):
    kw = dict(kw)
    return abi.make_params(*SHAPE, mu=0.02, Pr=0.72, gamma=1.4, L=(1.0, 0.9, 0.8), **kw)


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/ref_harness_strict missing: run `make -C oracle ref` first")
    g = abi.NS_NGC
    blob, meta = {}, []
    for name, kind, kw, seed, smooth, n in CASES:
        p = params_for(kw)
        W = wl.random_field(p, seed=seed, smooth=smooth)
        blob[name + "/W"] = W
        if kind == "rhs":
            R = O.ref_rhs(p, W, terms=n)
            blob[name + "/R"] = R[g:-g, g:-g, g:-g]
        else:
            Wn, Un, dts = O.ref_run(p, W, n)
            blob[name + "/Wn"] = Wn[g:-g, g:-g, g:-g]
            blob[name + "/Un"] = Un[g:-g, g:-g, g:-g]
            blob[name + "/dt"] = dts
        meta.append(dict(name=name, kind=kind, params=kw, seed=seed, smooth=smooth, n=n))
    blob["meta"] = np.frombuffer(json.dumps(dict(shape=SHAPE, cases=meta)).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1024:.0f} KiB, {len(CASES)} cases)")


if __name__ == "__main__":
    main()
