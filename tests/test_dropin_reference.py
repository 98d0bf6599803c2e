"""The drop-in itself: the UNMODIFIED reference time loop (TimeScheme::step,
src/time_scheme.cpp:3-70) driving the B200 operators through the C++ adapters
of 3dnssolver_b200/adapters/ns_b200_adapters.hpp, and the B200 GpuTimeScheme,
against the reference's own CPU operators in the same process
(oracle/_ref/ref_gpu_harness, built from the reference sources by oracle/Makefile)."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_harness")
W0 = os.path.join(ROOT, "tests", "golden", "golden_cases.npz")

CASES = [
    dict(conv=1, weights=0, order=2, bcx=0, bcy=0, bcz=0),
    dict(conv=2, weights=0, order=4, bcx=1, bcy=0, bcz=0),
    dict(conv=2, weights=1, order=6, bcx=1, bcy=1, bcz=1),
]


@pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/ref_gpu_harness not built here")
@pytest.mark.parametrize("case", CASES, ids=lambda c: "conv%(conv)d_cd%(order)d_bc%(bcx)d%(bcy)d%(bcz)d" % c)
def test_reference_time_loop_with_b200_operators(case, tmp_path):
    import importlib
    import numpy as np
    abi = importlib.import_module("3dnssolver_b200.abi")
    wl = importlib.import_module("3dnssolver_b200.workloads")
    p = abi.make_params(18, 14, 12, convection=case["conv"], weights=case["weights"],
                        diffusion_order=case["order"], bc=(case["bcx"], case["bcy"], case["bcz"]),
                        mu=0.02, cfl=0.3, L=(1.0, 0.9, 0.8))
    W = wl.random_field(p, seed=41, smooth=False)
    fin = tmp_path / "w.bin"
    np.ascontiguousarray(W).tofile(fin)
    args = [f"{k}={v!r}" for k, v in abi.params_dict(p).items()
            if k in ("dim", "nx", "ny", "nz", "Lx", "Ly", "Lz", "mu", "Pr", "gamma", "cfl", "conv",
                     "weights", "diff", "order", "bcx", "bcy", "bcz")]
    out = subprocess.run([EXE, "dropin", f"in={fin}", "steps=3"] + args, capture_output=True, text=True,
                         timeout=300, env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert out.returncode == 0, out.stderr
    r = json.loads(out.stdout.strip().splitlines()[-1])
    dtA, dtB, dtC = r["dt"]
    assert dtB == pytest.approx(dtA, rel=1e-13) and dtC == pytest.approx(dtA, rel=1e-13)
    assert max(r["operators"]) <= 1e-12, r
    assert max(r["time_scheme"]) <= 1e-12, r
