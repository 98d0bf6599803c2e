"""The oracle against the golden fixtures made by the reference itself (bit-exact)."""
import importlib

import numpy as np
import pytest

from conftest import interior, load_golden

abi = importlib.import_module("3dnssolver_b200.abi")

Z, META = load_golden()
CASES = META["cases"]


def _params(kw):
    return abi.make_params(*META["shape"], mu=0.02, Pr=0.72, gamma=1.4, L=(1.0, 0.9, 0.8), **kw)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_golden(case, oracle):
    p = _params(case["params"])
    W = Z[case["name"] + "/W"]
    if case["kind"] == "rhs":
        R = oracle.rhs(p, W, terms=case["n"])
        np.testing.assert_array_equal(interior(R), Z[case["name"] + "/R"])
    else:
        Wn, Un, dts = oracle.run(p, W, case["n"])
        np.testing.assert_array_equal(dts, Z[case["name"] + "/dt"])
        np.testing.assert_array_equal(interior(Wn), Z[case["name"] + "/Wn"])
        np.testing.assert_array_equal(interior(Un), Z[case["name"] + "/Un"])


def test_golden_inputs_are_the_seeded_workloads(wl):
    """The stored inputs are what workloads.random_field produces (generator unchanged)."""
    for case in CASES:
        p = _params(case["params"])
        W = wl.random_field(p, seed=case["seed"], smooth=case["smooth"])
        np.testing.assert_array_equal(W, Z[case["name"] + "/W"])


def test_golden_outputs_are_finite_and_nontrivial():
    for case in CASES:
        keys = ["/R"] if case["kind"] == "rhs" else ["/Wn", "/Un"]
        for k in keys:
            a = Z[case["name"] + k]
            assert np.isfinite(a).all()
            assert np.abs(a).max() > 0
