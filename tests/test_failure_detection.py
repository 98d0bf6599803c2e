"""Failure detection without a GPU fault: bad values are planted on the host (in
the uploaded initial condition), the device only computes with them, and the
state check of params.check_finite reports them as NS_ERR_NONFINITE.

The reference lets NaN propagate silently (its CFL minimum ignores NaN and the
time step falls back to the 1e10 sentinel, src/time_scheme.cpp:104-117); with
check_finite = 0 the library behaves the same way, which the last test pins."""
import importlib
import math

import numpy as np
import pytest

pkg = importlib.import_module("3dnssolver_b200")
wl = importlib.import_module("3dnssolver_b200.workloads")

pytestmark = pytest.mark.gpu
P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN


def _params(check, **kw):
    args = dict(convection=pkg.CONV_WENO5_CHAR, diffusion_order=2, bc=(N, P, P), mu=0.01, cfl=0.3,
                check_finite=check)
    args.update(kw)
    return pkg.make_params(14, 10, 8, **args)


@pytest.mark.parametrize("prec", [pkg.PREC_FP64, pkg.PREC_FP32])
@pytest.mark.parametrize("plant", ["nan_pressure", "inf_velocity", "negative_density"])
def test_planted_bad_cell_is_reported(prec, plant):
    p = _params(1, precision=prec)
    W = wl.random_field(p, seed=3, smooth=True)
    c = (3 + 6, 3 + 4, 3 + 2)
    if plant == "nan_pressure":
        W[c + (1,)] = math.nan
    elif plant == "inf_velocity":
        W[c + (2,)] = math.inf
    else:
        W[c + (0,)] = -0.5
    with pkg.Solver(p) as s:
        s.upload_primitive(W)
        with pytest.raises(pkg.NsError) as e:
            s.synchronize()  # the uploaded state itself is checked
        assert e.value.status == pkg.abi.NS_ERR_NONFINITE
        with pytest.raises(pkg.NsError) as e:
            s.advance(2)
        assert e.value.status == pkg.abi.NS_ERR_NONFINITE
        assert "interior cells" in str(e.value)


def test_time_step_reports_after_returning_the_state():
    p = _params(1)
    W = wl.random_field(p, seed=4, smooth=True)
    W[3 + 2, 3 + 2, 3 + 2, 1] = math.nan
    with pkg.Solver(p) as s:
        Wh = W.copy()
        with pytest.raises(pkg.NsError) as e:
            s.time_step(Wh)
        assert e.value.status == pkg.abi.NS_ERR_NONFINITE
    # the step ran and the state came back: the NaN spread to the stencil neighbourhood
    assert np.isnan(Wh[3:-3, 3:-3, 3:-3, 1]).sum() > 1


def test_clean_state_passes_the_check():
    p = _params(1)
    W = wl.random_field(p, seed=5, smooth=True)
    with pkg.Solver(p) as s:
        s.upload_primitive(W)
        s.advance(3)
        s.synchronize()
        Wh = W.copy()
        s.time_step(Wh)
    # interior cells (edge and corner ghost cells are never filled, as in the reference)
    assert np.isfinite(Wh[3:-3, 3:-3, 3:-3]).all()


def test_without_the_check_nan_propagates_silently_as_in_the_reference():
    p = _params(0)
    W = wl.random_field(p, seed=6, smooth=True)
    W[3 + 5, 3 + 5, 3 + 3, 1] = math.nan
    with pkg.Solver(p) as s:
        s.upload_primitive(W)
        s.advance(2)
        s.synchronize()
        d = s.diagnostics()
    assert d["nonfinite"]
    assert math.isfinite(d["dt"]) and d["dt"] > 0  # NaN never lowers the CFL minimum


@pytest.mark.gpu
def test_bounded_device_wait_gives_up_and_the_device_stays_usable():
    """Every TMA and tensor-core kernel waits on mbarriers with a poll limit; a wait
    on a phase that nothing completes must give up, report, and leave the context
    usable (no fault, no trap)."""
    ran_out, ms = pkg.wait_selftest(4096)
    assert ran_out
    assert ms < 1000.0
    p = pkg.make_params(12, 10, 9, convection=pkg.CONV_WENO5_CHAR, mu=0.01)
    with pkg.Solver(p) as s:
        s.upload_primitive(wl.random_field(p, seed=2))
        s.advance(1)
        s.synchronize()
