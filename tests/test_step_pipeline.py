"""ns_time_step with pinned host arrays overlaps its transfers with the stages
(the W upload in chunks of x-planes under the first stage's per-plane work, the
third stage chunk by chunk with each finished chunk of W downloaded while the
next computes).  The same call with pageable arrays runs the unpipelined step.
Both run the same kernels on the same cells, so the results must agree bit for
bit; the pipelined step is also held to the oracle like every other step.

The chunks are 64 x-planes, so the grids here have 2-3 chunks, including a
last chunk of 2 planes and one of 32.
"""
import importlib

import numpy as np
import pytest
import torch

from conftest import interior, rel_l2

pkg = importlib.import_module("3dnssolver_b200")
wl = importlib.import_module("3dnssolver_b200.workloads")

pytestmark = pytest.mark.gpu
P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN


def _same(a, b):
    """bit-for-bit equal (the corner ghost cells hold NaN in both)"""
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def _pinned_like(a):
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return t, out


# CFL numbers at which the oracle keeps these rough random states finite over
# four steps (at 0.4 they reach negative pressure within two or three)
CASES = [
    # (shape, dim, convection, weights, order, bc, semantics, cfl)
    ((160, 12, 20), 3, 2, 0, 2, (P, P, P), pkg.SEM_PHYSICAL, 0.2),
    ((130, 10, 12), 3, 2, 0, 2, (N, P, N), pkg.SEM_REFERENCE, 0.2),
    ((128, 9, 14), 3, 1, 1, 6, (P, N, P), pkg.SEM_PHYSICAL, 0.2),
    ((150, 11, 1), 2, 2, 0, 4, (N, P, P), pkg.SEM_PHYSICAL, 0.2),
    ((140, 8, 10), 3, 1, 0, 4, (N, N, N), pkg.SEM_REFERENCE, 0.1),
]


@pytest.mark.parametrize("shape,dim,conv,weights,order,bc,sem,cfl", CASES)
def test_pipelined_time_step_is_bit_identical(shape, dim, conv, weights, order, bc, sem, cfl):
    p = pkg.make_params(*shape, dim=dim, convection=conv, weights=weights, diffusion_order=order, bc=bc,
                        mu=0.02, cfl=cfl, semantics=sem)
    W0 = wl.random_field(p, seed=23, smooth=False)
    with pkg.Solver(p) as a, pkg.Solver(p) as b:
        Wa, Ua = W0.copy(), a.new_array()                  # pageable: the unpipelined step
        tW, Wb = _pinned_like(W0)
        tU, Ub = _pinned_like(b.new_array())               # pinned: the pipelined step
        for _ in range(3):
            da = a.time_step(Wa, Ua)
            db = b.time_step(Wb, Ub)
            assert da == db
            assert _same(Wa, Wb), "W differs between the pipelined and the unpipelined step"
            assert _same(Ua, Ub), "U differs between the pipelined and the unpipelined step"
            assert np.isfinite(interior(Wb)).all()
        # a device-resident step after a pipelined one starts from the same state
        a.advance(1)
        b.advance(1)
        assert _same(a.download_conservative(), b.download_conservative())
        assert _same(a.download_primitive(), b.download_primitive())
        del Wb, Ub
        del tW, tU


def test_pipelined_time_step_matches_oracle(oracle):
    p = pkg.make_params(150, 10, 12, convection=pkg.CONV_WENO5_CHAR, diffusion_order=2, bc=(N, P, P),
                        mu=0.02, cfl=0.2, semantics=pkg.SEM_PHYSICAL)
    W0 = wl.random_field(p, seed=29, smooth=False)
    Wo, Uo, dto = oracle.run(p, W0, 3)
    with pkg.Solver(p) as s:
        tW, Wg = _pinned_like(W0)
        dts = [s.time_step(Wg) for _ in range(3)]
        np.testing.assert_allclose(dts, dto, rtol=1e-13)
        err = rel_l2(interior(Wg), interior(Wo))
        assert (err <= 1e-12).all(), f"rel L2 per field {err}"
        del Wg, tW


def test_pipelined_time_step_without_u_download():
    """W only (the end-to-end benchmark's call): the pipelined step's W and the
    state it leaves on the device match the unpipelined call's."""
    p = pkg.make_params(192, 8, 16, convection=pkg.CONV_WENO5_CHAR, diffusion_order=2, mu=0.01, cfl=0.3,
                        semantics=pkg.SEM_PHYSICAL)
    W0 = wl.random_field(p, seed=31, smooth=True)
    with pkg.Solver(p) as a, pkg.Solver(p) as b:
        Wa = W0.copy()
        tW, Wb = _pinned_like(W0)
        for _ in range(2):
            a.time_step(Wa)
            b.time_step(Wb)
        assert _same(Wa, Wb) and np.isfinite(interior(Wb)).all()
        assert _same(a.download_conservative(), b.download_conservative())
        del Wb, tW


def test_registered_host_arrays_take_the_pipeline():
    """ns_host_register page-locks a caller's pageable array: the step on it
    takes the pipelined path (its chunked launches) and gives the same bits."""
    p = pkg.make_params(130, 10, 12, convection=pkg.CONV_WENO5_CHAR, diffusion_order=2, mu=0.02, cfl=0.2,
                        semantics=pkg.SEM_PHYSICAL)
    W0 = wl.random_field(p, seed=37, smooth=False)
    with pkg.Solver(p) as a, pkg.Solver(p) as b:
        Wa = W0.copy()
        Wb = W0.copy()
        pkg.host_register(Wb)
        try:
            for _ in range(2):
                a.time_step(Wa)
                b.time_step(Wb)
            assert _same(Wa, Wb) and np.isfinite(interior(Wb)).all()
            assert b.launches > a.launches
        finally:
            pkg.host_unregister(Wb)
