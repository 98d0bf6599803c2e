"""The no-allocation convection entry point against the allocating one.

ns_convection_solve_noalloc serves callers that may not allocate device memory
(hosts that hand out all device memory from their own pool, real-time loops
that cannot pay for cudaMalloc).  Its inputs and output are the caller's device
buffers and its face-flux scratch is an array compiled into the library, so
this test checks that it gives what ns_convection_solve gives, on two calls in
a row with different grids and data (stale scratch from the first call must not
leak into the second), that FP64 results also match the oracle's convection
residual, that the FP32 form and 2D grids (no z faces) match too, and that
grids too large for the array are refused.

This file is named to run last: a failure here leaves every other test already run.
"""
import ctypes
import importlib

import numpy as np
import pytest

from conftest import interior, rel_l2

pkg = importlib.import_module("3dnssolver_b200")
wl = importlib.import_module("3dnssolver_b200.workloads")

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the tolerance of the FP64 parity tests
TOL32 = 1e-5  # FP32 face arithmetic against the FP64 oracle


def _noalloc_fn():
    L = pkg.load_library()
    f = L.ns_convection_solve_noalloc
    f.argtypes = [ctypes.POINTER(pkg.NsParams), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _to_planes(a):
    """Reference host layout [i][j][k][q] -> 5 planes [q][i][j][k]."""
    return np.ascontiguousarray(np.moveaxis(a, -1, 0))


def _from_planes(a):
    return np.ascontiguousarray(np.moveaxis(a, 0, -1))


def _one_call(oracle, p, seed):
    import torch
    W0 = wl.random_field(p, seed=seed, smooth=False)
    W, U = oracle.prologue(p, W0)
    R0 = np.random.default_rng(seed).standard_normal(W.shape)
    with pkg.Solver(p) as s:
        R_ref = s.convection_solve(W, U, R0.copy())
    dW = torch.from_numpy(_to_planes(W)).cuda()
    dU = torch.from_numpy(_to_planes(U)).cuda()
    dR = torch.from_numpy(_to_planes(R0)).cuda()
    torch.cuda.synchronize()
    rc = _noalloc_fn()(ctypes.byref(p), dW.data_ptr(), dU.data_ptr(), dR.data_ptr(),
                       torch.cuda.current_stream().cuda_stream)
    assert rc == 0, pkg.load_library().ns_last_error_string()
    torch.cuda.synchronize()
    R = _from_planes(dR.cpu().numpy())
    # the same kernels as the allocating entry point, in either precision
    err = rel_l2(interior(R - R0), interior(R_ref - R0))
    assert (err <= TOL).all(), f"rel L2 per field against ns_convection_solve {err}"
    np.testing.assert_array_equal(R[:3], R0[:3])  # halos of R are not touched
    # and the oracle's ConvectionScheme::solve restatement
    p64 = pkg.make_params(p.nx, p.ny, p.nz, dim=p.dim, convection=p.convection, weights=p.weights,
                          bc=tuple(p.bc), mu=p.mu, semantics=p.semantics)
    Ro = oracle.convection_solve(p64, W, U, R0)
    err = rel_l2(interior(R - R0), interior(Ro - R0))
    tol = TOL32 if p.precision == pkg.PREC_FP32 else TOL
    assert (err <= tol).all(), f"rel L2 per field against the oracle {err}"


def test_noalloc_matches_allocating_entry_point_twice(oracle):
    P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN
    p1 = pkg.make_params(40, 36, 32, convection=pkg.CONV_WENO5_CHAR, bc=(N, P, P), mu=0.01)
    _one_call(oracle, p1, seed=21)
    p2 = pkg.make_params(17, 23, 12, convection=pkg.CONV_WENO5, weights=pkg.WEIGHTS_BORGES,
                         bc=(P, N, N), mu=0.01)
    _one_call(oracle, p2, seed=22)


def test_noalloc_fp32_and_2d_grids(oracle):
    P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN
    p1 = pkg.make_params(24, 20, 16, convection=pkg.CONV_WENO5_CHAR, bc=(P, N, P), mu=0.01,
                         precision=pkg.PREC_FP32)
    _one_call(oracle, p1, seed=23)
    p2 = pkg.make_params(30, 26, 1, dim=2, convection=pkg.CONV_WENO5_CHAR, bc=(N, P, P), mu=0.01)
    _one_call(oracle, p2, seed=24)
    p3 = pkg.make_params(30, 26, 1, dim=2, convection=pkg.CONV_WENO5, bc=(P, P, P), mu=0.01,
                         precision=pkg.PREC_FP32)
    _one_call(oracle, p3, seed=25)


def test_noalloc_refuses_grids_beyond_its_scratch():
    p = pkg.make_params(96, 96, 96, convection=pkg.CONV_WENO5_CHAR)
    rc = _noalloc_fn()(ctypes.byref(p), ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8),
                       None)
    assert rc == pkg.abi.NS_ERR_INVALID_ARG
    assert b"scratch" in pkg.load_library().ns_last_error_string()
