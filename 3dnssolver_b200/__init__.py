"""B200-native explicit right-hand side and SSP-RK3 time step of a 3D compressible
Navier-Stokes finite-difference solver (drop-in for the hot path of
hamsteri15/3DNSsolver).

The compute path is libns_b200.so (hand-written sm_100a kernels behind the C
ABI of include/ns_b200.h).  This module is a thin ctypes binding; there is no
CPU fallback: if the library is missing or no GPU is visible, calls raise.

Host arrays use the reference container layout (src/containers/array_4d.hpp:64-71):
numpy float64 arrays of shape (nx+6, ny+6, nz+6, 5), C order.
"""
import ctypes
import os

import numpy as np

from . import abi
from .abi import (BC_NEUMANN, BC_PERIODIC, CONV_NONE, CONV_WENO5, CONV_WENO5_CHAR, DIFF_CENTERED,
                  DIFF_NONE, PREC_FP32, PREC_FP64, SEM_PHYSICAL, SEM_REFERENCE, TERM_ALL,
                  TERM_CONVECTION, TERM_DIFFUSION, WEIGHTS_BORGES, WEIGHTS_SHU, NsDiagnostics,
                  NsParams, halo_shape, make_params)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libns_b200.so")

__all__ = ["Solver", "NsError", "make_params", "halo_shape", "load_library", "abi"]

_lib = None


class NsError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def load_library():
    """Loads libns_b200.so and declares the C prototypes; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                          "(python -c 'import __graft_entry__ as g; g.build()')")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER(NsParams)
    C = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    fp = ctypes.POINTER(ctypes.c_float)
    st = ctypes.c_int
    protos = {
        "ns_status_string": ([st], ctypes.c_char_p),
        "ns_last_error_string": ([], ctypes.c_char_p),
        "ns_abi_version": ([], ctypes.c_int),
        "ns_params_default": ([P], st),
        "ns_create": ([P, ctypes.POINTER(C)], st),
        "ns_destroy": ([C], None),
        "ns_set_stream": ([C, C], st),
        "ns_host_array_elems": ([P], ctypes.c_size_t),
        "ns_upload_primitive": ([C, dp], st),
        "ns_download_primitive": ([C, dp], st),
        "ns_download_conservative": ([C, dp], st),
        "ns_convection_solve": ([C, dp, dp, dp], st),
        "ns_diffusion_solve": ([C, dp, dp], st),
        "ns_rhs": ([C, dp, dp, ctypes.c_int], st),
        "ns_compute_dt": ([C, dp, dp], st),
        "ns_time_step": ([C, dp, dp, dp], st),
        "ns_advance": ([C, ctypes.c_int], st),
        "ns_synchronize": ([C], st),
        "ns_get_diagnostics": ([C, ctypes.POINTER(NsDiagnostics)], st),
        "ns_kernel_launches": ([C], ctypes.c_longlong),
        "ns_profile_step": ([C, ctypes.POINTER(ctypes.c_float), ctypes.c_int], st),
        "ns_sensor_init": ([ctypes.c_ulonglong, fp], st),
        "ns_sensor_harvest": ([C, C, C, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong),
                               ctypes.c_double], st),
        "ns_sensor_train": ([C, C, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                             ctypes.c_float, ctypes.c_ulonglong, fp, fp, C], st),
        "ns_sensor_gradients": ([C, C, ctypes.c_int, ctypes.c_float, fp, fp, fp, C], st),
        "ns_sensor_predict": ([C, ctypes.c_longlong, fp, C, C], st),
        "ns_set_sensor_weights": ([C, fp], st),
        "ns_fma_peak": ([ctypes.c_int, dp], st),
        "ns_wait_selftest": ([ctypes.c_uint, ctypes.POINTER(ctypes.c_int), dp], st),
        "ns_div_selftest": ([ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong)], st),
        "ns_get_dt": ([C, dp, dp], st),
        "ns_host_register": ([ctypes.c_void_p, ctypes.c_size_t], st),
        "ns_host_unregister": ([ctypes.c_void_p], st),
    }
    for name, (args, res) in protos.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(status, what):
    if status != 0:
        msg = load_library().ns_last_error_string().decode(errors="replace")
        raise NsError(status, f"{what}: {msg}")


def check_host_array(a, shape, writable=False):
    """Host arrays must be C-contiguous float64 of the reference layout's shape: the C ABI
    takes plain pointers, so an undersized or strided buffer is refused here, on the host."""
    if not isinstance(a, np.ndarray) or a.shape != tuple(shape) or a.dtype != np.float64 \
            or not a.flags["C_CONTIGUOUS"]:
        got = (getattr(a, "shape", None), getattr(a, "dtype", type(a).__name__))
        raise ValueError(f"expected a C-contiguous float64 array of shape {tuple(shape)}, got {got}")
    if writable and not a.flags["WRITEABLE"]:
        raise ValueError("array must be writable")
    return a


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fptr(a):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


# ---------------------------------------------------------------------------
# learned face sensor (device buffers are passed as integer device pointers,
# e.g. torch.Tensor.data_ptr())

SENSOR_FEATURES = 21
SENSOR_NPARAMS = 2145


def fma_peak(fp64=True):
    """Measured FMA throughput of the current device, TFLOP/s (2 flops per FMA)."""
    t = ctypes.c_double()
    _check(load_library().ns_fma_peak(1 if fp64 else 0, ctypes.byref(t)), "ns_fma_peak")
    return t.value


def wait_selftest(polls=4096):
    """Runs one bounded device wait on an mbarrier phase nothing completes;
    returns (ran_out, ms): ran_out is True when the wait gave up as it must."""
    r, t = ctypes.c_int(), ctypes.c_double()
    _check(load_library().ns_wait_selftest(int(polls), ctypes.byref(r), ctypes.byref(t)), "ns_wait_selftest")
    return bool(r.value), t.value


def host_register(a):
    """Page-locks the storage of numpy array a (ns_host_register), so that
    Solver.time_step on it overlaps its copies with the stages; release it with
    host_unregister before the array goes."""
    _check(load_library().ns_host_register(ctypes.c_void_p(a.ctypes.data), a.nbytes), "ns_host_register")


def host_unregister(a):
    _check(load_library().ns_host_unregister(ctypes.c_void_p(a.ctypes.data)), "ns_host_unregister")


def div_selftest(n=1 << 22, seed=7):
    """Largest ulp distances over n draws: (WENO quotient vs IEEE division,
    Newton-Raphson 1/sqrt vs CUDA's rsqrt)."""
    m = (ctypes.c_ulonglong * 2)()
    _check(load_library().ns_div_selftest(int(n), int(seed), m), "ns_div_selftest")
    return int(m[0]), int(m[1])


def sensor_init(seed):
    w = np.zeros(SENSOR_NPARAMS, dtype=np.float32)
    _check(load_library().ns_sensor_init(int(seed), _fptr(w)), "ns_sensor_init")
    return w


def sensor_train(feat_ptr, label_ptr, n, w, *, epochs=5, batch=65536, lr=1e-3, pos_weight=1.0,
                 seed=0, stream=0):
    """Adam training on device samples; returns (new weights, per-epoch mean loss)."""
    w = np.ascontiguousarray(w, dtype=np.float32).copy()
    losses = np.zeros(epochs, dtype=np.float32)
    _check(load_library().ns_sensor_train(ctypes.c_void_p(feat_ptr), ctypes.c_void_p(label_ptr),
                                          int(n), int(epochs), int(batch), float(lr),
                                          float(pos_weight), int(seed), _fptr(w), _fptr(losses),
                                          ctypes.c_void_p(stream)), "ns_sensor_train")
    return w, losses


def sensor_gradients(feat_ptr, label_ptr, n, w, pos_weight=1.0, stream=0):
    w = np.ascontiguousarray(w, dtype=np.float32)
    g = np.zeros(SENSOR_NPARAMS, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    _check(load_library().ns_sensor_gradients(ctypes.c_void_p(feat_ptr), ctypes.c_void_p(label_ptr),
                                              int(n), float(pos_weight), _fptr(w), _fptr(g),
                                              _fptr(loss), ctypes.c_void_p(stream)),
           "ns_sensor_gradients")
    return g, float(loss[0])


def sensor_predict(feat_ptr, n, w, logit_ptr, stream=0):
    w = np.ascontiguousarray(w, dtype=np.float32)
    _check(load_library().ns_sensor_predict(ctypes.c_void_p(feat_ptr), int(n), _fptr(w),
                                            ctypes.c_void_p(logit_ptr), ctypes.c_void_p(stream)),
           "ns_sensor_predict")


class Solver:
    """One device context (ns_ctx): parameters, device state and stream.

    Mirrors the reference objects of the hot path: convection_solve is
    ConvectionScheme::solve, diffusion_solve is DiffusionScheme::solve,
    time_step is TimeScheme::step, advance(n) is n iterations of the Driver loop.
    """

    def __init__(self, params):
        self.lib = load_library()
        self.params = params
        self.shape = halo_shape(params)
        h = ctypes.c_void_p()
        _check(self.lib.ns_create(ctypes.byref(params), ctypes.byref(h)), "ns_create")
        self.h = h

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.ns_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers ----------------------------------------------------------
    def _arr(self, a, writable=False):
        return check_host_array(a, self.shape, writable)

    def new_array(self):
        return np.zeros(self.shape, dtype=np.float64)

    # -- state --------------------------------------------------------------
    def set_stream(self, stream_ptr):
        _check(self.lib.ns_set_stream(self.h, ctypes.c_void_p(stream_ptr)), "ns_set_stream")

    def upload_primitive(self, W):
        _check(self.lib.ns_upload_primitive(self.h, _dptr(self._arr(W))), "ns_upload_primitive")

    def download_primitive(self, out=None):
        out = self.new_array() if out is None else self._arr(out, True)
        _check(self.lib.ns_download_primitive(self.h, _dptr(out)), "ns_download_primitive")
        return out

    def download_conservative(self, out=None):
        out = self.new_array() if out is None else self._arr(out, True)
        _check(self.lib.ns_download_conservative(self.h, _dptr(out)), "ns_download_conservative")
        return out

    # -- operators ------------------------------------------------------------
    def convection_solve(self, W, U, R=None):
        """R += convective residual (ConvectionScheme::solve); returns R."""
        R = self.new_array() if R is None else self._arr(R, True)
        _check(self.lib.ns_convection_solve(self.h, _dptr(self._arr(W)), _dptr(self._arr(U)),
                                            _dptr(R)), "ns_convection_solve")
        return R

    def diffusion_solve(self, W, R=None):
        """R += viscous residual (DiffusionScheme::solve); returns R."""
        R = self.new_array() if R is None else self._arr(R, True)
        _check(self.lib.ns_diffusion_solve(self.h, _dptr(self._arr(W)), _dptr(R)),
               "ns_diffusion_solve")
        return R

    def rhs(self, W, terms=TERM_ALL, R=None):
        R = self.new_array() if R is None else self._arr(R, True)
        _check(self.lib.ns_rhs(self.h, _dptr(self._arr(W)), _dptr(R), int(terms)), "ns_rhs")
        return R

    def compute_dt(self, W):
        dt = ctypes.c_double()
        _check(self.lib.ns_compute_dt(self.h, _dptr(self._arr(W)), ctypes.byref(dt)),
               "ns_compute_dt")
        return dt.value

    def time_step(self, W, U=None):
        """One TimeScheme::step of host W in place (U, if given, receives the conservative state)."""
        self._arr(W, True)
        if U is not None:
            self._arr(U, True)
        dt = ctypes.c_double()
        _check(self.lib.ns_time_step(self.h, _dptr(W), _dptr(U) if U is not None else None,
                                     ctypes.byref(dt)), "ns_time_step")
        return dt.value

    def advance(self, nsteps):
        _check(self.lib.ns_advance(self.h, int(nsteps)), "ns_advance")

    def get_dt(self):
        """(dt of the last step, time accumulated over the steps taken)."""
        dt, t = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.ns_get_dt(self.h, ctypes.byref(dt), ctypes.byref(t)), "ns_get_dt")
        return dt.value, t.value

    def synchronize(self):
        _check(self.lib.ns_synchronize(self.h), "ns_synchronize")

    def diagnostics(self):
        d = NsDiagnostics()
        _check(self.lib.ns_get_diagnostics(self.h, ctypes.byref(d)), "ns_get_diagnostics")
        return {
            "steps": d.steps, "dt": d.dt, "next_dt": d.next_dt, "time": d.time, "mass": d.mass,
            "momentum": list(d.momentum), "energy": d.energy, "kinetic": d.kinetic,
            "enstrophy": d.enstrophy, "nonfinite": bool(d.nonfinite),
            "sensor_fraction": d.sensor_fraction,
        }

    def sensor_harvest(self, feat_ptr, label_ptr, capacity, rel_threshold=1e-3):
        """Features/labels of every face of the current state into device buffers; returns the row count."""
        cnt = ctypes.c_longlong()
        _check(self.lib.ns_sensor_harvest(self.h, ctypes.c_void_p(feat_ptr), ctypes.c_void_p(label_ptr),
                                          int(capacity), ctypes.byref(cnt), float(rel_threshold)),
               "ns_sensor_harvest")
        return cnt.value

    def set_sensor_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(self.lib.ns_set_sensor_weights(self.h, _fptr(w)), "ns_set_sensor_weights")

    def faces(self):
        """Faces per stage along the convected axes (rows of one harvest)."""
        p = self.params
        n = [(p.nx + 1) * p.ny * p.nz, p.nx * (p.ny + 1) * p.nz, p.nx * p.ny * (p.nz + 1)]
        return sum(n[:3 if p.dim == 3 else 2])

    PROFILE_CLASSES = ("step_begin", "fill_prim", "face_x", "face_y", "face_z", "update",
                       "stage_fused", "sensor", "xface_update", "viscous")

    def profile_step(self):
        """One device-resident step with events between kernels: {kernel class: ms}."""
        n = len(self.PROFILE_CLASSES)
        ms = (ctypes.c_float * n)()
        _check(self.lib.ns_profile_step(self.h, ms, n), "ns_profile_step")
        return dict(zip(self.PROFILE_CLASSES, [float(x) for x in ms]))

    @property
    def launches(self):
        return int(self.lib.ns_kernel_launches(self.h))
