"""ctypes binding of the CPU oracle and runner of the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The product path
(3dnssolver_b200) never imports this module.
"""
import ctypes
import importlib
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libns_oracle.so")
REF_STRICT = os.path.join(HERE, "_ref", "ref_harness_strict")
REF_TIMED = os.path.join(HERE, "_ref", "ref_harness_timed")

_abi = importlib.import_module("3dnssolver_b200.abi")
NsParams = _abi.NsParams
halo_shape = _abi.halo_shape
params_dict = _abi.params_dict

_lib = None
# int fn(void* user, int what, double* data): what 0 = dt minimum, 1 = x ghost planes of U
SLAB_EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double))


def build():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(NsParams)
        dp = ctypes.POINTER(ctypes.c_double)
        for name, args in {
            "nso_convection_solve": [P, dp, dp, dp],
            "nso_diffusion_solve": [P, dp, dp],
            "nso_face_flux": [P, ctypes.c_int, dp, dp, dp],
            "nso_prologue": [P, dp, dp],
            "nso_rhs": [P, dp, dp, ctypes.c_int],
            "nso_compute_dt": [P, dp, dp],
            "nso_time_step": [P, dp, dp, dp],
            "nso_run": [P, dp, dp, ctypes.c_int, dp],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.nso_slab_run.argtypes = [P, dp, dp, ctypes.c_int, dp, SLAB_EXCHANGE_FN, ctypes.c_void_p]
        L.nso_slab_run.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed ({rc})")


def prologue(p, W):
    """Stage-1 prologue: returns (W, U) halo'd after prim->cons, boundary fill, cons->prim."""
    W = np.ascontiguousarray(W, dtype=np.float64).copy()
    U = np.zeros_like(W)
    _check(lib().nso_prologue(ctypes.byref(p), _ptr(W), _ptr(U)), "prologue")
    return W, U


def rhs(p, W, terms=3):
    R = np.zeros(halo_shape(p))
    W = np.ascontiguousarray(W, dtype=np.float64)
    _check(lib().nso_rhs(ctypes.byref(p), _ptr(W), _ptr(R), terms), "rhs")
    return R


def convection_solve(p, W, U, R=None):
    R = np.zeros(halo_shape(p)) if R is None else R.copy()
    _check(lib().nso_convection_solve(ctypes.byref(p), _ptr(np.ascontiguousarray(W)),
                                      _ptr(np.ascontiguousarray(U)), _ptr(R)), "convection")
    return R


def diffusion_solve(p, W, R=None):
    R = np.zeros(halo_shape(p)) if R is None else R.copy()
    _check(lib().nso_diffusion_solve(ctypes.byref(p), _ptr(np.ascontiguousarray(W)), _ptr(R)),
           "diffusion")
    return R


def face_flux(p, d, W, U):
    f = np.zeros(halo_shape(p))
    _check(lib().nso_face_flux(ctypes.byref(p), d, _ptr(np.ascontiguousarray(W)),
                               _ptr(np.ascontiguousarray(U)), _ptr(f)), "face_flux")
    return f


def compute_dt(p, W):
    dt = ctypes.c_double()
    _check(lib().nso_compute_dt(ctypes.byref(p), _ptr(np.ascontiguousarray(W)), ctypes.byref(dt)),
           "dt")
    return dt.value


def run(p, W, nsteps):
    """nsteps reference time steps; returns (W, U, dts)."""
    W = np.ascontiguousarray(W, dtype=np.float64).copy()
    U = np.zeros_like(W)
    dts = np.zeros(max(nsteps, 1))
    _check(lib().nso_run(ctypes.byref(p), _ptr(W), _ptr(U), nsteps, _ptr(dts)), "run")
    return W, U, dts[:nsteps]


def slab_run(p, W, nsteps, exchange):
    """nsteps on one slab (bc[0] = NS_BC_EXTERNAL); exchange(what, data) fills the x ghost
    planes of U (what = 1, data: the halo'd AoS array) or returns the minimum over slabs
    of a CFL minimum (what = 0, data: a 1-element array it updates).  Returns (W, U, dts)."""
    W = np.ascontiguousarray(W, dtype=np.float64).copy()
    U = np.zeros_like(W)
    dts = np.zeros(max(nsteps, 1))
    shape = W.shape

    def cb(user, what, data):
        try:
            exchange(what, np.ctypeslib.as_array(data, shape=(1,) if what == 0 else shape))
            return 0
        except Exception:
            import traceback
            traceback.print_exc()
            return 1

    fn = SLAB_EXCHANGE_FN(cb)
    _check(lib().nso_slab_run(ctypes.byref(p), _ptr(W), _ptr(U), nsteps, _ptr(dts), fn, None), "slab_run")
    return W, U, dts[:nsteps]


# ---------------------------------------------------------------------------
# reference harness (the unmodified reference sources, built by `make -C oracle ref`)

def ref_available(strict=True):
    return os.path.exists(REF_STRICT if strict else REF_TIMED)


def _ref_args(p):
    d = params_dict(p)
    keys = ["dim", "nx", "ny", "nz", "Lx", "Ly", "Lz", "mu", "Pr", "gamma", "cfl", "conv",
            "weights", "diff", "order", "bcx", "bcy", "bcz"]
    return [f"{k}={d[k]!r}" for k in keys]


def ref_rhs(p, W, terms=3, dump_state=False):
    n = int(np.prod(halo_shape(p)))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "w.bin"), os.path.join(td, "r.bin")
        np.ascontiguousarray(W, dtype=np.float64).tofile(fin)
        subprocess.run([REF_STRICT, "rhs", f"in={fin}", f"out={fout}", f"terms={terms}",
                        f"dump_state={int(dump_state)}"] + _ref_args(p), check=True,
                       env=dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4")))
        raw = np.fromfile(fout, dtype=np.float64)
    R = raw[:n].reshape(halo_shape(p))
    if dump_state:
        return R, raw[n:2 * n].reshape(halo_shape(p)), raw[2 * n:3 * n].reshape(halo_shape(p))
    return R


def ref_run(p, W, nsteps):
    n = int(np.prod(halo_shape(p)))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "w.bin"), os.path.join(td, "s.bin")
        np.ascontiguousarray(W, dtype=np.float64).tofile(fin)
        subprocess.run([REF_STRICT, "step", f"in={fin}", f"out={fout}", f"steps={nsteps}"]
                       + _ref_args(p), check=True,
                       env=dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4")))
        raw = np.fromfile(fout, dtype=np.float64)
        dts = np.fromfile(fout + ".dt", dtype=np.float64)
    return raw[:n].reshape(halo_shape(p)), raw[n:].reshape(halo_shape(p)), dts


def ref_bench(p, steps, warmup=1, threads=None, timed=True, ic="shear"):
    """Times the reference's TimeScheme::step on a synthetic shear layer (ic="shear") or
    Taylor-Green vortex (ic="tgv"); returns the JSON dict."""
    import json
    exe = REF_TIMED if timed else REF_STRICT
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    out = subprocess.run([exe, "bench", f"in={ic}", f"steps={steps}", f"warmup={warmup}"]
                         + _ref_args(p), check=True, capture_output=True, text=True, env=env)
    return json.loads(out.stdout.strip().splitlines()[-1])
