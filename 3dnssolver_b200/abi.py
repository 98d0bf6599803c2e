"""ctypes description of the C ABI declared in include/ns_b200.h.

The structs here must stay field-for-field identical to the header; the
CPU test suite checks the sizes against the compiled library.
"""
import ctypes

NS_NGC = 3
NS_NQ = 5

NS_OK = 0
NS_ERR_INVALID_ARG = 1
NS_ERR_OOM = 2
NS_ERR_CUDA = 3
NS_ERR_NONFINITE = 4
NS_ERR_TIMEOUT = 5
NS_ERR_UNSUPPORTED = 6
NS_ERR_NO_DEVICE = 7

CONV_NONE, CONV_WENO5, CONV_WENO5_CHAR = 0, 1, 2
WEIGHTS_SHU, WEIGHTS_BORGES = 0, 1
DIFF_NONE, DIFF_CENTERED = 0, 1
BC_PERIODIC, BC_NEUMANN, BC_EXTERNAL = 0, 1, 2
EXCHANGE_DT, EXCHANGE_HALO = 0, 1
PREC_FP64, PREC_FP32 = 0, 1
SEM_REFERENCE, SEM_PHYSICAL = 0, 1
TERM_CONVECTION, TERM_DIFFUSION, TERM_ALL = 1, 2, 3


class NsParams(ctypes.Structure):
    """Mirror of ns_params (hot-path fields of the reference Params, src/params.hpp:20-43)."""

    _fields_ = [
        ("dim", ctypes.c_int),
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("nz", ctypes.c_int),
        ("Lx", ctypes.c_double),
        ("Ly", ctypes.c_double),
        ("Lz", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("Pr", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("convection", ctypes.c_int),
        ("weights", ctypes.c_int),
        ("diffusion", ctypes.c_int),
        ("diffusion_order", ctypes.c_int),
        ("bc", ctypes.c_int * 3),
        ("precision", ctypes.c_int),
        ("semantics", ctypes.c_int),
        ("sensor", ctypes.c_int),
        ("sensor_threshold", ctypes.c_double),
        ("check_finite", ctypes.c_int),
        ("slab_x0", ctypes.c_int),
        ("slab_nx", ctypes.c_int),
        ("slab_periodic", ctypes.c_int),
        ("sensor_period", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


class NsDiagnostics(ctypes.Structure):
    """Mirror of ns_diagnostics."""

    _fields_ = [
        ("steps", ctypes.c_longlong),
        ("dt", ctypes.c_double),
        ("next_dt", ctypes.c_double),
        ("time", ctypes.c_double),
        ("mass", ctypes.c_double),
        ("momentum", ctypes.c_double * 3),
        ("energy", ctypes.c_double),
        ("kinetic", ctypes.c_double),
        ("enstrophy", ctypes.c_double),
        ("nonfinite", ctypes.c_int),
        ("sensor_fraction", ctypes.c_double),
    ]


def make_params(nx, ny, nz, *, dim=3, L=(1.0, 1.0, 1.0), mu=1e-3, Pr=0.72, gamma=1.4, cfl=0.5,
                convection=CONV_WENO5, weights=WEIGHTS_SHU, diffusion=DIFF_CENTERED,
                diffusion_order=2, bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC),
                precision=PREC_FP64, semantics=SEM_REFERENCE, sensor=0, sensor_threshold=0.5,
                check_finite=0, slab=None, sensor_period=1):
    """slab = (x0, nx_global, periodic): this context is the slab of cells x0..x0+nx-1 of a
    domain of nx_global cells along x split across ranks (bc[0] becomes BC_EXTERNAL)."""
    p = NsParams()
    p.dim, p.nx, p.ny, p.nz = dim, nx, ny, nz
    p.Lx, p.Ly, p.Lz = L
    p.mu, p.Pr, p.gamma, p.cfl = mu, Pr, gamma, cfl
    p.convection, p.weights = convection, weights
    p.diffusion, p.diffusion_order = diffusion, diffusion_order
    for a in range(3):
        p.bc[a] = bc[a]
    p.precision, p.semantics = precision, semantics
    p.sensor, p.sensor_threshold = sensor, sensor_threshold
    p.check_finite = check_finite
    p.sensor_period = sensor_period
    if slab is not None:
        p.bc[0] = BC_EXTERNAL
        p.slab_x0, p.slab_nx, p.slab_periodic = int(slab[0]), int(slab[1]), int(bool(slab[2]))
    return p


def params_dict(p):
    """Plain-dict view of an NsParams (for logs and the reference harness)."""
    return {
        "dim": p.dim, "nx": p.nx, "ny": p.ny, "nz": p.nz,
        "Lx": p.Lx, "Ly": p.Ly, "Lz": p.Lz, "mu": p.mu, "Pr": p.Pr, "gamma": p.gamma,
        "cfl": p.cfl, "conv": p.convection, "weights": p.weights, "diff": p.diffusion,
        "order": p.diffusion_order, "bcx": p.bc[0], "bcy": p.bc[1], "bcz": p.bc[2],
        "precision": p.precision, "semantics": p.semantics, "sensor": p.sensor,
    }


def halo_shape(p):
    """Shape of a host array in the reference layout: (nx+6, ny+6, nz+6, 5)."""
    return (p.nx + 2 * NS_NGC, p.ny + 2 * NS_NGC, p.nz + 2 * NS_NGC, NS_NQ)
