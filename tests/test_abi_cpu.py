"""C-ABI checks that need no GPU: the library loads, exports every declared
symbol, its structs match the ctypes mirror, and validation errors come back
as status codes before any device work."""
import ctypes
import importlib
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pkg = importlib.import_module("3dnssolver_b200")
HEADER = os.path.join(ROOT, "include", "ns_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^NS_API [^;(]*?\b(ns_\w+)\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib_path = pkg.LIB_PATH
    assert os.path.exists(lib_path), "libns_b200.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (ns_\w+)$", out, flags=re.M))
    decl = declared_symbols()
    assert len(decl) >= 20
    missing = [s for s in decl if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    L = pkg.load_library()
    for s in decl:
        assert hasattr(L, s)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ns_b200.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(ns_params), sizeof(ns_diagnostics),'
                   ' offsetof(ns_params, sensor_threshold), offsetof(ns_diagnostics, sensor_fraction));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(pkg.NsParams)
    assert vals[1] == ctypes.sizeof(pkg.NsDiagnostics)
    assert vals[2] == pkg.NsParams.sensor_threshold.offset
    assert vals[3] == pkg.NsDiagnostics.sensor_fraction.offset


def test_abi_version_and_status_strings():
    L = pkg.load_library()
    assert L.ns_abi_version() == 1
    assert L.ns_status_string(0) == b"ok"
    assert L.ns_status_string(1) == b"invalid argument"


def test_params_default_and_host_elems():
    L = pkg.load_library()
    p = pkg.NsParams()
    assert L.ns_params_default(ctypes.byref(p)) == 0
    assert (p.dim, p.nx, p.diffusion_order, p.gamma) == (3, 64, 2, 1.4)
    assert L.ns_host_array_elems(ctypes.byref(p)) == 70 * 70 * 70 * 5


@pytest.mark.parametrize("field,value", [
    ("nx", 2), ("dim", 4), ("diffusion_order", 3), ("gamma", 1.0), ("cfl", 0.0),
    ("convection", 7), ("precision", 3), ("semantics", 5), ("Lx", -1.0), ("check_finite", 2),
])
def test_invalid_params_rejected_before_device_work(field, value):
    p = pkg.make_params(8, 8, 8)
    setattr(p, field, value)
    with pytest.raises(pkg.NsError) as e:
        pkg.Solver(p)
    assert e.value.status == 1


def test_bad_boundary_and_sensor_combinations_rejected():
    p = pkg.make_params(8, 8, 8)
    p.bc[1] = 9
    with pytest.raises(pkg.NsError):
        pkg.Solver(p)
    p = pkg.make_params(8, 8, 8, sensor=1)  # sensor needs the characteristic FP32 form
    with pytest.raises(pkg.NsError):
        pkg.Solver(p)


def test_no_device_is_reported_not_crashed():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(pkg.NsError) as e:
        pkg.Solver(pkg.make_params(8, 8, 8))
    assert e.value.status == 7


def test_host_buffers_of_the_wrong_shape_or_type_are_refused_on_the_host():
    """Fault injection on the host: the C ABI takes plain pointers, so the binding refuses
    undersized, mistyped or strided host buffers before any call crosses it."""
    shape = pkg.halo_shape(pkg.make_params(8, 6, 4))
    good = np.zeros(shape)
    assert pkg.check_host_array(good, shape) is good
    for bad in (np.zeros(shape[:-1] + (4,)), np.zeros(shape, dtype=np.float32),
                np.zeros((shape[0] - 1,) + shape[1:]), np.zeros(shape)[:, :, ::-1],
                np.zeros(int(np.prod(shape)))):
        with pytest.raises(ValueError):
            pkg.check_host_array(bad, shape)
    ro = np.zeros(shape)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        pkg.check_host_array(ro, shape, writable=True)


def test_host_register_checks_its_arguments_on_the_host():
    L = pkg.load_library()
    assert L.ns_host_register(None, 64) == pkg.abi.NS_ERR_INVALID_ARG
    buf = np.zeros(8)
    assert L.ns_host_register(ctypes.c_void_p(buf.ctypes.data), 0) == pkg.abi.NS_ERR_INVALID_ARG
    assert L.ns_host_unregister(None) == pkg.abi.NS_ERR_INVALID_ARG
    assert "NULL" in L.ns_last_error_string().decode()
