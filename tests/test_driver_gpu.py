"""The input.xml driver on the GPU: its fields after a few steps against the
oracle advanced from the same initial condition (FP64 1e-12 relative L2, FP32
at FP32 accuracy), its printed dt against the oracle's, and a restart from a
written fields file reproducing the uninterrupted run bit for bit."""
import importlib
import os
import re

import numpy as np
import pytest

from conftest import DRIVER, driver_xml, interior, rel_l2, run_driver

pkg = importlib.import_module("3dnssolver_b200")
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")]

N = pkg.BC_NEUMANN
P = pkg.BC_PERIODIC


def fields(path, n):
    return np.fromfile(path).reshape(n[0], n[1], n[2], 5)


def dts_of(stdout):
    return np.array([float(m) for m in re.findall(r"dt: ([0-9.eE+-]+)", stdout)])


CASES = [
    # case, grid, box, boundary strings, ns bc, char, diffusion order, steps
    ("sod_x", (24, 6, 4), (1.0, 0.25, 0.25), ("Neumann", "Neumann") + ("Periodic",) * 4, (N, P, P), 1, 2, 4),
    ("shear_3d", (12, 10, 8), (1.0, 1.0, 1.0), ("Periodic",) * 6, (P, P, P), 0, 4, 3),
    ("case6", (12, 12, 4), (1.0, 1.0, 1.0), ("Neumann",) * 4 + ("Periodic",) * 2, (N, N, P), 1, 6, 3),
]


@pytest.mark.parametrize("case,n,L,bcs,bc,char,order,steps", CASES, ids=[c[0] for c in CASES])
def test_driver_run_matches_oracle(tmp_path, oracle, case, n, L, bcs, bc, char, order, steps):
    xml = driver_xml(case=case, n=n, L=L, bc=bcs, char=char, diff_order=order, mu=1e-3, end_t=10.0,
                     interval=1000)
    r = run_driver(tmp_path, xml, "--dump-ic", tmp_path / "ic.bin")
    assert r.returncode == 0, r.stderr
    W0 = np.fromfile(tmp_path / "ic.bin").reshape(n[0] + 6, n[1] + 6, n[2] + 6, 5)
    r = run_driver(tmp_path, xml, "--max-steps", steps, "--results", tmp_path / "res")
    assert r.returncode == 0, r.stderr + r.stdout
    Wg = fields(tmp_path / "res" / f"fields_{steps}_p_0.dat", n)
    p = pkg.make_params(*n, L=L, mu=1e-3, Pr=0.72, gamma=1.4, cfl=0.4, convection=2 if char else 1,
                        diffusion_order=order, bc=bc)
    Wo, _, dto = oracle.run(p, W0, steps)
    err = rel_l2(Wg, interior(Wo))
    assert (err[:4] <= 1e-12).all(), err
    np.testing.assert_allclose(dts_of(r.stdout), dto, rtol=1e-5)  # printed with 6 digits
    t, it = open(tmp_path / "res" / f"fields_{steps}_p_0.time").read().split()
    assert int(it) == steps and abs(float(t) - dto.sum()) <= 1e-12 * dto.sum()


def test_driver_fp32_close_to_oracle(tmp_path, oracle):
    n, L = (24, 6, 4), (1.0, 0.25, 0.25)
    bcs = ("Neumann", "Neumann") + ("Periodic",) * 4
    xml = driver_xml(case="sod_x", n=n, L=L, bc=bcs, mu=1e-3, end_t=10.0, interval=1000)
    run_driver(tmp_path, xml, "--dump-ic", tmp_path / "ic.bin", check=True)
    W0 = np.fromfile(tmp_path / "ic.bin").reshape(n[0] + 6, n[1] + 6, n[2] + 6, 5)
    r = run_driver(tmp_path, xml, "--max-steps", 4, "--precision", "fp32", "--results", tmp_path / "res")
    assert r.returncode == 0, r.stderr
    Wg = fields(tmp_path / "res" / "fields_4_p_0.dat", n)
    p = pkg.make_params(*n, L=L, mu=1e-3, Pr=0.72, gamma=1.4, cfl=0.4, convection=2, diffusion_order=2,
                        bc=(N, P, P))
    Wo, _, _ = oracle.run(p, W0, 4)
    err = rel_l2(Wg, interior(Wo))
    assert (err[:2] <= 1e-5).all(), err


def test_restart_reproduces_the_uninterrupted_run(tmp_path):
    n = (16, 8, 8)
    xml = driver_xml(case="shear_3d", n=n, L=(1.0, 1.0, 1.0), bc=("Periodic",) * 6, end_t=10.0, interval=3)
    r = run_driver(tmp_path, xml, "--max-steps", 6, "--results", tmp_path / "a")
    assert r.returncode == 0, r.stderr
    for it in (0, 3, 6):
        assert (tmp_path / "a" / f"fields_{it}_p_0.dat").exists()
    assert (tmp_path / "a" / "mesh_p_0.dat").stat().st_size == n[0] * n[1] * n[2] * 3 * 8
    r = run_driver(tmp_path, xml, "--restart", tmp_path / "a" / "fields_3_p_0.dat", "--max-steps", 3,
                   "--results", tmp_path / "b")
    assert r.returncode == 0, r.stderr
    a = np.fromfile(tmp_path / "a" / "fields_6_p_0.dat")
    b = np.fromfile(tmp_path / "b" / "fields_6_p_0.dat")
    np.testing.assert_array_equal(a.view(np.int64), b.view(np.int64))
    assert open(tmp_path / "a" / "fields_6_p_0.time").read() == open(tmp_path / "b" / "fields_6_p_0.time").read()


def test_runs_to_end_time(tmp_path):
    xml = driver_xml(case="sod_x", n=(32, 4, 4), L=(1.0, 0.25, 0.25),
                     bc=("Neumann", "Neumann") + ("Periodic",) * 4, end_t=0.01, interval=1000)
    r = run_driver(tmp_path, xml, "--results", tmp_path / "res")
    assert r.returncode == 0, r.stderr
    times = [float(m) for m in re.findall(r"Flow time: ([0-9.eE+-]+)", r.stdout)]
    assert times[-1] >= 0.01 and (len(times) == 1 or times[-2] < 0.01)
