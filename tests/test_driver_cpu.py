"""The input.xml driver (3dnssolver_b200/lib/ns_b200_driver) without a GPU:
reading and checking the reference's input schema (src/io/reader.cpp,
src/params.cpp:3-147), the mapping to ns_params, and the initial conditions
against the reference's own src/testcases.cpp (fixtures in
tests/golden/driver_ic.npz, generated by tests/golden/make_driver_golden.py)."""
import json
import os

import numpy as np
import pytest

from conftest import DRIVER, ROOT, driver_xml, run_driver

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")

IC = os.path.join(ROOT, "tests", "golden", "driver_ic.npz")


def check(tmp_path, **kw):
    r = run_driver(tmp_path, driver_xml(**kw), "--check")
    assert r.returncode == 0, r.stderr + r.stdout
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_params_mapping(tmp_path):
    q = check(tmp_path)
    assert (q["nx"], q["ny"], q["nz"], q["dim"]) == (8, 6, 4, 3)
    assert (q["Lx"], q["Ly"], q["Lz"]) == (2.0, 1.0, 0.5)
    assert q["convection"] == 2 and q["weights"] == 0 and q["diffusion"] == 1
    assert q["bc"] == [1, 0, 0]  # Neumann x, periodic y/z
    assert q["cfl"] == 0.4 and q["end_t"] == 1.0 and q["precision"] == 0
    q = check(tmp_path, char=0, weights="Borges", diff_order=6, bc=("Periodic",) * 6)
    assert q["convection"] == 1 and q["weights"] == 1 and q["diffusion_order"] == 6 and q["bc"] == [0, 0, 0]
    # CenteredConvection and "none" act as no convection; "Shen" and "none" as no diffusion
    # (Driver::create_*_operator, src/driver.cpp:74-105)
    q = check(tmp_path, scheme="Centered", order=2, diff="Shen")
    assert q["convection"] == 0 and q["diffusion"] == 0


@pytest.mark.parametrize("kw,msg", [
    (dict(drop=("Grid",)), "Grid"),
    (dict(drop=("CFLmax",)), "CFLmax"),
    (dict(drop=("RiemannSolver",)), "RiemannSolver"),
    (dict(case="vortex"), "Testcase: vortex is not valid"),
    (dict(scheme="Upwind"), "Convection scheme: Upwind is not valid"),
    (dict(order=3), "Convection scheme order: 3 is not valid"),
    (dict(weights="Mapped"), "Weight type: Mapped is not valid"),
    (dict(diff_order=8), "Diffusion scheme order: 8 is not valid"),
    (dict(fmt="Vtk"), "Output file format: Vtk is not valid"),
    (dict(bc=("Wall",) + ("Periodic",) * 5), "Boundary condition: Wall is not valid"),
])
def test_invalid_input_exits_like_the_reference(tmp_path, kw, msg):
    r = run_driver(tmp_path, driver_xml(**kw), "--check")
    assert r.returncode == 1
    assert msg in r.stdout + r.stderr


@pytest.mark.parametrize("kw,msg", [
    (dict(case="jet"), "sets no initial state"),
    (dict(bc=("Neumann", "Periodic", "Periodic", "Periodic", "Periodic", "Periodic")), "West/East"),
    (dict(riemann="HLLC"), "RiemannSolver HLLC"),
])
def test_inputs_the_reference_cannot_run_are_reported(tmp_path, kw, msg):
    r = run_driver(tmp_path, driver_xml(**kw), "--check")
    assert r.returncode == 1 and msg in r.stderr


def test_malformed_xml_and_command_line(tmp_path):
    r = run_driver(tmp_path, driver_xml().replace("</Grid>", "</Gird>"), "--check")
    assert r.returncode == 1 and "closes" in r.stderr
    r = run_driver(tmp_path, driver_xml(), "--bogus")
    assert r.returncode == 2
    r = run_driver(tmp_path, driver_xml(), "--precision", "fp16")
    assert r.returncode == 2


@pytest.mark.parametrize("case", ["sod_x", "sod_y", "sod_z", "case3", "case4", "case6", "case12", "case15",
                                  "case17", "shear_xy", "shear_3d"])
def test_initial_conditions_match_the_reference_bitwise(tmp_path, case):
    z = np.load(IC)
    nx, ny, nz, Lx, Ly, Lz = z["grid"]
    xml = driver_xml(case=case, n=(int(nx), int(ny), int(nz)), L=(Lx, Ly, Lz))
    r = run_driver(tmp_path, xml, "--dump-ic", tmp_path / "ic.bin")
    assert r.returncode == 0, r.stderr
    w = np.fromfile(tmp_path / "ic.bin")
    ref = z[case].ravel()
    assert w.shape == ref.shape
    np.testing.assert_array_equal(w.view(np.int64), ref.view(np.int64))


def test_restart_file_checks(tmp_path):
    """A checkpoint of the wrong size or without its .time file is refused before any device work."""
    xml = driver_xml(n=(4, 3, 2))
    good = np.zeros(4 * 3 * 2 * 5)
    (tmp_path / "short_p_0.dat").write_bytes(good[:-1].tobytes())
    (tmp_path / "short_p_0.time").write_text("0.5 10\n")
    r = run_driver(tmp_path, xml, "--restart", tmp_path / "short_p_0.dat")
    assert r.returncode == 4 and "fewer than" in r.stderr
    (tmp_path / "long_p_0.dat").write_bytes(np.zeros(good.size + 1).tobytes())
    (tmp_path / "long_p_0.time").write_text("0.5 10\n")
    r = run_driver(tmp_path, xml, "--restart", tmp_path / "long_p_0.dat")
    assert r.returncode == 4 and "more than" in r.stderr
    (tmp_path / "notime_p_0.dat").write_bytes(good.tobytes())
    r = run_driver(tmp_path, xml, "--restart", tmp_path / "notime_p_0.dat")
    assert r.returncode == 4 and ".time" in r.stderr


def test_restart_dump_reproduces_the_checkpoint(tmp_path):
    """--restart with --dump-ic writes the checkpoint's interior into the halo'd layout."""
    n = (4, 3, 2)
    xml = driver_xml(n=n)
    W = np.random.default_rng(3).standard_normal((n[0], n[1], n[2], 5))
    (tmp_path / "f_p_0.dat").write_bytes(W.tobytes())
    (tmp_path / "f_p_0.time").write_text("1.25 7\n")
    r = run_driver(tmp_path, xml, "--restart", tmp_path / "f_p_0.dat", "--dump-ic", tmp_path / "w.bin")
    assert r.returncode == 0, r.stderr
    full = np.fromfile(tmp_path / "w.bin").reshape(n[0] + 6, n[1] + 6, n[2] + 6, 5)
    np.testing.assert_array_equal(full[3:-3, 3:-3, 3:-3], W)
    assert not full[:3].any() and not full[-3:].any()
