import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_cases.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def abi():
    return importlib.import_module("3dnssolver_b200.abi")


@pytest.fixture(scope="session")
def wl():
    return importlib.import_module("3dnssolver_b200.workloads")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def load_golden():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta


def interior(a, g=3):
    return a[g:-g, g:-g, g:-g]


def rel_l2(a, b):
    """Relative L2 error of a against b per conserved field (last axis)."""
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    num = np.sqrt(((a - b) ** 2).sum(axis=0))
    den = np.sqrt((b ** 2).sum(axis=0))
    return num / np.maximum(den, 1e-300)


DRIVER = os.path.join(ROOT, "3dnssolver_b200", "lib", "ns_b200_driver")


def driver_xml(case="sod_x", dim=3, n=(8, 6, 4), L=(2.0, 1.0, 0.5), mu=1e-4, Pr=0.72, gamma=1.4,
               end_t=1.0, cfl=0.4, fmt="Binary", interval=2, bc=("Neumann", "Neumann", "Periodic",
               "Periodic", "Periodic", "Periodic"), scheme="Weno", order=5, char=1, weights="Shu",
               riemann="LaxFriedrichs", diff="Centered", diff_order=2, nproc=(1, 1, 1), drop=()):
    """An input.xml in the reference's schema (src/io/reader.cpp); `drop` removes elements."""
    parts = {
        "Geometry": [("Dim", dim), ("Lx", L[0]), ("Ly", L[1]), ("Lz", L[2])],
        "Grid": [("Nx", n[0]), ("Ny", n[1]), ("Nz", n[2])],
        "FluidProperties": [("Mu", mu), ("Pr", Pr), ("Gamma", gamma)],
        "Time": [("EndT", end_t), ("CFLmax", cfl)],
        "OutputProperties": [("FileFormat", fmt), ("OutputInterval", interval)],
        "InitialConditions": [("Case", case)],
        "BoundaryConditions": list(zip(["West", "East", "South", "North", "Front", "Back"], bc)),
    }
    out = ['<?xml version="1.0" ?>', "<Input>"]
    for sec, items in parts.items():
        if sec in drop:
            continue
        out.append(f"  <{sec}>")
        out += [f"    <{k}> {v} </{k}>" for k, v in items if k not in drop]
        out.append(f"  </{sec}>")
    if "NumericalSchemes" not in drop:
        conv = [("Scheme", scheme), ("Order", order), ("CharacteristicSpace", char), ("WeightType", weights),
                ("RiemannSolver", riemann)]
        out.append("  <NumericalSchemes>")
        out.append("    <ConvectionScheme>")
        out += [f"      <{k}> {v} </{k}>" for k, v in conv if k not in drop]
        out.append("    </ConvectionScheme>")
        out.append("    <DiffusionScheme> <Scheme> %s </Scheme> <Order> %d </Order> </DiffusionScheme>"
                   % (diff, diff_order))
        out.append("  </NumericalSchemes>")
    out.append("  <!-- one GPU runs the whole domain -->")
    out.append("  <DomainDecomposition> <NprocX> %d </NprocX> <NprocY> %d </NprocY> <NprocZ> %d </NprocZ>"
               " </DomainDecomposition>" % nproc)
    out.append("</Input>")
    return "\n".join(out) + "\n"


def run_driver(tmp_path, xml, *args, check=False):
    import subprocess
    f = tmp_path / "input.xml"
    f.write_text(xml)
    return subprocess.run([DRIVER, "--input", str(f), *map(str, args)], capture_output=True, text=True,
                          cwd=tmp_path, check=check)
