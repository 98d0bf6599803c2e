"""Slab decomposition on the GPU path: the domain split along x over ranks, each
rank a process with its own context (bc[0] = NS_BC_EXTERNAL) that steps with the
exchange callback of 3dnssolver_b200.slab.  This run has one GPU, so the ranks
share it and exchange host-staged ghost planes over gloo; the exchange callback
only enqueues copies and host-side transfers (no kernel waits on another rank).
NCCL on device buffers is the same callback with host_staged=False.

The slabs put together must equal the single-domain GPU run (same kernels, same
cells read; rounding-level at most) and the oracle at the FP64 parity bar."""
import importlib
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_l2

pkg = importlib.import_module("3dnssolver_b200")
wl = importlib.import_module("3dnssolver_b200.workloads")
slab = importlib.import_module("3dnssolver_b200.slab")

pytestmark = pytest.mark.gpu
P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, pbytes, W_global, nsteps, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = pkg.NsParams.from_buffer_copy(pbytes)
        ex = slab.HaloExchange(rank, world, periodic=p.bc[0] == P, host_staged=True)
        s = slab.SlabSolver(p, rank, world, ex)
        s.upload_primitive(W_global)
        s.advance(nsteps)
        U = s.download_conservative()
        dt, t = s.get_dt()
        s.close()
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), U=U[3:-3, 3:-3, 3:-3], dt=dt, t=t)
    finally:
        dist.destroy_process_group()


CASES = [
    # (shape, world, bc, conv, order, precision, semantics)
    ((24, 10, 12), 2, (P, P, P), 2, 2, pkg.PREC_FP64, pkg.SEM_REFERENCE),
    ((27, 8, 10), 3, (N, P, N), 2, 4, pkg.PREC_FP64, pkg.SEM_REFERENCE),
    ((20, 12, 8), 2, (N, N, P), 1, 6, pkg.PREC_FP64, pkg.SEM_PHYSICAL),
    # the TMA-staged y/z faces and CD-2 viscous march on slabs with exchanged and Neumann x ends
    ((26, 9, 35), 2, (N, N, P), 2, 2, pkg.PREC_FP64, pkg.SEM_PHYSICAL),
    ((40, 10, 12), 2, (P, P, N), 2, 2, pkg.PREC_FP32, pkg.SEM_REFERENCE),
    ((33, 9, 8), 3, (N, P, P), 2, 4, pkg.PREC_FP32, pkg.SEM_PHYSICAL),
    ((24, 8, 8), 2, (P, P, P), pkg.CONV_NONE, 2, pkg.PREC_FP64, pkg.SEM_REFERENCE),
]


@pytest.mark.parametrize("shape,world,bc,conv,order,prec,sem", CASES)
def test_gpu_slabs_equal_the_single_domain(oracle, tmp_path, shape, world, bc, conv, order, prec, sem):
    import torch.multiprocessing as mp
    p = pkg.make_params(*shape, convection=conv, diffusion_order=order, bc=bc, mu=0.02, cfl=0.3,
                        L=(1.2, 0.9, 0.8), precision=prec, semantics=sem)
    W0 = wl.random_field(p, seed=sum(shape) + 7 * world, smooth=False)
    nsteps = 4
    with pkg.Solver(p) as s:
        s.upload_primitive(W0)
        s.advance(nsteps)
        Ug = s.download_conservative()[3:-3, 3:-3, 3:-3]
        dtg, tg = s.get_dt()
    mp.start_processes(_worker, args=(world, _free_port(), bytes(p), W0, nsteps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    U = np.concatenate([z["U"] for z in parts])
    for z in parts:
        assert float(z["dt"]) == pytest.approx(dtg, rel=1e-14)
        assert float(z["t"]) == pytest.approx(tg, rel=1e-14)
    err = rel_l2(U, Ug)
    assert (err <= 1e-13).all(), f"slabs vs single domain: rel L2 per field {err}"
    if prec == pkg.PREC_FP64:
        Wo, Uo, dto = oracle.run(p, W0, nsteps)
        err = rel_l2(U, Uo[3:-3, 3:-3, 3:-3])
        assert (err[:4] <= 1e-12).all(), f"slabs vs oracle: rel L2 per field {err}"


def _nccl_single_rank(rank, port, pbytes, W_global, nsteps, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        p = pkg.NsParams.from_buffer_copy(pbytes)
        s = slab.SlabSolver(p, 0, 1, slab.HaloExchange(0, 1, periodic=True, host_staged=False))
        s.upload_primitive(W_global)
        s.advance(nsteps)
        U = s.download_conservative()
        s.close()
        np.save(os.path.join(outdir, "U.npy"), U[3:-3, 3:-3, 3:-3])
    finally:
        dist.destroy_process_group()


def test_device_transport_one_periodic_rank_over_nccl(tmp_path):
    """The device-buffer transport (host_staged=False: NCCL all-reduce of the dt slot
    through its device address, ghost planes copied on the device) on one periodic
    rank, whose ghost planes are its own: equal to the single-domain run."""
    import torch.multiprocessing as mp
    p = pkg.make_params(16, 12, 10, convection=2, diffusion_order=2, bc=(P, N, P), mu=0.02, cfl=0.3)
    W0 = wl.random_field(p, seed=71, smooth=False)
    with pkg.Solver(p) as s:
        s.upload_primitive(W0)
        s.advance(3)
        Ug = s.download_conservative()[3:-3, 3:-3, 3:-3]
    mp.start_processes(_nccl_single_rank, args=(_free_port(), bytes(p), W0, 3, str(tmp_path)), nprocs=1,
                       join=True, start_method="spawn")
    err = rel_l2(np.load(tmp_path / "U.npy"), Ug)
    assert (err <= 1e-13).all(), err
