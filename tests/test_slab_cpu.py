"""Slab decomposition along x on CPU ranks (gloo, no GPU): every rank advances its
slab with the oracle's slab mode, and the ghost planes and the dt minimum travel
through 3dnssolver_b200.slab.HaloExchange, the transport the GPU ranks use.  The
slabs put together must equal the single-domain oracle bit for bit: the exchange
brings in exactly the cells the single domain reads (communicator.cpp:16-57 and
the MPI_Allreduce(MIN) of time_scheme.cpp:127-136 on a 1-D decomposition)."""
import importlib
import os
import socket
import struct
import sys

import numpy as np
import pytest

from conftest import ROOT

pkg = importlib.import_module("3dnssolver_b200")
wl = importlib.import_module("3dnssolver_b200.workloads")
slab = importlib.import_module("3dnssolver_b200.slab")
P, N = pkg.BC_PERIODIC, pkg.BC_NEUMANN


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pack(U, side, nx):
    """[q][layer][j][k] of the three outer interior planes of a side (halo'd AoS input)."""
    planes = U[3:6] if side == 0 else U[nx:nx + 3]
    return np.ascontiguousarray(np.moveaxis(planes[:, 3:-3, 3:-3, :], -1, 0)).reshape(-1)


def _unpack(U, side, nx, buf, shape):
    planes = np.moveaxis(buf.reshape(5, 3, shape[1] - 6, shape[2] - 6), 0, -1)
    if side == 0:
        U[0:3, 3:-3, 3:-3, :] = planes
    else:
        U[nx + 3:nx + 6, 3:-3, 3:-3, :] = planes


def _worker(rank, world, port, pbytes, W_global, nsteps, outdir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = pkg.NsParams.from_buffer_copy(pbytes)
        q = slab.slab_params(p, rank, world)
        W = slab.split_state(W_global, p, rank, world)
        ex = slab.HaloExchange(rank, world, periodic=p.bc[0] == P)
        nx = q.nx

        def exchange(what, data):
            if what == 0:
                bits = struct.unpack("<q", struct.pack("<d", float(data[0])))[0]
                t = torch.tensor([bits], dtype=torch.int64)
                ex.min_u64(t)
                data[0] = struct.unpack("<d", struct.pack("<q", int(t.item())))[0]
                return
            n = 15 * q.ny * q.nz
            slo = torch.from_numpy(_pack(data, 0, nx)) if ex.lo is not None else None
            shi = torch.from_numpy(_pack(data, 1, nx)) if ex.hi is not None else None
            rlo, rhi = torch.zeros(n, dtype=torch.float64), torch.zeros(n, dtype=torch.float64)
            ex.exchange(slo, shi, rlo, rhi)
            if ex.lo is not None:
                _unpack(data, 0, nx, rlo.numpy(), data.shape)
            if ex.hi is not None:
                _unpack(data, 1, nx, rhi.numpy(), data.shape)

        Wn, Un, dts = O.slab_run(q, W, nsteps, exchange)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), W=Wn[3:-3, 3:-3, 3:-3], U=Un[3:-3, 3:-3, 3:-3], dt=dts)
    finally:
        dist.destroy_process_group()


CASES = [
    # (shape, world, bc, conv, order, weights, semantics)
    ((20, 10, 8), 2, (P, P, P), 2, 4, 0, pkg.SEM_REFERENCE),
    ((21, 8, 6), 3, (N, P, N), 2, 2, 0, pkg.SEM_REFERENCE),
    ((18, 9, 7), 2, (N, N, P), 1, 6, 1, pkg.SEM_REFERENCE),
    ((16, 8, 8), 2, (P, N, P), 2, 2, 0, pkg.SEM_PHYSICAL),
    ((19, 8, 6), 3, (N, P, P), 1, 4, 0, pkg.SEM_PHYSICAL),
    ((12, 7, 6), 1, (P, P, P), 2, 2, 0, pkg.SEM_REFERENCE),
]


@pytest.mark.parametrize("shape,world,bc,conv,order,weights,sem", CASES)
def test_slabs_equal_the_single_domain(oracle, tmp_path, shape, world, bc, conv, order, weights, sem):
    import torch.multiprocessing as mp
    p = pkg.make_params(*shape, convection=conv, diffusion_order=order, weights=weights, bc=bc, mu=0.02,
                        cfl=0.3, L=(1.0, 0.9, 0.8), semantics=sem)
    W0 = wl.random_field(p, seed=sum(shape) + world, smooth=False)
    nsteps = 3
    Wo, Uo, dto = oracle.run(p, W0, nsteps)
    mp.start_processes(_worker, args=(world, _free_port(), bytes(p), W0, nsteps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    W = np.concatenate([z["W"] for z in parts])
    U = np.concatenate([z["U"] for z in parts])
    for z in parts:
        np.testing.assert_array_equal(z["dt"], dto)  # the reduced dt is the global one
    np.testing.assert_array_equal(U, Uo[3:-3, 3:-3, 3:-3])
    np.testing.assert_array_equal(W, Wo[3:-3, 3:-3, 3:-3])


def test_split_extent_and_slab_params():
    assert slab.split_extent(10, 3) == [(0, 4), (4, 3), (7, 3)]
    p = pkg.make_params(12, 8, 8, L=(3.0, 1.0, 1.0), bc=(N, P, P))
    q = slab.slab_params(p, 1, 2)
    assert (q.nx, q.slab_x0, q.slab_nx, q.slab_periodic, q.bc[0]) == (6, 6, 12, 0, pkg.abi.BC_EXTERNAL)
    assert q.Lx / q.nx == p.Lx / p.nx
    with pytest.raises(ValueError):
        slab.slab_params(pkg.make_params(5, 8, 8), 1, 2)  # 3 and 2 cells: 2 is below three ghost planes
    assert slab.neighbours(0, 3, True) == (2, 1) and slab.neighbours(0, 3, False) == (None, 1)
    assert slab.neighbours(2, 3, False) == (1, None)
