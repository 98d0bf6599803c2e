"""Slab decomposition of the domain along x, one slab per rank (one rank per GPU).

The reference splits its domain over MPI ranks in a Cartesian decomposition
(src/decomposition.cpp:116-143), exchanges three ghost planes per face with
MPI_Sendrecv before every stage (src/communicator.cpp:16-143) and reduces dt with
MPI_Allreduce(MIN) (src/time_scheme.cpp:127-136).  Here the domain is split
along x (the slowest device axis, so a side's planes are 5 contiguous runs per
field); every rank's context is created with bc[0] = NS_BC_EXTERNAL and steps
with an exchange callback that

  * packs its outer interior planes (ns_slab_pack), sends them to its x
    neighbours and unpacks theirs into its ghost planes (ns_slab_unpack), and
  * replaces its CFL minimum by the minimum over all ranks.

Transport: torch.distributed point-to-point operations and an all-reduce, on the
device buffers with NCCL (over NVLink/NVSwitch), or host-staged with gloo.  All
device work is ordered on the context's stream, which is torch's current stream
of the rank's device; no kernel waits on another rank.
"""
import ctypes
import importlib

import numpy as np

_pkg = importlib.import_module(__package__)
_abi = importlib.import_module(__package__ + ".abi")

NG = _abi.NS_NGC
INT64_MAX = (1 << 63) - 1
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p)


def split_extent(nx, world):
    """(x0, nx_local) of every rank: nx cells split as evenly as possible, lower ranks first."""
    base, extra = divmod(nx, world)
    out, x0 = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((x0, n))
        x0 += n
    return out


def slab_params(p, rank, world):
    """The parameters of rank's slab of the global parameters p (same dx as the global grid)."""
    x0, n = split_extent(p.nx, world)[rank]
    if n < NG:
        raise ValueError(f"slab of {n} cells along x: every slab needs at least {NG} (one neighbour's ghost planes)")
    q = _abi.NsParams.from_buffer_copy(p)
    q.nx = n
    q.Lx = p.Lx * n / p.nx
    q.slab_x0, q.slab_nx = x0, p.nx
    q.slab_periodic = 1 if p.bc[0] == _abi.BC_PERIODIC else 0
    q.bc[0] = _abi.BC_EXTERNAL
    return q


def split_state(W, p, rank, world):
    """Rank's halo'd host array cut from a global halo'd host array (ghost planes included)."""
    x0, n = split_extent(p.nx, world)[rank]
    return np.ascontiguousarray(W[x0:x0 + n + 2 * NG])


def neighbours(rank, world, periodic):
    lo = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic else None)
    return lo, hi


class HaloExchange:
    """Moves packed ghost planes between x neighbours and reduces the CFL minimum.

    Every rank posts, in this order: send its upper planes up, receive its lower
    ghost planes from below, send its lower planes down, receive its upper ghost
    planes from above.  Transfers between one pair of ranks then match in order
    (NCCL matches point-to-point operations in order; gloo by tag as well), also
    when both neighbours are the same rank (two ranks, periodic)."""

    def __init__(self, rank, world, periodic, group=None, host_staged=False):
        self.rank, self.world = rank, world
        self.lo, self.hi = neighbours(rank, world, periodic)
        self.group = group
        self.host_staged = host_staged

    def exchange(self, send_lo, send_hi, recv_lo, recv_hi):
        """send_lo/send_hi: packed lower/upper interior planes (None where no neighbour);
        recv_lo/recv_hi receive the lower/upper ghost planes."""
        import torch
        import torch.distributed as dist
        if self.lo is not None and self.lo == self.rank:  # one periodic rank: its own planes
            recv_lo.copy_(send_hi)
            recv_hi.copy_(send_lo)
            return
        ops = []
        if self.hi is not None:
            ops.append(dist.P2POp(dist.isend, send_hi, self.hi, self.group, tag=1))
        if self.lo is not None:
            ops.append(dist.P2POp(dist.irecv, recv_lo, self.lo, self.group, tag=1))
        if self.lo is not None:
            ops.append(dist.P2POp(dist.isend, send_lo, self.lo, self.group, tag=2))
        if self.hi is not None:
            ops.append(dist.P2POp(dist.irecv, recv_hi, self.hi, self.group, tag=2))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def min_u64(self, t):
        """In place: the minimum over ranks of a 1-element int64 tensor holding the bits of a
        positive double, or -1 (all ones) for none."""
        import torch
        import torch.distributed as dist
        v = torch.where(t == -1, torch.full_like(t, INT64_MAX), t)
        dist.all_reduce(v, op=dist.ReduceOp.MIN, group=self.group)
        t.copy_(torch.where(v == INT64_MAX, torch.full_like(v, -1), v))


class _DevPtr:
    """A device address as an array for torch.as_tensor (shares the memory)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


class SlabSolver:
    """One rank's slab of a global problem: a Solver on bc[0] = NS_BC_EXTERNAL whose
    steps exchange ghost planes and dt with the other ranks through `exchange`
    (a HaloExchange).  The context and the exchange's torch operations share one
    stream (`stream`, or a new one): the callback's copies and collectives are
    then ordered after the kernels that produce their inputs."""

    def __init__(self, global_params, rank, world, exchange, stream=None):
        import torch
        self.global_params = global_params
        self.rank, self.world = rank, world
        self.params = slab_params(global_params, rank, world)
        self.solver = _pkg.Solver(self.params)
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.solver.set_stream(self.stream.cuda_stream)
        self.ex = exchange
        L = self.solver.lib
        L.ns_set_exchange.argtypes = [ctypes.c_void_p, EXCHANGE_FN, ctypes.c_void_p]
        L.ns_set_exchange.restype = ctypes.c_int
        L.ns_slab_elems.argtypes = [ctypes.c_void_p]
        L.ns_slab_elems.restype = ctypes.c_size_t
        for name in ("ns_slab_pack", "ns_slab_unpack"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            getattr(L, name).restype = ctypes.c_int
        L.ns_slab_dt_slot.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.ns_slab_dt_slot.restype = ctypes.c_int
        self.L = L
        n = int(L.ns_slab_elems(self.solver.h))
        dev = torch.device("cuda", torch.cuda.current_device())
        self.buf = {k: torch.empty(n, dtype=torch.float64, device=dev) for k in ("slo", "shi", "rlo", "rhi")}
        if exchange.host_staged:
            self.hbuf = {k: torch.empty(n, dtype=torch.float64) for k in self.buf}
        self.error = None
        self._cb = EXCHANGE_FN(self._callback)  # kept alive with the solver
        _pkg._check(L.ns_set_exchange(self.solver.h, self._cb, None), "ns_set_exchange")

    # -- the exchange callback (called from inside ns_advance / ns_time_step) --
    def _callback(self, user, ctx, what, stream):
        import torch
        try:
            with torch.cuda.stream(self.stream):
                if what == _abi.EXCHANGE_DT:
                    self._reduce_dt()
                else:
                    self._halo()
            return 0
        except Exception as e:  # reported by the step's status
            self.error = e
            return _abi.NS_ERR_CUDA

    def _reduce_dt(self):
        import torch
        ptr = ctypes.c_void_p()
        _pkg._check(self.L.ns_slab_dt_slot(self.solver.h, ctypes.byref(ptr)), "ns_slab_dt_slot")
        t = torch.as_tensor(_DevPtr(ptr.value, 1, "<i8"), device="cuda")
        if self.ex.host_staged:
            h = t.cpu()
            self.ex.min_u64(h)
            t.copy_(h)
        else:
            self.ex.min_u64(t)

    def _halo(self):
        h, b, ex = self.solver.h, self.buf, self.ex
        if ex.lo is not None:
            _pkg._check(self.L.ns_slab_pack(h, 0, b["slo"].data_ptr()), "ns_slab_pack")
        if ex.hi is not None:
            _pkg._check(self.L.ns_slab_pack(h, 1, b["shi"].data_ptr()), "ns_slab_pack")
        if ex.host_staged:
            hb = self.hbuf
            for k in ("slo", "shi"):
                hb[k].copy_(b[k])
            ex.exchange(hb["slo"], hb["shi"], hb["rlo"], hb["rhi"])
            for k in ("rlo", "rhi"):
                b[k].copy_(hb[k])
        else:
            ex.exchange(b["slo"], b["shi"], b["rlo"], b["rhi"])
        if ex.lo is not None:
            _pkg._check(self.L.ns_slab_unpack(h, 0, b["rlo"].data_ptr()), "ns_slab_unpack")
        if ex.hi is not None:
            _pkg._check(self.L.ns_slab_unpack(h, 1, b["rhi"].data_ptr()), "ns_slab_unpack")

    # -- the Solver surface the slab path needs --
    def upload_primitive(self, W_global_or_local):
        W = W_global_or_local
        if W.shape[0] != self.params.nx + 2 * NG:
            W = split_state(W, self.global_params, self.rank, self.world)
        self.solver.upload_primitive(W)

    def advance(self, n):
        try:
            self.solver.advance(n)
        except _pkg.NsError:
            if self.error is not None:
                raise RuntimeError(f"halo exchange failed on rank {self.rank}") from self.error
            raise

    def download_conservative(self):
        return self.solver.download_conservative()

    def diagnostics(self):
        return self.solver.diagnostics()

    def get_dt(self):
        return self.solver.get_dt()

    def close(self):
        self.solver.close()
