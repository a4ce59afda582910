"""z-slab decomposition of one multiphase domain across ranks.

The reference advances one domain in one process (OpenMP over its cell
sweeps, MaterKit/src/mkFluidsUser.cpp:70); here one multiphase domain is cut
into contiguous runs of z planes, one per rank — one process per GPU under
``torch.distributed``, or several slabs in one process — and the slabs trade
plane-sized runs between the two kernels of every loop.  What crosses a slab
face follows from the in-place (AA) streaming and is listed by the library
(``mk_slab_transfers``): the 5 populations with e_z = -+1 of both D3Q19
lattices before and after every odd loop, and one phi plane per face every
loop.  The library enforces the order of the steps (``mk_slab_next``).

Three pieces:

* :class:`Slab` — one slab handle of the C ABI.
* :class:`TorchTransport` — the exchange between ranks over a
  ``torch.distributed`` process group: with NCCL the runs go straight from and
  into the slab's device arrays, ordered on the slab's own CUDA stream (no host
  synchronisation); with gloo they are staged through host memory.  A run
  whose peer is this rank (a periodic z axis on one rank) is a local copy.
* :class:`SlabRun` — drives one slab through its loops with a transport and
  reduces the diagnostics with one FP64 all-reduce.

``advance_local`` advances the slabs of one process together with the
library's in-process exchange (``mk_slab_exchange_local``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from .solver import Solver, _check

EXCHANGES = (A.MK_SLAB_FILL, A.MK_SLAB_PHI, A.MK_SLAB_RETURN)
RUNS = (A.MK_SLAB_RUN_PHI, A.MK_SLAB_RUN_COLLIDE)

# raw FP64 sums a slab contributes to the global diagnostics
_SUMS = ("mass", "mx", "my", "mz", "phi_sum", "solid", "fluid", "heat", "solute", "n_bad")


def split(nz: int, rank: int, nranks: int) -> tuple[int, int]:
    """(first global plane, planes owned) of `rank` among `nranks` slabs."""
    z0, n = C.c_int32(), C.c_int32()
    _check(A.load().mk_slab_split(int(nz), int(rank), int(nranks), C.byref(z0), C.byref(n)))
    return z0.value, n.value


def plan(params: A.MkParams, rank: int, nranks: int, stage: int) -> list[A.MkSlabXfer]:
    """The transfers of one exchange stage of `rank` (host only, no device)."""
    buf = (A.MkSlabXfer * A.MK_SLAB_MAX_XFER)()
    n = C.c_int32()
    _check(A.load().mk_slab_plan(C.byref(params), int(rank), int(nranks), int(stage), buf, A.MK_SLAB_MAX_XFER,
                                 C.byref(n)))
    return [buf[k] for k in range(n.value)]


class _Cuda:
    """A device run exposed to torch through the CUDA array interface."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class Slab(Solver):
    """The slab of rank `rank` among `nranks` of the multiphase case `params`
    (global sizes), on the current device.  Its arrays hold the owned planes
    plus one ghost plane on each side; :meth:`owned` returns the owned ones."""

    def __init__(self, params: A.MkParams, rank: int, nranks: int):
        self._lib = A.load()
        self._h = C.c_void_p()
        self.global_params = params
        _check(self._lib.mk_create_slab(C.byref(params), int(rank), int(nranks), C.byref(self._h)))
        self.params = A.MkParams()
        _check(self._lib.mk_get_params(self._h, C.byref(self.params)), self._h)
        r, n, z0, nown, nzg = (C.c_int32() for _ in range(5))
        _check(self._lib.mk_slab_info(self._h, C.byref(r), C.byref(n), C.byref(z0), C.byref(nown), C.byref(nzg)),
               self._h)
        self.rank, self.nranks, self.z0, self.nz_own, self.nz_global = r.value, n.value, z0.value, nown.value, nzg.value
        prec = self.params.precision
        self._pop_type = {A.MK_PREC_FP64: "<f8", A.MK_PREC_FP32: "<f4"}.get(prec, "<u2")
        self._phi_type = "<f8" if prec == A.MK_PREC_FP64 else "<f4"

    # -- protocol --------------------------------------------------------------
    def next(self) -> int:
        return int(self._lib.mk_slab_next(self._h))

    def transfers(self, stage: int) -> list[A.MkSlabXfer]:
        buf = (A.MkSlabXfer * A.MK_SLAB_MAX_XFER)()
        n = C.c_int32()
        _check(self._lib.mk_slab_transfers(self._h, int(stage), buf, A.MK_SLAB_MAX_XFER, C.byref(n)), self._h)
        return [buf[k] for k in range(n.value)]

    def done(self, stage: int) -> None:
        _check(self._lib.mk_slab_done(self._h, int(stage)), self._h)

    def run(self, action: int) -> None:
        _check(self._lib.mk_slab_run(self._h, int(action)), self._h)

    def run_tensor(self, x: A.MkSlabXfer):
        """The run of transfer `x` as a torch tensor over the slab's device memory."""
        import torch
        typestr = self._phi_type if x.array == 2 else self._pop_type
        return torch.as_tensor(_Cuda(x.ptr, x.count, typestr), device=f"cuda:{torch.cuda.current_device()}")

    # -- output ----------------------------------------------------------------
    def owned(self, name: str, dtype=np.float64) -> np.ndarray:
        """Field over the owned planes, (nz_own, ny, nx)."""
        return self.field(name, dtype)[1:-1]

    def diag_sums(self) -> tuple[np.ndarray, float]:
        """This slab's share of the global diagnostics: the FP64 sums and the
        largest speed."""
        d = self.diagnostics()
        fluid = float(self.fluid_cells())
        sums = np.array([d["mass"], *d["momentum"], d["phi_sum"], d["solid_frac"] * fluid, fluid, d["heat"],
                         d["solute"], float(d["n_bad"])], dtype=np.float64)
        return sums, float(d["max_speed"])


def combine(sums: np.ndarray, max_speed: float) -> dict:
    """Global diagnostics from the summed slab shares."""
    v = dict(zip(_SUMS, (float(s) for s in sums)))
    return {"mass": v["mass"], "momentum": [v["mx"], v["my"], v["mz"]], "phi_sum": v["phi_sum"],
            "solid_frac": v["solid"] / v["fluid"] if v["fluid"] > 0 else 0.0, "heat": v["heat"],
            "solute": v["solute"], "max_speed": float(max_speed), "n_bad": int(round(v["n_bad"])),
            "fluid_cells": int(round(v["fluid"]))}


def advance_local(slabs: list[Slab], nsteps: int) -> None:
    """Advance the slabs of one decomposition (slabs[r] is rank r) by nsteps
    loops, exchanging through the library's in-process copies."""
    lib = A.load()
    arr = (C.c_void_p * len(slabs))(*[s.handle for s in slabs])
    target = slabs[0].step + int(nsteps)
    while True:
        act = slabs[0].next()
        if act == A.MK_SLAB_RUN_PHI and slabs[0].step == target:
            return
        if act in EXCHANGES:
            _check(lib.mk_slab_exchange_local(arr, len(slabs), act))
        else:
            for s in slabs:
                s.run(act)


class TorchTransport:
    """Slab exchanges over a torch.distributed process group (NCCL or gloo)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.backend = dist.get_backend(group)
        self.rank = dist.get_rank(group)

    def _global(self, peer: int) -> int:
        return peer if self.group is None else self.dist.get_global_rank(self.group, peer)

    def exchange(self, slab, stage: int) -> None:
        """Carry out `stage` for `slab` (every rank calls it with the same stage)."""
        import torch
        xs = slab.transfers(stage)
        # device slabs: every copy and transfer is ordered on the slab's own
        # stream, after its kernels and before its next one
        stream = torch.cuda.ExternalStream(slab.stream()) if isinstance(slab, Slab) else None
        if self.backend != "nccl":
            slab.sync()
        ctx = torch.cuda.stream(stream) if stream is not None else _Null()
        with ctx:
            # local runs first (a periodic axis on one rank)
            sends = {x.tag: x for x in xs if x.send and x.peer == self.rank}
            for x in xs:
                if not x.send and x.peer == self.rank:
                    slab.run_tensor(x).copy_(slab.run_tensor(sends[x.tag]))
            remote = [x for x in xs if x.peer != self.rank]
            if self.backend == "nccl":
                ops = [self.dist.P2POp(self.dist.isend if x.send else self.dist.irecv, slab.run_tensor(x),
                                       self._global(x.peer), self.group) for x in remote]
                if ops:
                    for w in self.dist.batch_isend_irecv(ops):
                        w.wait()  # orders the slab's stream after the transfers
            else:
                works, landing = [], []
                for x in remote:
                    t = slab.run_tensor(x)
                    host = t.to("cpu", copy=True) if x.send else torch.empty(t.shape, dtype=t.dtype)
                    fn = self.dist.isend if x.send else self.dist.irecv
                    works.append(fn(host, self._global(x.peer), group=self.group, tag=int(x.tag)))
                    if not x.send:
                        landing.append((t, host))
                for w in works:
                    w.wait()
                for t, host in landing:
                    t.copy_(host)
        slab.done(stage)


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class SlabRun:
    """One rank's part of a slab-decomposed run."""

    def __init__(self, slab, transport: TorchTransport):
        self.slab = slab
        self.transport = transport

    def advance(self, nsteps: int) -> None:
        target = self.slab.step + int(nsteps)
        while True:
            act = self.slab.next()
            if act == A.MK_SLAB_RUN_PHI and self.slab.step == target:
                return
            if act in EXCHANGES:
                self.transport.exchange(self.slab, act)
            else:
                self.slab.run(act)

    def diagnostics(self) -> dict:
        """Global diagnostics: one FP64 all-reduce of the slab sums (the
        largest speed rides along in this rank's own slot)."""
        import torch
        dist = self.transport.dist
        sums, vmax = self.slab.diag_sums()
        n = dist.get_world_size(self.transport.group)
        buf = np.zeros(len(sums) + n)
        buf[:len(sums)] = sums
        buf[len(sums) + self.transport.rank] = vmax
        dev = "cuda" if self.transport.backend == "nccl" else "cpu"
        t = torch.from_numpy(buf).to(dev)
        dist.all_reduce(t, group=self.transport.group)
        out = t.cpu().numpy()
        return combine(out[:len(sums)], float(out[len(sums):].max()))

    def gather(self, name: str) -> np.ndarray:
        """The global field (nz, ny, nx) assembled from every rank's owned
        planes (on every rank)."""
        import torch
        dist = self.transport.dist
        own = np.ascontiguousarray(self.slab.owned(name))
        n = dist.get_world_size(self.transport.group)
        p = self.slab.global_params
        nmax = -(-p.nz // n)
        pad = np.zeros((nmax, p.ny, p.nx))
        pad[:own.shape[0]] = own
        dev = "cuda" if self.transport.backend == "nccl" else "cpu"
        t = torch.from_numpy(pad).to(dev)
        parts = [torch.empty_like(t) for _ in range(n)]
        dist.all_gather(parts, t, group=self.transport.group)
        out = []
        for r in range(n):
            _, k = split(p.nz, r, n)
            out.append(parts[r].cpu().numpy()[:k])
        return np.concatenate(out, axis=0)
