"""A single domain decomposed into x slabs, one per rank.

Replaces the multi-GPU library's decomposition
(ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU/mpi.cu:104-276: sendrecv_U of
3 ghost layers by host-staged MPI_Sendrecv; resistiveMHD2D.cu:550,574:
MPI_Allreduce of dt and of the crash flag) for the single-GPU library's step,
over the C ABI's slab entry points (include/rmhd2d.h, rmhd2d_create_slab).

Each slab owns a contiguous range of the interior columns i (x; columns are
contiguous in the state planes, so a halo is 3 rows of memory per field) and
carries 3 halo columns on each side that borders another slab.  A step is the
library's stage kernels and ghost fill on every slab with halo exchanges in
between (``SlabDomain.step``), and the CFL maximum, cell 0's NaN test and the
crash flag combined across slabs with one max-reduction of three int64 words
per step.  The result is bit for bit the whole-domain solver's.

Two ways to connect the slabs:

* ``SlabDomain`` -- one slab per rank of a torch.distributed process group:
  halo columns move by point-to-point send/recv (NCCL over NVLink between
  GPUs; gloo on CPU hosts), the words by an all-reduce (MAX).
* ``SlabGroup`` -- several slabs in one process (on one device), exchanged
  by copies: the same algorithm without a process group.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .solver import Solver

SLAB_LO, SLAB_HI, SLAB_ORIGIN = 1, 2, 4
GHOST = 3


def partition(n_interior: int, parts: int) -> list[tuple[int, int]]:
    """(first interior column, count) of each slab: as even as possible, the
    first n_interior % parts slabs one column wider.  Every slab owns at
    least 6 columns, the smallest interior a solver accepts."""
    if parts < 1 or n_interior < 6 * parts:
        raise ValueError(f"{n_interior} interior columns cannot give {parts} slabs of at least 6 columns")
    base, extra = divmod(n_interior, parts)
    out, start = [], 0
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        out.append((start, n))
        start += n
    return out


class _Slab:
    """One slab's solver, its part of the domain and its exchange buffers.
    ``torch_device`` is where the buffers live (the GPU of the solver, or the
    CPU for a host build of the library)."""

    def __init__(self, setup, index: int, parts: int, *, precision: str, device: int, torch_device, stream=None):
        import torch

        self.setup = setup
        self.index, self.parts = index, parts
        x0, n = partition(setup.nx - 2 * GHOST, parts)[index]
        self.x0, self.n = x0, n
        periodic = setup.bc == "periodic"
        self.lo_halo = periodic or index > 0
        self.hi_halo = periodic or index < parts - 1
        sides = (SLAB_LO if self.lo_halo else 0) | (SLAB_HI if self.hi_halo else 0) | (SLAB_ORIGIN if index == 0 else 0)
        lib = _lib.load()
        cfg = Solver.make_config(n + 2 * GHOST, setup.ny, setup.dx, setup.dy, gamma=setup.gamma, cfl=setup.cfl,
                                 eps=setup.eps, eta=setup.eta, bc=setup.bc, bc_y=setup.bc_y, precision=precision,
                                 device=device)
        cfg.stream = stream
        h = ctypes.c_void_p()
        _lib.check(lib.rmhd2d_create_slab(ctypes.byref(cfg), sides, ctypes.byref(h)), None)
        self.solver = Solver._member(h, n + 2 * GHOST, setup.ny)
        self.solver._owned = True
        self._lib = lib
        nd = ctypes.c_longlong()
        self._ck(lib.rmhd2d_slab_halo_doubles(h, ctypes.byref(nd)))
        mk = lambda: torch.empty(nd.value, dtype=torch.float64, device=torch_device)  # noqa: E731
        self.send = [mk(), mk()]     # [low side, high side]
        self.recv = [mk(), mk()]
        self.words = torch.zeros(3, dtype=torch.int64, device=torch_device)
        cols = slice(x0, x0 + n + 2 * GHOST)   # columns of the whole array this slab's array covers
        if setup.eta_table is not None:
            self.solver.set_eta_table(setup.eta_table[cols])
        self.solver.set_state(setup.state[cols], apply_boundary=False)

    @property
    def h(self):
        return self.solver._h

    def _ck(self, st: int) -> None:
        _lib.check(st, self.h)

    def pack(self, state: int) -> None:
        for side, on in ((0, self.lo_halo), (1, self.hi_halo)):
            if on:
                self._ck(self._lib.rmhd2d_slab_pack(self.h, state, side, ctypes.c_void_p(self.send[side].data_ptr())))

    def unpack(self, state: int) -> None:
        for side, on in ((0, self.lo_halo), (1, self.hi_halo)):
            if on:
                self._ck(self._lib.rmhd2d_slab_unpack(self.h, state, side,
                                                      ctypes.c_void_p(self.recv[side].data_ptr())))

    def stage(self, k: int) -> None:
        self._ck(self._lib.rmhd2d_slab_stage(self.h, k))

    def fill(self, which: int) -> None:
        self._ck(self._lib.rmhd2d_slab_fill(self.h, which))

    def refresh_rate(self) -> None:
        self._ck(self._lib.rmhd2d_slab_refresh_rate(self.h))

    def get_words(self) -> None:
        self._ck(self._lib.rmhd2d_slab_get_words(self.h, ctypes.c_void_p(self.words.data_ptr())))

    def set_words(self) -> None:
        self._ck(self._lib.rmhd2d_slab_set_words(self.h, ctypes.c_void_p(self.words.data_ptr())))

    def close(self) -> None:
        self.solver.close()


class _OnStream:
    """The slabs' stream as torch's current stream (a no-op on the CPU):
    the library's kernels, the exchange copies, send/recv and the
    all-reduce are then ordered by one stream."""

    def __init__(self, torch_device):
        import torch

        self.stream = torch.cuda.Stream(device=torch_device) if torch_device.type == "cuda" else None
        self.handle = self.stream.cuda_stream if self.stream is not None else None

    def __enter__(self):
        import torch

        if self.stream is not None:
            self._ctx = torch.cuda.stream(self.stream)
            self._ctx.__enter__()
        return self

    def __exit__(self, *exc):
        if self.stream is not None:
            self._ctx.__exit__(*exc)


def _step(slabs, exchange, combine) -> None:
    """One RK2 step of all slabs (include/rmhd2d.h gives the order)."""
    for s in slabs:
        s.stage(1)
    exchange(1)
    for s in slabs:
        s.fill(1)
    exchange(1)
    for s in slabs:
        s.stage(2)
    exchange(0)
    for s in slabs:
        s.fill(2)
    exchange(0)
    combine()


def _start(slabs, exchange, combine) -> None:
    """Ghost fill and CFL reduction of the initial state (the reference's
    initializeU ends with the boundary)."""
    exchange(0)
    for s in slabs:
        s.fill(0)
    exchange(0)
    for s in slabs:
        s.refresh_rate()
    combine()


class SlabDomain:
    """This rank's slab of ``setup``'s domain, decomposed over the ranks of
    a torch.distributed process group (``group``; default the world).

    ``device`` is the CUDA ordinal of the solver; ``torch_device`` the torch
    device of the exchange buffers (``cuda:<device>``, or ``cpu`` for a host
    build of the library).  On a GPU the slab's kernels, its exchange buffers'
    copies, the send/recv and the all-reduce all run on one stream of the
    slab's own."""

    def __init__(self, setup, *, precision: str = "fp64_exact", device: int = 0, torch_device=None, group=None):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if torch_device is None:
            torch_device = torch.device("cuda", device)
        torch_device = torch.device(torch_device)
        self._on = _OnStream(torch_device)
        with self._on:
            self.slab = _Slab(setup, self.rank, self.world, precision=precision, device=device,
                              torch_device=torch_device, stream=self._on.handle)
            _start([self.slab], self._exchange, self._combine)

    def _peer(self, r: int) -> int:
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def _exchange(self, state: int) -> None:
        s = self.slab
        s.pack(state)
        left, right = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        if self.world == 1:
            # periodic x on one slab: each halo is the slab's own far edge
            s.recv[0].copy_(s.send[1])
            s.recv[1].copy_(s.send[0])
        else:
            # sends in the order (low, high), receives in the order (high,
            # low): with two ranks on a periodic domain both messages of a
            # pair run between the same two ranks and are matched in order
            P2P = self.dist.P2POp
            ops = []
            if s.lo_halo:
                ops.append(P2P(self.dist.isend, s.send[0], self._peer(left), self.group, tag=1))
            if s.hi_halo:
                ops.append(P2P(self.dist.isend, s.send[1], self._peer(right), self.group, tag=2))
            if s.hi_halo:
                ops.append(P2P(self.dist.irecv, s.recv[1], self._peer(right), self.group, tag=1))
            if s.lo_halo:
                ops.append(P2P(self.dist.irecv, s.recv[0], self._peer(left), self.group, tag=2))
            if ops:
                for req in self.dist.batch_isend_irecv(ops):
                    req.wait()
        s.unpack(state)

    def _combine(self) -> None:
        s = self.slab
        s.get_words()
        self.dist.all_reduce(s.words, op=self.dist.ReduceOp.MAX, group=self.group)
        s.set_words()

    def step(self) -> None:
        with self._on:
            _step([self.slab], self._exchange, self._combine)

    def run(self, nsteps: int) -> None:
        for _ in range(int(nsteps)):
            self.step()

    @property
    def columns(self) -> tuple[int, int]:
        """(first, count) of the interior columns this slab owns."""
        return self.slab.x0, self.slab.n

    def get_state(self) -> np.ndarray:
        """This slab's array: its own columns with 3 columns on each side."""
        return self.slab.solver.get_state()

    @property
    def dt(self) -> float:
        return self.slab.solver.dt

    @property
    def total_time(self) -> float:
        return self.slab.solver.total_time

    def check_crashed(self) -> bool:
        return self.slab.solver.check_crashed()

    def close(self) -> None:
        self.slab.close()


class SlabGroup:
    """``parts`` slabs of ``setup``'s domain in this process, on one device,
    exchanged by device copies: the decomposition without a process group."""

    def __init__(self, setup, parts: int, *, precision: str = "fp64_exact", device: int = 0, torch_device=None):
        import torch

        if torch_device is None:
            torch_device = torch.device("cuda", device)
        torch_device = torch.device(torch_device)
        self._on = _OnStream(torch_device)
        self.setup = setup
        with self._on:
            self.slabs = [_Slab(setup, r, parts, precision=precision, device=device, torch_device=torch_device,
                                stream=self._on.handle) for r in range(parts)]
            _start(self.slabs, self._exchange, self._combine)

    def _exchange(self, state: int) -> None:
        n = len(self.slabs)
        for s in self.slabs:
            s.pack(state)
        for r, s in enumerate(self.slabs):
            if s.lo_halo:
                s.recv[0].copy_(self.slabs[(r - 1) % n].send[1])
            if s.hi_halo:
                s.recv[1].copy_(self.slabs[(r + 1) % n].send[0])
        for s in self.slabs:
            s.unpack(state)

    def _combine(self) -> None:
        for s in self.slabs:
            s.get_words()
        w = self.slabs[0].words.clone()
        for s in self.slabs[1:]:
            w = w.maximum(s.words)
        for s in self.slabs:
            s.words.copy_(w)
            s.set_words()

    def step(self) -> None:
        with self._on:
            _step(self.slabs, self._exchange, self._combine)

    def run(self, nsteps: int) -> None:
        for _ in range(int(nsteps)):
            self.step()

    def get_state(self) -> np.ndarray:
        """The whole domain's array assembled from the slabs: each slab's own
        columns, and the domain's x-wall ghost columns from the edge slabs
        (with periodic x they are the halos of the first and last slab)."""
        out = np.empty_like(self.setup.state)
        for k, s in enumerate(self.slabs):
            a = s.solver.get_state()
            out[GHOST + s.x0:GHOST + s.x0 + s.n] = a[GHOST:GHOST + s.n]
            if k == 0:
                out[:GHOST] = a[:GHOST]
            if k == len(self.slabs) - 1:
                out[-GHOST:] = a[-GHOST:]
        return out

    @property
    def dt(self) -> float:
        return self.slabs[0].solver.dt

    @property
    def total_time(self) -> float:
        return self.slabs[0].solver.total_time

    def check_crashed(self) -> bool:
        return any(s.solver.check_crashed() for s in self.slabs)

    def close(self) -> None:
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
