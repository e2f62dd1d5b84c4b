"""x-slab decomposition of one flowfield over ranks.

Replaces the reference's MPI layer for the step: Flowfield::Mpi_Boundary
(src/Flowfield.cpp:775-1083: two planes of the primitives per x face, sent to
the neighbours after the physical boundary fill) and the MPI_Reduce/MPI_Bcast
of dt in Flowfield::CFLcondition (:242-272).  One slab per rank, one rank per
GPU; the halo buffers are device memory packed and unpacked by the library
(eu3d_halo_pack / eu3d_halo_unpack) and moved by NCCL send/recv over NVLink
through torch.distributed; dt is an in-place all-reduce MIN of the device
scalar.  Every rank takes the same collective steps in the same order.

A step of one slab, as `eu3d_step` does it on a single rank:

    CFL: local dt -> all-reduce MIN -> time += dt
    boundary fill -> halo exchange [-> wedge band -> halo exchange]
    stage 1 (advection; SSP-RK: + stage-1 update and decode)
    SSP-RK2/RK3: boundary fill -> halo exchange [...] -> stage 2
    SSP-RK3: boundary fill -> halo exchange [...] -> stage 3
    chemistry

With an immersed wedge the band is filled again after the first exchange (its
mirror sources near a slab face are the neighbour's cells) and a second
exchange hands the refilled solid cells to the neighbours.

Layouts: "partition" gives every interior cell to one rank; "reference"
reproduces the reference's mesh blocks (src/Mesh.cpp:77-93), where
neighbouring slabs share their end node and the exchange skips it.

`SlabRun` drives the slabs this process holds through a step in lockstep;
a transport carries out the collective points: `TorchTransport` (one slab per
process, torch.distributed: NCCL for device buffers, gloo for host ones) or
`LoopbackTransport` (all slabs in this process).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import gpu
from .readers import Grid


def slab_extents(total_ni: int, nranks: int, layout: str = "partition"):
    """[(i0, n)] per rank: the first interior cell (global interior index) and
    the count of interior cells of each slab."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    if layout == "partition":
        base, extra = divmod(total_ni, nranks)
        out, i0 = [], 0
        for r in range(nranks):
            n = base + (1 if r < extra else 0)
            out.append((i0, n))
            i0 += n
    elif layout == "reference":
        # src/Mesh.cpp:77-93: (total - 1) / blocks + 1 nodes, the last one shared
        n = (total_ni - 1) // nranks + 1
        out = [(r * (n - 1), n) for r in range(nranks)]
        if out[-1][0] + n != total_ni:
            raise ValueError("the reference layout needs total_ni - 1 divisible by the rank count")
    else:
        raise ValueError(f"unknown layout {layout!r}")
    if any(n < 3 for _, n in out):
        raise ValueError("every slab needs at least 3 interior cells")
    return out


def slab_grid(grid: Grid, i0: int, n: int) -> Grid:
    """The slab's grid: interior cells i0 .. i0+n-1 of `grid` with their ghost nodes."""
    return dataclasses.replace(grid, ni=n, xnode=np.array(grid.xnode[i0:i0 + n + 2 * grid.bc], dtype=np.float64))


@dataclasses.dataclass
class StepSpec:
    react: int = gpu.REACT_IMEX
    type_: int = 0
    timeadv: int = gpu.ADV_EE
    diff: int = gpu.DIFF_MUSCL2
    bc_kind: int = gpu.BC_RSBI
    cfl: float = 0.0
    final_time: float = 1.0

    def kw(self) -> dict:
        return dataclasses.asdict(self)


class Slab:
    """One rank's slab.  Subclasses supply the operations on the state."""

    def __init__(self, rank: int, nranks: int, overlap: int, wedge: bool):
        self.rank, self.nranks, self.overlap, self.wedge = rank, nranks, overlap, wedge

    def sides(self):
        """Faces with a neighbour: 0 (low x) and/or 1 (high x)."""
        out = []
        if self.rank > 0:
            out.append(0)
        if self.rank < self.nranks - 1:
            out.append(1)
        return out

    def neighbour(self, side: int) -> int:
        return self.rank - 1 if side == 0 else self.rank + 1

    # the operations (subclasses)
    def cfl_local(self, cfl, final_time): raise NotImplementedError
    def dt_buffer(self): raise NotImplementedError
    def advance_time(self): raise NotImplementedError
    def boundary(self, kind): raise NotImplementedError
    def wedge_fill(self): raise NotImplementedError
    def pack(self, side): raise NotImplementedError
    def recv_buffer(self, side): raise NotImplementedError
    def unpack(self, side): raise NotImplementedError
    def part(self, part, spec: StepSpec): raise NotImplementedError

    def step(self, spec: StepSpec):
        """One step as a generator; it yields at the collective points."""
        if spec.cfl != 0:
            self.cfl_local(spec.cfl, spec.final_time)
            yield "min"
            self.advance_time()
        yield from self._fill(spec.bc_kind)
        self.part(gpu.PART_STAGE1, spec)
        if spec.timeadv in (gpu.ADV_SSPRK2, gpu.ADV_SSPRK3):
            yield from self._fill(spec.bc_kind)
            self.part(gpu.PART_STAGE2, spec)
        if spec.timeadv == gpu.ADV_SSPRK3:
            yield from self._fill(spec.bc_kind)
            self.part(gpu.PART_STAGE3, spec)
        self.part(gpu.PART_REACT, spec)

    def _fill(self, kind):
        self.boundary(kind)
        yield "halo"
        if self.wedge:
            self.wedge_fill()
            yield "halo"


class _CudaArray:
    """A device pointer as a one-element FP64 CUDA array (zero-copy view for torch)."""

    def __init__(self, ptr: int):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<f8", "data": (ptr, False), "version": 3}


class DeviceSlab(Slab):
    """A slab on this process's GPU: a gpu.DeviceFlowfield over slab_grid().
    Halo buffers are torch CUDA tensors; collectives run on the handle's stream."""

    def __init__(self, dev: gpu.DeviceFlowfield, rank: int, nranks: int, overlap: int = 0, wedge: bool = False):
        super().__init__(rank, nranks, overlap, wedge)
        import torch
        self.torch = torch
        self.d = dev
        nb = dev.halo_bytes()
        self._send = {s: torch.empty(nb, dtype=torch.uint8, device=f"cuda:{dev.device}") for s in (0, 1)}
        self._recv = {s: torch.empty(nb, dtype=torch.uint8, device=f"cuda:{dev.device}") for s in (0, 1)}
        self._dt = torch.as_tensor(_CudaArray(dev.dt_device_ptr), device=f"cuda:{dev.device}")
        self.stream = torch.cuda.ExternalStream(dev.stream, device=f"cuda:{dev.device}")

    def cfl_local(self, cfl, final_time):
        self.d.cfl_local(cfl, final_time)

    def dt_buffer(self):
        return self._dt

    def advance_time(self):
        self.d.advance_time()

    def boundary(self, kind):
        self.d.boundary(kind)

    def wedge_fill(self):
        self.d.wedge_fill()

    def pack(self, side):
        self.d.halo_pack(side, self._send[side].data_ptr(), self.overlap)
        return self._send[side]

    def recv_buffer(self, side):
        return self._recv[side]

    def unpack(self, side):
        self.d.halo_unpack(side, self._recv[side].data_ptr())

    def part(self, part, spec):
        self.d.step_part(part, **spec.kw())


class LoopbackTransport:
    """All ranks' slabs live in this process (tests, one GPU): buffers are
    copied directly, dt is the minimum over the slabs."""

    def _sync(self, slabs):
        for s in slabs:
            if isinstance(s, DeviceSlab):
                s.torch.cuda.synchronize(s.d.device)

    def min(self, slabs):
        self._sync(slabs)
        bufs = [s.dt_buffer() for s in slabs]
        m = min(float(b[0]) for b in bufs)
        for b in bufs:
            b.fill_(m)
        self._sync(slabs)

    def halo(self, slabs):
        sent = {(s.rank, side): s.pack(side) for s in slabs for side in s.sides()}
        self._sync(slabs)
        for s in slabs:
            for side in s.sides():
                # my low face receives the left neighbour's high-side planes and vice versa
                src = sent[(s.neighbour(side), 1 - side)]
                s.recv_buffer(side).copy_(src)
        self._sync(slabs)
        for s in slabs:
            for side in s.sides():
                s.unpack(side)


class TorchTransport:
    """One slab per process; torch.distributed carries the collectives (NCCL for
    CUDA buffers on the slab's stream, gloo for host buffers)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def _ctx(self, slab):
        if isinstance(slab, DeviceSlab):
            return slab.torch.cuda.stream(slab.stream)
        import contextlib
        return contextlib.nullcontext()

    def min(self, slabs):
        (s,) = slabs
        with self._ctx(s):
            self.dist.all_reduce(s.dt_buffer(), op=self.dist.ReduceOp.MIN, group=self.group)

    def halo(self, slabs):
        (s,) = slabs
        dist = self.dist
        with self._ctx(s):
            ops = []
            for side in s.sides():
                peer = s.neighbour(side)
                ops.append(dist.P2POp(dist.isend, s.pack(side), peer, group=self.group))
                ops.append(dist.P2POp(dist.irecv, s.recv_buffer(side), peer, group=self.group))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
            for side in s.sides():
                s.unpack(side)


class SlabRun:
    """Steps the slabs this process holds, in lockstep, through a transport."""

    def __init__(self, slabs, transport):
        self.slabs = list(slabs)
        self.transport = transport

    def step(self, spec: StepSpec):
        gens = [s.step(spec) for s in self.slabs]
        while True:
            reqs = [next(g, None) for g in gens]
            if all(r is None for r in reqs):
                return
            if any(r != reqs[0] for r in reqs):
                raise RuntimeError(f"slabs reached different collective points: {reqs}")
            getattr(self.transport, reqs[0])(self.slabs)

    def run(self, nsteps: int, spec: StepSpec):
        for _ in range(nsteps):
            self.step(spec)


__all__ = ["slab_extents", "slab_grid", "StepSpec", "Slab", "DeviceSlab", "LoopbackTransport", "TorchTransport",
           "SlabRun"]
