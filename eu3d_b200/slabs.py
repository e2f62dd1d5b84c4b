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

With `dlb` set and the adaptive trapezoid (react TRAPEZOID, type 1), the
chemistry is load balanced across the slabs as the reference's
DynamicLoadBalancer does it (src/LoadBalance.cpp:8-159, src/Euler.cpp:380-700):

    predict -> all-gather the loads -> plan (same on every rank; skipped while
    the load degree (max - mean) / max is at most dlb_tol) -> rows selected ->
    all-reduce the cells per transfer -> packets to the receivers -> own cells
    -> received cells -> results back to the senders -> unpacked

With `dlb` set and the learned chemistry (react SURROGATE) the same protocol
balances its FP64 fallback: the predict half is the gate, network and apply,
a rank's load the length of its fallback list, and the transfers take the
last slots of that list (the rejected cells gather at the detonation front,
so the slabs it crosses carry most of them).

The result equals the unbalanced step bit for bit.

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
    dlb: bool = False       # balance the adaptive trapezoid / the learned chemistry's fallback across ranks
    dlb_tol: float = 0.0    # ... when the load degree exceeds this

    def kw(self) -> dict:
        d = dataclasses.asdict(self)
        del d["dlb"], d["dlb_tol"]
        return d

    def balanced(self) -> bool:
        return self.dlb and ((self.react == gpu.REACT_TRAPEZOID and self.type_ == 1)
                             or self.react == gpu.REACT_SURROGATE)

    def balance_kind(self) -> str:
        """"sur": the learned chemistry's fallback list; "trap": the adaptive trapezoid's rows."""
        return "sur" if self.react == gpu.REACT_SURROGATE else "trap"


class Slab:
    """One rank's slab.  Subclasses supply the operations on the state."""

    def __init__(self, rank: int, nranks: int, overlap: int, wedge: bool):
        self.rank, self.nranks, self.overlap, self.wedge = rank, nranks, overlap, wedge
        self.kind = "trap"  # what the balancing operations move (StepSpec.balance_kind)

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
    # load balancing (of self.kind): chem_load() -> int; dlb_select(amounts)
    # -> cells per transfer; dlb_pack(); dlb_guest(seg_cells); dlb_unpack();
    # and the packet segments out_seg(t) / in_seg(t) / guest_seg(t) /
    # back_seg(t) of transfer t
    def chem_load(self): raise NotImplementedError
    def dlb_select(self, amounts): raise NotImplementedError
    def dlb_alloc(self, n_out, n_in): raise NotImplementedError
    def dlb_pack(self): raise NotImplementedError
    def dlb_guest(self, seg_cells): raise NotImplementedError
    def dlb_unpack(self): raise NotImplementedError

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
        if spec.balanced():
            yield from self._balanced_chemistry(spec)
        else:
            self.part(gpu.PART_REACT, spec)

    def _balanced_chemistry(self, spec):
        self.kind = spec.balance_kind()
        sur = self.kind == "sur"
        predict = gpu.PART_SUR_PREDICT if sur else gpu.PART_CHEM_PREDICT
        work = gpu.PART_SUR_WORK if sur else gpu.PART_CHEM_WORK
        self.part(predict, spec)
        self.load = int(self.chem_load())
        yield "loads"  # -> self.loads, every rank's load in rank order
        plan = gpu.dlb_plan(self.loads) if gpu.load_degree(self.loads) > spec.dlb_tol else []
        self.plan = plan
        self.last_plan = plan
        if not plan:
            self.part(work, spec)
            return
        self.mine = [t for t, (s, _, _) in enumerate(plan) if s == self.rank]
        self.theirs = [t for t, (_, r, _) in enumerate(plan) if r == self.rank]
        cells = self.dlb_select([plan[t][2] for t in self.mine])
        self.sent = {t: int(c) for t, c in zip(self.mine, cells)}
        yield "dlb_counts"  # -> self.counts: cells of every transfer, in plan order
        c = self.counts
        self.dlb_alloc(sum(c[t] for t in self.mine), sum(c[t] for t in self.theirs))
        self.dlb_pack()
        # the packets travel while this rank integrates the cells it kept (the
        # reference overlaps its non-blocking sends the same way,
        # src/Euler.cpp:488-518); the guest work waits for them
        yield "dlb_out_start"
        self.part(work, spec)
        yield "dlb_out_wait"
        self.dlb_guest([c[t] for t in self.theirs])
        yield "dlb_back"
        self.dlb_unpack()

    def _offsets(self, ts, fields):
        """{transfer: (start, end)} of the segments of transfers ts, concatenated
        in that order, `fields` values per cell"""
        out, o = {}, 0
        for t in ts:
            n = self.counts[t] * fields
            out[t] = (o, o + n)
            o += n
        return out

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
        # load-balancing packets travel on this stream while the handle's
        # stream integrates the rank's own cells
        self.side = torch.cuda.Stream(device=f"cuda:{dev.device}")

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

    # load balancing: packets are torch CUDA tensors of doubles; self.kind
    # picks the trapezoid's rows or the learned chemistry's fallback list
    def chem_load(self):
        return self.d.sur_load() if self.kind == "sur" else self.d.chem_load()

    def dlb_select(self, amounts):
        if self.kind == "sur":
            return self.d.sdlb_select(amounts)
        cells, _ = self.d.dlb_select(amounts)
        return cells

    def _fields(self):
        if self.kind == "sur":
            return gpu.SDLB_OUT_FIELDS, gpu.SDLB_BACK_FIELDS
        return gpu.DLB_OUT_FIELDS, gpu.DLB_BACK_FIELDS

    def dlb_alloc(self, n_out, n_in):
        dev, f64 = f"cuda:{self.d.device}", self.torch.float64
        fo, fb = self._fields()
        self._out = self.torch.empty(max(1, n_out * fo), dtype=f64, device=dev)
        self._back_in = self.torch.empty(max(1, n_out * fb), dtype=f64, device=dev)
        self._in = self.torch.empty(max(1, n_in * fo), dtype=f64, device=dev)
        self._guest = self.torch.empty(max(1, n_in * fb), dtype=f64, device=dev)
        self._o_out = self._offsets(self.mine, fo)
        self._o_back = self._offsets(self.mine, fb)
        self._o_in = self._offsets(self.theirs, fo)
        self._o_guest = self._offsets(self.theirs, fb)

    def dlb_pack(self):
        (self.d.sdlb_pack if self.kind == "sur" else self.d.dlb_pack)(self._out.data_ptr())

    def dlb_guest(self, seg_cells):
        guest = self.d.sdlb_guest if self.kind == "sur" else self.d.dlb_guest
        guest(seg_cells, self._in.data_ptr(), self._guest.data_ptr())

    def dlb_unpack(self):
        (self.d.sdlb_unpack if self.kind == "sur" else self.d.dlb_unpack)(self._back_in.data_ptr())

    def out_seg(self, t):
        a, b = self._o_out[t]
        return self._out[a:b]

    def back_seg(self, t):
        a, b = self._o_back[t]
        return self._back_in[a:b]

    def in_seg(self, t):
        a, b = self._o_in[t]
        return self._in[a:b]

    def guest_seg(self, t):
        a, b = self._o_guest[t]
        return self._guest[a:b]


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

    def loads(self, slabs):
        allv = [s.load for s in sorted(slabs, key=lambda s: s.rank)]
        for s in slabs:
            s.loads = allv

    def dlb_counts(self, slabs):
        plan = slabs[0].plan
        counts = [0] * len(plan)
        for s in slabs:
            for t, c in s.sent.items():
                counts[t] = c
        for s in slabs:
            s.counts = counts

    def _by_rank(self, slabs):
        return {s.rank: s for s in slabs}

    def dlb_out_start(self, slabs):
        self._sync(slabs)
        by = self._by_rank(slabs)
        for t, (snd, rcv, _) in enumerate(slabs[0].plan):
            if by[rcv].counts[t]:
                by[rcv].in_seg(t).copy_(by[snd].out_seg(t))
        self._sync(slabs)

    def dlb_out_wait(self, slabs):
        pass  # the copies above are complete

    def dlb_back(self, slabs):
        self._sync(slabs)
        by = self._by_rank(slabs)
        for t, (snd, rcv, _) in enumerate(slabs[0].plan):
            if by[rcv].counts[t]:
                by[snd].back_seg(t).copy_(by[rcv].guest_seg(t))
        self._sync(slabs)


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

    def _vec(self, s, values):
        import torch
        dev = f"cuda:{s.d.device}" if isinstance(s, DeviceSlab) else "cpu"
        return torch.tensor(values, dtype=torch.int64, device=dev)

    def loads(self, slabs):
        (s,) = slabs
        with self._ctx(s):
            mine = self._vec(s, [s.load])
            allv = [self._vec(s, [0]) for _ in range(self.dist.get_world_size(self.group))]
            self.dist.all_gather(allv, mine, group=self.group)
        s.loads = [int(v.item()) for v in allv]

    def dlb_counts(self, slabs):
        (s,) = slabs
        counts = [0] * len(s.plan)
        for t, c in s.sent.items():
            counts[t] = c
        with self._ctx(s):
            v = self._vec(s, counts)
            self.dist.all_reduce(v, op=self.dist.ReduceOp.SUM, group=self.group)
        s.counts = [int(x) for x in v.tolist()]

    def _p2p(self, s, sends, recvs, side=False):
        """Posts the sends and receives; returns their requests.  side: on
        a device slab, issue them on the slab's side stream (after the
        packets are packed on its own stream), so that the slab's stream runs
        on while they travel."""
        dist = self.dist
        ops = [dist.P2POp(dist.isend, buf, peer, group=self.group) for buf, peer in sends]
        ops += [dist.P2POp(dist.irecv, buf, peer, group=self.group) for buf, peer in recvs]
        if not ops:
            return []
        if side and isinstance(s, DeviceSlab):
            s.side.wait_stream(s.stream)
            with s.torch.cuda.stream(s.side):
                return dist.batch_isend_irecv(ops)
        with self._ctx(s):
            return dist.batch_isend_irecv(ops)

    def _wait(self, s, reqs):
        # NCCL: the slab's stream waits for the transfers; gloo: the host waits
        with self._ctx(s):
            for req in reqs:
                req.wait()

    def dlb_out_start(self, slabs):
        (s,) = slabs
        plan = s.plan
        sends = [(s.out_seg(t), plan[t][1]) for t in s.mine if s.counts[t]]
        recvs = [(s.in_seg(t), plan[t][0]) for t in s.theirs if s.counts[t]]
        s._dlb_reqs = self._p2p(s, sends, recvs, side=True)

    def dlb_out_wait(self, slabs):
        (s,) = slabs
        self._wait(s, getattr(s, "_dlb_reqs", []))
        s._dlb_reqs = []

    def dlb_back(self, slabs):
        (s,) = slabs
        plan = s.plan
        sends = [(s.guest_seg(t), plan[t][0]) for t in s.theirs if s.counts[t]]
        recvs = [(s.back_seg(t), plan[t][1]) for t in s.mine if s.counts[t]]
        self._wait(s, self._p2p(s, sends, recvs))


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
