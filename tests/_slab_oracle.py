"""The oracle as a slab of the x-slab decomposition (test infrastructure):
implements eu3d_b200.slabs.Slab on an oracle field so that the product's
SlabRun and transports drive the reference's algorithm on the CPU.

Halo fields are the ones Flowfield::Mpi_Boundary sends
(src/Flowfield.cpp:796-806): D, U, V, W, P, T, H, Gamma, C and the species.
The stage arithmetic of SSP-RK2 repeats orc_step's (oracle/eu3d_oracle.c)."""
from __future__ import annotations

import numpy as np
import torch

from eu3d_b200 import gpu
from eu3d_b200.slabs import Slab

HALO3 = ["D", "U", "V", "W", "P", "T", "H", "Gamma", "C"]


class OracleSlab(Slab):
    def __init__(self, o, rank, nranks, overlap=0):
        super().__init__(rank, nranks, overlap, wedge=False)
        self.o = o
        self._dt = torch.zeros(1, dtype=torch.float64)
        n = sum(o.view(f)[0:2].size for f in HALO3) + o.view("Yi")[0:2].size
        self._recv = {s: torch.zeros(n, dtype=torch.float64) for s in (0, 1)}
        self._cs0 = None

    def _planes(self, i0):
        o = self.o
        return [o.view(f)[i0:i0 + 2] for f in HALO3] + [o.view("Yi")[i0:i0 + 2]]

    def cfl_local(self, cfl, final_time):
        t0 = self.o.time
        self.o.cfl(cfl, final_time)
        self.o.time = t0
        self._dt[0] = self.o.dt

    def dt_buffer(self):
        return self._dt

    def advance_time(self):
        self.o.dt = float(self._dt[0])
        self.o.time = self.o.time + self.o.dt

    def boundary(self, kind):
        self.o.boundary(kind)

    def pack(self, side):
        o = self.o
        i0 = o.bc + self.overlap if side == 0 else o.ni + o.bc - 2 - self.overlap
        return torch.from_numpy(np.concatenate([a.ravel() for a in self._planes(i0)]))

    def recv_buffer(self, side):
        return self._recv[side]

    def unpack(self, side):
        o = self.o
        i0 = 0 if side == 0 else o.ni + o.bc
        buf, off = self._recv[side].numpy(), 0
        for a in self._planes(i0):
            a[...] = buf[off:off + a.size].reshape(a.shape)
            off += a.size

    def _interior(self, name):
        o, b = self.o, self.o.bc
        return o.view(name)[b:o.ni + b, b:o.nj + b, b:o.nk + b]

    def part(self, part, spec):
        o = self.o
        rk = spec.timeadv in (gpu.ADV_SSPRK2, gpu.ADV_SSPRK3)
        if part == gpu.PART_STAGE1:
            if rk:
                self._cs0 = o.view("CS").copy()
                o.advection(gpu.ADV_EE, spec.diff)
                cs = self._interior("CS")
                cs += self._interior("RHS")
                o.update_after_cs()
            else:
                o.advection(spec.timeadv, spec.diff)
        elif part in (gpu.PART_STAGE2, gpu.PART_STAGE3):
            # SSP-RK2: 1/2, 1/2; SSP-RK3 (Shu-Osher): 3/4, 1/4 then 1/3, 2/3
            wn, ws = ((0.5, 0.5) if spec.timeadv == gpu.ADV_SSPRK2 else
                      (0.75, 0.25) if part == gpu.PART_STAGE2 else (1.0 / 3.0, 2.0 / 3.0))
            last = spec.timeadv == gpu.ADV_SSPRK2 or part == gpu.PART_STAGE3
            o.advection(gpu.ADV_EE, spec.diff)
            b = o.bc
            cs0 = self._cs0[b:o.ni + b, b:o.nj + b, b:o.nk + b]
            cs, rhs = self._interior("CS"), self._interior("RHS")
            cs[...] = wn * cs0 + ws * (cs + rhs)
            o.update_after_cs()
            if last:
                o.view("RHS")[...] = 0.0
        elif part == gpu.PART_REACT:
            if rk:
                if spec.react == gpu.REACT_IMEX:
                    o.partial_t()
                    o.imex()
                elif spec.react == gpu.REACT_TRAPEZOID:
                    o.trapezoid(spec.type_)
            elif spec.react == gpu.REACT_TRAPEZOID:
                o.trapezoid(spec.type_)
            elif spec.react == gpu.REACT_IMEX:
                o.imex()
            else:
                o.update_after_adv()
                o.explicit()
