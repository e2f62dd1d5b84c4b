"""A host-memory slab for the load-balancing protocol tests (CPU, no GPU).

Its chemistry is a stand-in with the property the device path relies on: a
cell's result depends only on its own value and its predicted count.  The
packets follow the device layout (field-major per segment, a count of -1 for a
solid cell) with two fields: value and count.  The row picker is the
library's (eu3d_dlb_select_rows); plan, load degree and collectives are the
ones eu3d_b200.slabs uses with device slabs."""
from __future__ import annotations

import numpy as np
import torch

from eu3d_b200 import gpu
from eu3d_b200.slabs import Slab

FIELDS = 2


def predict(vals):
    return 1 + (np.floor(vals * 7.0).astype(np.int64) % 5) * (1 + (vals > 0.8) * 20)


def chem(vals, counts):
    out = vals.copy()
    for n in range(int(counts.max(initial=0))):
        live = counts > n
        out[live] = out[live] * 0.999 + 0.5 / (n + 1)
    return out


class HostSlab(Slab):
    def __init__(self, vals, solid, rank, nranks):
        super().__init__(rank, nranks, 0, False)
        self.vals = np.array(vals, dtype=np.float64)  # (rows, width)
        self.solid = np.array(solid, dtype=bool)
        self.cnt = np.zeros(self.vals.shape, dtype=np.int64)
        self.away = (0, 0)

    def step(self, spec):
        if spec.balanced():
            yield from self._balanced_chemistry(spec)
        else:
            self.part(gpu.PART_REACT, spec)

    def part(self, part, spec):
        if part in (gpu.PART_CHEM_PREDICT, gpu.PART_REACT):
            self.cnt = predict(self.vals)
            self.away = (0, 0)
        if part in (gpu.PART_CHEM_WORK, gpu.PART_REACT):
            live = ~self.solid
            live[self.away[0]:self.away[1]] = False
            self.vals[live] = chem(self.vals[live], self.cnt[live])

    def chem_load(self):
        return int(self.cnt[~self.solid].sum())

    def dlb_select(self, amounts):
        rowload = np.where(self.solid, 0, self.cnt).sum(axis=1)
        bounds, _ = gpu.dlb_select_rows(rowload, amounts)
        self.bounds = bounds
        return (np.diff(bounds) * self.vals.shape[1]).astype(np.int64)

    def dlb_alloc(self, n_out, n_in):
        z = lambda n: torch.zeros(max(1, n * FIELDS), dtype=torch.float64)
        self._out, self._back, self._in, self._guest = z(n_out), z(n_out), z(n_in), z(n_in)
        self._o_out = self._offsets(self.mine, FIELDS)
        self._o_in = self._offsets(self.theirs, FIELDS)

    def dlb_pack(self):
        w = self.vals.shape[1]
        for p, t in enumerate(self.mine):
            r0, r1 = self.bounds[p], self.bounds[p + 1]
            v = self.vals[r0:r1].reshape(-1)
            c = np.where(self.solid[r0:r1], -1, self.cnt[r0:r1]).reshape(-1)
            a, b = self._o_out[t]
            self._out[a:b] = torch.from_numpy(np.concatenate([v, c.astype(np.float64)]))
            assert b - a == (r1 - r0) * w * FIELDS
        self.away = (int(self.bounds[0]), int(self.bounds[-1]))

    def dlb_guest(self, seg_cells):
        for t, n in zip(self.theirs, seg_cells):
            a, b = self._o_in[t]
            seg = self._in[a:b].numpy()
            v, c = seg[:n], seg[n:].astype(np.int64)
            live = c >= 0
            res = v.copy()
            res[live] = chem(v[live], c[live])
            self._guest[a:b] = torch.from_numpy(np.concatenate([res, c.astype(np.float64)]))

    def dlb_unpack(self):
        for p, t in enumerate(self.mine):
            r0, r1 = self.bounds[p], self.bounds[p + 1]
            a, b = self._o_out[t]
            n = (b - a) // FIELDS
            if n == 0:
                continue
            back = self._back[a:b].numpy()
            v = back[:n].reshape(r1 - r0, -1)
            keep = self.solid[r0:r1]
            self.vals[r0:r1] = np.where(keep, self.vals[r0:r1], v)

    def out_seg(self, t):
        a, b = self._o_out[t]
        return self._out[a:b]

    def back_seg(self, t):
        a, b = self._o_out[t]
        return self._back[a:b]

    def in_seg(self, t):
        a, b = self._o_in[t]
        return self._in[a:b]

    def guest_seg(self, t):
        a, b = self._o_in[t]
        return self._guest[a:b]


def make_slabs(nranks, rows=12, width=5, seed=0):
    """Rank 0 hot (large counts), the others cool; a few solid cells."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(nranks):
        vals = rng.uniform(0.0, 0.75, (rows, width))
        if r == 0:
            vals[: rows // 2] = rng.uniform(0.8, 1.0, (rows // 2, width))
        solid = np.zeros((rows, width), dtype=bool)
        solid[1, 2] = solid[rows - 1, 0] = True
        out.append((vals, solid))
    return out


def unbalanced(slabs_data):
    return [np.where(s, v, chem(v, predict(v))) for v, s in slabs_data]


# ----------------------------------------------------------------------------
# The learned chemistry's fallback list (the "sur" kind of the protocol): the
# cells above a threshold are "rejected" and listed; the stand-in integration
# depends only on the cell's own value; a sender's transfers take the last
# slots of its list, as eu3d_sdlb_select does.  One field per packet cell.
def rejected(vals, solid):
    return (vals > 0.6) & ~solid


def chem_one(v):
    out = v.copy()
    for n in range(6):
        out = out * 0.997 + 0.25 / (n + 1) * np.sin(out)
    return out


class HostListSlab(Slab):
    def __init__(self, vals, solid, rank, nranks, order_seed=0):
        super().__init__(rank, nranks, 0, False)
        self.vals = np.array(vals, dtype=np.float64)
        self.solid = np.array(solid, dtype=bool)
        self.rng = np.random.default_rng(order_seed + 7 * rank)
        self.list = np.zeros(0, dtype=np.int64)
        self.keep = 0

    def step(self, spec):
        if spec.balanced():
            yield from self._balanced_chemistry(spec)
        else:
            self.part(gpu.PART_REACT, spec)

    def part(self, part, spec):
        flat = self.vals.reshape(-1)
        if part in (gpu.PART_SUR_PREDICT, gpu.PART_REACT):
            # the device appends with atomics: the list order is arbitrary
            self.list = self.rng.permutation(np.flatnonzero(rejected(self.vals, self.solid).reshape(-1)))
            self.keep = len(self.list)
        if part in (gpu.PART_SUR_WORK, gpu.PART_REACT):
            kept = self.list[:self.keep]
            flat[kept] = chem_one(flat[kept])

    def chem_load(self):
        return len(self.list)

    def dlb_select(self, amounts):
        left, cells = len(self.list), []
        for a in amounts:
            c = min(int(a), left)
            cells.append(c)
            left -= c
        self.keep = left
        self.seg = np.concatenate([[0], np.cumsum(cells)]).astype(np.int64)
        return np.array(cells, dtype=np.int64)

    def dlb_alloc(self, n_out, n_in):
        z = lambda n: torch.zeros(max(1, n), dtype=torch.float64)
        self._out, self._back, self._in, self._guest = z(n_out), z(n_out), z(n_in), z(n_in)
        self._o_out = self._offsets(self.mine, 1)
        self._o_in = self._offsets(self.theirs, 1)

    def dlb_pack(self):
        flat = self.vals.reshape(-1)
        for p, t in enumerate(self.mine):
            a, b = self._o_out[t]
            slots = self.list[self.keep + self.seg[p]:self.keep + self.seg[p + 1]]
            self._out[a:b] = torch.from_numpy(flat[slots].copy())

    def dlb_guest(self, seg_cells):
        for t in self.theirs:
            a, b = self._o_in[t]
            self._guest[a:b] = torch.from_numpy(chem_one(self._in[a:b].numpy()))

    def dlb_unpack(self):
        flat = self.vals.reshape(-1)
        for p, t in enumerate(self.mine):
            a, b = self._o_out[t]
            slots = self.list[self.keep + self.seg[p]:self.keep + self.seg[p + 1]]
            flat[slots] = self._back[a:b].numpy()

    def out_seg(self, t):
        a, b = self._o_out[t]
        return self._out[a:b]

    def back_seg(self, t):
        a, b = self._o_out[t]
        return self._back[a:b]

    def in_seg(self, t):
        a, b = self._o_in[t]
        return self._in[a:b]

    def guest_seg(self, t):
        a, b = self._o_in[t]
        return self._guest[a:b]


def unbalanced_list(slabs_data, steps=1):
    out = []
    for v, s in slabs_data:
        v = v.copy()
        for _ in range(steps):
            m = rejected(v, s)
            v[m] = chem_one(v[m])
        out.append(v)
    return out
