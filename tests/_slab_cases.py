"""Shared set-up of the x-slab decomposition tests: one seeded full-domain
oracle, the slabs cut from it, and the interior comparison."""
from __future__ import annotations

import numpy as np

from _cases import QUIRKS_FIXED, fill_state
from eu3d_b200.readers import make_grid
from eu3d_b200.slabs import slab_extents, slab_grid
from pyoracle import Oracle

# every array of an oracle field that a step reads or writes
FIELDS = ["U", "V", "W", "P", "D", "T", "C", "Ma", "Wav", "Rgas", "Cp", "H", "E", "Gamma", "Mc", "Yi", "Di", "CS",
          "RHS", "Partion_T"]


def dyadic_grid(ni, nj, nk):
    """Nodes on multiples of 1/128 m: every node spacing is exact, so the CFL
    spacing xnode[1] - xnode[0] is the same on every slab."""
    h = 1.0 / 128
    return make_grid(ni, 0.0, (ni - 1) * h, nj, 0.0, (nj - 1) * h, nk, 0.0, (nk - 1) * h, 2, fixed_ghosts=True)


def full_oracle(mech, dims, seed=3, quirks=QUIRKS_FIXED):
    o = Oracle(mech, dyadic_grid(*dims), quirks)
    fill_state(o, seed, 1100.0, 2600.0)
    o.dt = 1e-8
    return o


def cut(mech, full, nranks, layout, quirks=QUIRKS_FIXED):
    """Oracle slabs holding the full field's cells (ghost planes included)."""
    g = dyadic_grid(full.ni, full.nj, full.nk)
    out = []
    for i0, n in slab_extents(full.ni, nranks, layout):
        o = Oracle(mech, slab_grid(g, i0, n), quirks)
        for f in FIELDS:
            o.view(f)[...] = full.view(f)[i0:i0 + n + 2 * g.bc]
        o.dt, o.time = full.dt, full.time
        out.append((i0, n, o))
    return out


def interior(o, name):
    b = o.bc
    return o.view(name)[b:o.ni + b, b:o.nj + b, b:o.nk + b]


def assert_slabs_equal_full(full, pieces, names=("CS", "T", "P", "Yi")):
    for i0, n, o in pieces:
        for f in names:
            a = interior(o, f)
            b = interior(full, f)[i0:i0 + n]
            assert np.all(np.isfinite(b)), f
            assert np.array_equal(a, b), (f, i0, n, np.max(np.abs(a - b)))
        assert o.time == full.time and o.dt == full.dt
