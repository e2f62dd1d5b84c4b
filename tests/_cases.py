"""Seeded synthetic states shared by the oracle-pin tests, the GPU parity
tests and tests/golden/make_golden.py.

A state is built on the oracle (the CPU restatement) from smooth seeded
fields of P, T, U, V, W and mass fractions with a little noise (so that the
limiter takes every branch), then completed with FieldInitial's arithmetic
(orc_prims_from_state).  The temperature window decides which NASA range is
exercised; states for the reference policy stay below 1000 K because the
reference's high-range enthalpy defect drives its chemistry non-finite there.
"""
from __future__ import annotations

import numpy as np

from eu3d_b200.readers import make_grid
from pyoracle import Oracle

QUIRKS_REF = 0x1FF
QUIRKS_FIXED = 0x000


def small_grid(ni=10, nj=6, nk=4, fixed_ghosts=True, lx=0.01, ly=0.006, lz=0.004):
    return make_grid(ni, 0.0, lx, nj, 0.0, ly, nk, 0.0, lz, 2, fixed_ghosts=fixed_ghosts)


def fill_state(o: Oracle, seed: int, tlo: float, thi: float, radicals: float = 1e-3, noise: float = 0.02):
    """Seeded, smooth-plus-noise primitive state on every cell of o."""
    rng = np.random.default_rng(seed)
    NI, NJ, NK, NS = o.NI, o.NJ, o.NK, o.NS
    x = np.linspace(0, 2 * np.pi, NI)[:, None, None]
    y = np.linspace(0, 2 * np.pi, NJ)[None, :, None]
    z = np.linspace(0, 2 * np.pi, NK)[None, None, :]
    ph = rng.uniform(0, 2 * np.pi, 8)
    smooth = 0.5 + 0.25 * (np.sin(x + ph[0]) * np.cos(y + ph[1]) + np.sin(z + ph[2]) * np.cos(x + ph[3]))
    T = tlo + (thi - tlo) * np.clip(smooth + noise * rng.standard_normal((NI, NJ, NK)), 0, 1)
    P = 101325.0 * (1.0 + 0.3 * np.sin(y + ph[4]) * np.sin(z + ph[5]) + noise * rng.standard_normal((NI, NJ, NK)))
    U = 300.0 * np.sin(x + ph[6]) + 30 * rng.standard_normal((NI, NJ, NK))
    V = 200.0 * np.cos(y + ph[7]) + 20 * rng.standard_normal((NI, NJ, NK))
    W = 100.0 * np.sin(z + ph[0]) + 10 * rng.standard_normal((NI, NJ, NK))
    sp = o.mech.species
    X = np.zeros((NI, NJ, NK, NS))
    X[..., sp.index("H2")] = 2.0 * (1 + 0.3 * np.sin(x + y))
    X[..., sp.index("O2")] = 1.0 * (1 + 0.2 * np.cos(y + z))
    X[..., sp.index("N2")] = 3.76
    for r in ("H", "O", "OH", "HO2", "H2O2"):
        X[..., sp.index(r)] = radicals * rng.uniform(0.2, 1.0, (NI, NJ, NK))
    X[..., sp.index("H2O")] = 0.3 * rng.uniform(0.0, 1.0, (NI, NJ, NK))
    Y = X * o.mech.mw
    Y /= Y.sum(axis=-1, keepdims=True)
    o.view("P")[...] = P
    o.view("T")[...] = T
    o.view("U")[...] = U
    o.view("V")[...] = V
    o.view("W")[...] = W
    o.view("Yi")[...] = Y
    o.prims_from_state()
    return o


def make_oracle(mech, seed=1, quirks=QUIRKS_FIXED, tlo=1100.0, thi=2600.0, grid=None, radicals=1e-3):
    g = grid or small_grid(fixed_ghosts=(quirks == QUIRKS_FIXED))
    o = Oracle(mech, g, quirks)
    fill_state(o, seed, tlo, thi, radicals)
    return o, g


STATE_OUT = ["CS", "T", "U", "V", "W", "P", "D", "H", "Gamma", "E", "Yi"]


def interior(a, bc=2):
    return a[bc:-bc, bc:-bc, bc:-bc]


def field_err(a, b):
    """max |a - b| / max |b| over a whole array (the field-normalised error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / scale)


def rel_err(a, b, mask=None):
    """Per-variable relative error: each variable is normalised by its own
    largest magnitude, and the worst variable is returned.  A 3D field
    (ni, nj, nk) is one variable; the last axis of a per-cell vector field
    (species mass fractions, the 13 conserved variables) indexes its
    variables, so a radical at Y ~ 1e-6 is held to the same relative bar as
    N2.  mask (ni, nj, nk), optional: only these cells count (the fluid cells
    of an immersed wedge)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
        vec = a.ndim == 2
    else:
        vec = a.ndim == 4
    if not vec:
        return field_err(a, b)
    return max(field_err(a[..., v], b[..., v]) for v in range(a.shape[-1]))
