"""Order of accuracy of the time and space schemes on the oracle (CPU).

Time:

EE (TimeAdv::EE, src/TimeAdv.cpp:29-43), SSP-RK2 and SSP-RK3 (Shu and Osher,
J. Comput. Phys. 77, 1988; new -- the reference's TVD_RK3 is a stub,
src/TimeAdv.cpp:57-67) on a smooth 1D wave without chemistry and with the
first-order reconstruction (MUSCL_1), whose right-hand side is smooth: with
the spatial operator fixed, the difference between runs at dt and dt/2 falls
by 2^p for a scheme of order p.

Space: the flux residual per unit time (Advection + EE with dt = 1) of one
smooth state on grids of 65, 129 and 257 nodes against 1025 nodes, at the
shared nodes of the middle half of the domain, in the field-relative L1
norm: MUSCL_1 first order, MUSCL_2 (include/Differ.hpp:149-238) and the WENO
option (third-order Jiang-Shu reconstruction, new) second order -- the
primitives are cell values of a finite-volume scheme, which caps the
residual at second order whatever the reconstruction.  In the max norm both
limited reconstructions fall to first order at the smooth extrema.

The GPU path reproduces these schemes to 1e-10 (tests/test_gpu_parity.py).
"""
import numpy as np
import pytest

from _cases import QUIRKS_FIXED, fill_state, interior, small_grid
from eu3d_b200 import gpu
from eu3d_b200.readers import make_grid
from pyoracle import Oracle


def _wave(mech, nsteps, timeadv, t_end=4e-7):
    g = small_grid(32, 4, 4, lx=0.032, ly=0.004, lz=0.004)
    o = Oracle(mech, g, QUIRKS_FIXED)
    fill_state(o, 5, 1100.0, 1300.0, 1e-6, noise=0.0)
    x = np.linspace(0, 2 * np.pi, o.NI)[:, None, None]
    o.view("U")[...] = 100.0 * np.sin(x) + 50.0
    o.view("V")[...] = 0.0
    o.view("W")[...] = 0.0
    o.view("T")[...] = 1200.0 + 50.0 * np.cos(x)
    o.view("P")[...] = 101325.0
    o.view("Yi")[...] = o.view("Yi")[:1, :1, :1].copy()  # one composition everywhere
    o.prims_from_state()
    for _ in range(nsteps):
        o.dt = t_end / nsteps
        o.step(gpu.REACT_NONE, 0, timeadv, gpu.DIFF_MUSCL1, 0.0, 1.0, gpu.BC_TRANSMISSIVE)
    return interior(o.view("CS")).copy()


@pytest.mark.parametrize("timeadv,order", [(gpu.ADV_EE, 1), (gpu.ADV_SSPRK2, 2), (gpu.ADV_SSPRK3, 3)],
                         ids=["ee", "ssprk2", "ssprk3"])
def test_temporal_order(mech, timeadv, order):
    runs = [_wave(mech, n, timeadv) for n in (8, 16, 32)]
    d1 = np.abs(runs[0] - runs[1]).max()
    d2 = np.abs(runs[1] - runs[2]).max()
    ratio = d1 / d2
    assert 2 ** order * 0.85 < ratio < 2 ** order * 1.2, (d1, d2, ratio)


def _residual(mech, n, diff, length=0.064):
    g = make_grid(n, 0.0, length, 2, 0.0, 0.001, 2, 0.0, 0.001, 2, fixed_ghosts=True)
    o = Oracle(mech, g, QUIRKS_FIXED)
    fill_state(o, 5, 1100.0, 1300.0, 1e-6, noise=0.0)
    x = g.xnode[:, None, None] / length * 2 * np.pi
    o.view("U")[...] = 100.0 * np.sin(x) + 50.0
    o.view("V")[...] = 0.0
    o.view("W")[...] = 0.0
    o.view("T")[...] = 1200.0 + 50.0 * np.cos(x)
    o.view("P")[...] = 101325.0 * (1.0 + 0.05 * np.sin(2 * x))
    sp = mech.species
    X = np.zeros(mech.NS)
    X[sp.index("H2")], X[sp.index("O2")], X[sp.index("N2")] = 2.0, 1.0, 3.76
    Y = X * mech.mw
    o.view("Yi")[...] = Y / Y.sum()
    o.prims_from_state()
    o.boundary(gpu.BC_TRANSMISSIVE)
    o.dt = 1.0
    o.advection(gpu.ADV_EE, diff)
    b = g.bc
    return g.xnode[b:-b], o.view("RHS")[b:-b, b, b, :].copy()


@pytest.mark.parametrize("diff,lo,hi", [(gpu.DIFF_MUSCL1, 1.7, 2.7), (gpu.DIFF_MUSCL2, 3.5, 4.6),
                                        (gpu.DIFF_WENO, 3.4, 4.6)], ids=["muscl1", "muscl2", "weno"])
def test_spatial_order(mech, diff, lo, hi):
    length, fine = 0.064, 1025
    xf, rf = _residual(mech, fine, diff, length)
    errs = []
    for n in (65, 129, 257):
        x, r = _residual(mech, n, diff, length)
        ref = rf[::(fine - 1) // (n - 1)]
        mid = (x > 0.25 * length) & (x < 0.75 * length)
        rel = np.abs(r[mid] - ref[mid]).mean(axis=0) / np.abs(ref[mid]).mean(axis=0).clip(1e-300)
        errs.append(rel[[2, 8, 9, 12]].max())  # two species, x momentum, energy
    ratios = [errs[0] / errs[1], errs[1] / errs[2]]
    assert all(lo < q < hi for q in ratios), (errs, ratios)
