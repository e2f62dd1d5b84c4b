"""Temporal order of the time schemes on the oracle (CPU).

EE (TimeAdv::EE, src/TimeAdv.cpp:29-43), SSP-RK2 and SSP-RK3 (Shu and Osher,
J. Comput. Phys. 77, 1988; new -- the reference's TVD_RK3 is a stub,
src/TimeAdv.cpp:57-67) on a smooth 1D wave without chemistry and with the
first-order reconstruction (MUSCL_1), whose right-hand side is smooth: with
the spatial operator fixed, the difference between runs at dt and dt/2 falls
by 2^p for a scheme of order p.  The GPU path reproduces these schemes to
1e-10 (tests/test_gpu_parity.py, imex_rk2/imex_rk3).
"""
import numpy as np
import pytest

from _cases import QUIRKS_FIXED, fill_state, interior, small_grid
from eu3d_b200 import gpu
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
