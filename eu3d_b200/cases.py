"""Initial/boundary set-ups of the benchmark configurations (new: the
reference hard-codes only its RSBI case, src/Flowfield.cpp:159-230,
src/Reaction.cpp:339-398, and leaves the ZND/ODW boundaries empty or unfed).

Thermodynamic completion of a primitive state (P, T, U, V, W, Y) uses the
arithmetic of Flowfield::FieldInitial (src/Flowfield.cpp:193-229) with the
NASA-9 polynomials of Reaction::GetCpi/GetHi (src/Reaction.cpp:893-926).
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

from .readers import Grid, Mechanism, R_UNIVERSAL, make_grid, stoichiometric_h2_air

ATM = 101325.0


def species_thermo(mech: Mechanism, T, fixed: bool = True):
    """Per-species Cp_i, H_i in kJ/(kg K), kJ/kg (GetCpi/GetHi with Ri).
    fixed=False keeps the reference's high-range enthalpy constant defect."""
    T = np.asarray(T, dtype=np.float64)
    Tb = T[..., None]
    hi = Tb >= 1000.0
    c = [np.where(hi, mech.c1[k], mech.c0[k]) for k in range(9)]
    b1 = c[7] if fixed else mech.c0[7]
    ri = mech.ri
    cp = ri * (c[0] * Tb ** -2.0 + c[1] / Tb + c[2] + c[3] * Tb + c[4] * Tb ** 2 + c[5] * Tb ** 3 + c[6] * Tb ** 4)
    h = ri * (-c[0] / Tb + c[1] * np.log(Tb) + c[2] * Tb + c[3] * Tb ** 2 / 2 + c[4] * Tb ** 3 / 3 + c[5] * Tb ** 4 / 4
              + c[6] * Tb ** 5 / 5 + b1)
    return cp, h


def complete_state(mech: Mechanism, P, T, U, V, W, Y, fixed: bool = True) -> dict:
    """D, H, E, Gamma, C and the conserved vector from a primitive state."""
    P, T, U, V, W = (np.asarray(a, dtype=np.float64) for a in (P, T, U, V, W))
    Y = np.asarray(Y, dtype=np.float64)
    sdiv = np.sum(Y / mech.mw, axis=-1)
    Wav = 1.0 / sdiv
    Rgas = R_UNIVERSAL * 1000 / Wav
    D = P / (Rgas * T)
    cpi, hi = species_thermo(mech, T, fixed)
    ei = hi - mech.ri * T[..., None]
    Cp = np.sum(cpi * Y, axis=-1) * 1000
    H = np.sum(Y * hi, axis=-1) * 1000
    E = np.sum(Y * ei, axis=-1) * 1000
    G = Cp / (Cp - R_UNIVERSAL * sdiv * 1000)
    C = np.sqrt(G * P / D)
    CS = np.concatenate([D[..., None] * Y, (D * U)[..., None], (D * V)[..., None], (D * W)[..., None],
                         (D * E + 0.5 * (U ** 2 + V ** 2 + W ** 2) * D)[..., None]], axis=-1)
    return dict(D=D, H=H, E=E, Gamma=G, C=C, Cp=Cp, Rgas=Rgas, CS=CS)


@dataclasses.dataclass
class OdwCase:
    """3D (or 2D with nk = 2) oblique detonation over a wedge."""

    grid: Grid
    P: float
    T: float
    U: float
    Y: np.ndarray
    wedge: tuple  # (x0, y0, tan(angle))
    inflow: dict  # planes (nj, nk) / (nj, nk, NS)
    free: dict    # completed free-stream state


def odw_case(mech: Mechanism, ni: int, nj: int, nk: int, L: float = 0.2, mach: float = 7.0, P: float = 0.1 * ATM,
             T: float = 300.0, wedge_deg: float = 25.0, wedge_x: float = 0.1, pert: float = 0.01, seed: int = 0,
             fixed: bool = True) -> OdwCase:
    """Stoichiometric H2-air at Mach `mach`, P, T over a wedge starting at
    x = wedge_x * L.  Domain L x L/2, z extent (nk - 1) dx (cubic cells).
    The inflow density carries a seeded `pert` relative perturbation at
    constant pressure (T scaled inversely)."""
    dx = L / (ni - 1)
    g = make_grid(ni, 0.0, L, nj, 0.0, L / 2, nk, 0.0, max(nk - 1, 1) * dx, 2, fixed_ghosts=True)
    Y = stoichiometric_h2_air(mech)
    st = complete_state(mech, P, T, 0.0, 0.0, 0.0, Y, fixed)
    U = mach * float(st["C"])
    free = complete_state(mech, P, T, U, 0.0, 0.0, Y, fixed)
    rng = np.random.default_rng(seed)
    eps = pert * rng.uniform(-1.0, 1.0, (g.nj, g.nk))
    Tin = T / (1.0 + eps)
    Pin = np.full_like(Tin, P)
    Yin = np.broadcast_to(Y, (g.nj, g.nk, mech.NS)).copy()
    z = np.zeros_like(Tin)
    inl = complete_state(mech, Pin, Tin, z + U, z, z, Yin, fixed)
    inflow = dict(U=z + U, V=z, W=z, P=Pin, D=inl["D"], T=Tin, H=inl["H"], E=inl["E"], G=inl["Gamma"], Y=Yin)
    wedge = (wedge_x * L, 0.0, float(np.tan(np.radians(wedge_deg))))
    return OdwCase(g, P, T, U, Y, wedge, inflow, free)


def setup_odw(dev, case: OdwCase) -> None:
    """Uniform free stream everywhere, ODM inflow planes, wedge boundary."""
    dev.init_uniform(case.P, case.T, case.U, 0.0, 0.0, case.Y)
    f = case.inflow
    dev.set_inflow(f["U"], f["V"], f["W"], f["P"], f["D"], f["T"], f["H"], f["E"], f["G"], f["Y"])
    dev.set_wedge(*case.wedge)


def znd_case(mech: Mechanism, ni: int = 4000, L: float = 0.1, fixed: bool = True):
    """1D ZND detonation initiation: stoichiometric H2-air at 300 K, 1 atm;
    driver x < 5 mm of H2O:N2 = 2:3.76 at 3000 K, 30 atm.  nj = nk = 2 (the
    smallest extents the reference's mesh accepts)."""
    g = make_grid(ni, 0.0, L, 2, 0.0, L / (ni - 1), 2, 0.0, L / (ni - 1), 2, fixed_ghosts=True)
    NI, NJ, NK = g.ni + 4, g.nj + 4, g.nk + 4
    x = np.broadcast_to(g.xnode[:, None, None], (NI, NJ, NK))
    drv = x < 0.005
    Yu = stoichiometric_h2_air(mech)
    Yd = np.zeros(mech.NS)
    Yd[mech.species.index("H2O")] = 2.0 * mech.mw[mech.species.index("H2O")]
    Yd[mech.species.index("N2")] = 3.76 * mech.mw[mech.species.index("N2")]
    Yd /= Yd.sum()
    P = np.where(drv, 30 * ATM, ATM)
    T = np.where(drv, 3000.0, 300.0)
    Y = np.where(drv[..., None], Yd, Yu)
    z = np.zeros_like(P)
    st = complete_state(mech, P, T, z, z, z, Y, fixed)
    return g, dict(P=P, T=T, U=z, V=z, W=z, Yi=Y, **st)


def upload_primitive_state(dev, st: dict) -> None:
    """Upload a completed host state (dict of reference-layout arrays)."""
    for n in ("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "Yi", "CS"):
        dev.upload(n, st[n])


STATE_FIELDS = ("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "Yi", "CS")


def extrude_state(src, dst, k_src: int = None, i0: int = 0) -> None:
    """Copy the state of one z plane of handle `src` (default: its first
    interior plane) into every plane of handle `dst`: a spanwise-uniform 3D
    state from a 2D solution.  dst takes src's x planes i0 .. i0 + dst.NI - 1
    (ghosts included; i0 > 0 for an x slab of src's extent) and all of its y
    extent."""
    if src.NJ != dst.NJ or i0 < 0 or i0 + dst.NI > src.NI:
        raise ValueError("extrude_state: extents differ")
    k = src.grid.bc if k_src is None else k_src
    for n in STATE_FIELDS:
        a = src.download(n)[i0:i0 + dst.NI, :, k]
        b = np.ascontiguousarray(np.broadcast_to(a[:, :, None], (dst.NI, dst.NJ, dst.NK) + a.shape[2:]))
        dst.upload(n, b)
        del b


__all__ = ["extrude_state", "STATE_FIELDS", "complete_state", "species_thermo", "odw_case", "setup_odw", "znd_case", "upload_primitive_state",
           "OdwCase", "ATM"]
