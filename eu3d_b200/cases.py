"""Initial/boundary set-ups of the benchmark configurations: the 1D ZND
detonation, the 2D/3D oblique detonation over a wedge and the 3D reactive
shock-bubble interaction (new: the reference hard-codes only its 2D RSBI
case, src/Flowfield.cpp:159-230, src/Reaction.cpp:339-398, and leaves the
ZND/ODW boundaries empty or unfed).

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


def real_sph_harm(l: int, m: int, theta, phi):
    """Real orthonormal spherical harmonic of degree l, order m at polar angle
    theta and azimuth phi (m > 0: the cosine form, m < 0: the sine form)."""
    from scipy.special import sph_harm_y
    y = sph_harm_y(l, abs(m), theta, phi)
    if m == 0:
        return np.real(y)
    s = np.sqrt(2.0) * (-1.0) ** m
    return s * (np.real(y) if m > 0 else np.imag(y))


def radial_perturbation(lmax: int = 8, seed: int = 0, samples: int = 181):
    """f(theta, phi): a seeded sum of the real spherical harmonics of degrees
    1..lmax with standard-normal coefficients, scaled so that its largest
    magnitude over the sphere (sampled on a samples x 2 samples theta-phi
    grid) is 1."""
    rng = np.random.default_rng(seed)
    coef = {(l, m): rng.standard_normal() for l in range(1, lmax + 1) for m in range(-l, l + 1)}

    def raw(th, ph):
        out = np.zeros(np.broadcast(th, ph).shape)
        for (l, m), c in coef.items():
            out += c * real_sph_harm(l, m, th, ph)
        return out

    th = np.linspace(0.0, np.pi, samples)[:, None]
    ph = np.linspace(0.0, 2.0 * np.pi, 2 * samples, endpoint=False)[None, :]
    scale = np.max(np.abs(raw(th, ph)))
    return lambda theta, phi: raw(theta, phi) / scale


@dataclasses.dataclass
class RsbiCase:
    """3D reactive shock-bubble interaction on a cube of side W."""

    grid: Grid
    state: dict      # completed state on every cell, ghosts included (reference layout)
    shock_x: float   # initial shock position [m]; post-shock gas for x < shock_x
    centre: tuple    # bubble centre [m]
    radius: float    # unperturbed bubble radius [m]
    post: dict       # post-shock P, T, U


def rsbi_case(mech: Mechanism, n: int = 256, W: float = 0.1, mach: float = 2.0, P: float = ATM, T: float = 300.0,
              radius: float = 0.25, centre: float = 0.5, amp: float = 0.02, lmax: int = 8, width_cells: float = 2.0,
              shock_x: float = 0.1, seed: int = 0, fixed: bool = True, chunk: int = 16) -> RsbiCase:
    """Mach `mach` planar shock in air (O2:N2 = 1:3.76 molar, T, P) moving in
    +x from x = shock_x W towards a stoichiometric H2-O2 bubble (H2:O2 = 2:1)
    of radius `radius` W centred at `centre` W in every direction, at the
    same pressure and temperature.  The post-shock state follows the
    normal-shock relations of Flowfield::FieldInitial (src/Flowfield.cpp:
    172-174: gamma 1.4, R 287 J/(kg K)).  The bubble surface is
    r = R (1 + amp f(theta, phi)) with f the seeded spherical-harmonic sum of
    degrees 1..lmax (radial_perturbation, largest magnitude 1, so amp is the
    largest relative deviation); the composition crosses it as
    chi = (1 - tanh((r - R(theta, phi)) / (width_cells dx))) / 2, the bubble's
    mass fraction.  The perturbation is evaluated within 12 interface widths
    of the perturbed shell; beyond them chi is taken with R = radius W, where
    the tanh is within 1e-10 of its limits either way.  Cubic cells, n^3 of
    them; the state is completed with FieldInitial's arithmetic
    (complete_state) in x chunks of `chunk` planes."""
    dx = W / (n - 1)
    g = make_grid(n, 0.0, W, n, 0.0, W, n, 0.0, W, 2, fixed_ghosts=True)
    NI, NJ, NK = g.ni + 4, g.nj + 4, g.nk + 4
    NS = mech.NS
    Ya = np.zeros(NS)
    Ya[mech.species.index("O2")] = 1.0 * mech.mw[mech.species.index("O2")]
    Ya[mech.species.index("N2")] = 3.76 * mech.mw[mech.species.index("N2")]
    Ya /= Ya.sum()
    Yb = np.zeros(NS)
    Yb[mech.species.index("H2")] = 2.0 * mech.mw[mech.species.index("H2")]
    Yb[mech.species.index("O2")] = 1.0 * mech.mw[mech.species.index("O2")]
    Yb /= Yb.sum()
    m2 = mach * mach
    U_post = mach * (1 - (2 + 0.40 * m2) / (2.40 * m2)) * np.sqrt(1.40 * 287 * T)
    P_post = P * (1 + 2 * 1.4 / 2.4 * (m2 - 1.0))
    T_post = T * (2 + 0.40 * m2) / (2.40 * m2) * P_post / P
    c = (centre * W,) * 3
    R0 = radius * W
    st = {k: np.empty((NI, NJ, NK)) for k in ("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "C")}
    st["Yi"] = np.empty((NI, NJ, NK, NS))
    st["CS"] = np.empty((NI, NJ, NK, NS + 4))
    f = radial_perturbation(lmax, seed)
    wid = width_cells * dx
    band = amp * R0 + 12.0 * wid
    y = g.ynode[None, :, None] - c[1]
    z = g.znode[None, None, :] - c[2]
    for i0 in range(0, NI, chunk):
        sl = slice(i0, min(i0 + chunk, NI))
        x = g.xnode[sl][:, None, None] - c[0]
        r = np.sqrt(x * x + y * y + z * z)
        R = np.full_like(r, R0)
        near = np.abs(r - R0) <= band
        if near.any():
            xb, yb, zb = (np.broadcast_to(a, r.shape)[near] for a in (x, y, z))
            rb = r[near]
            theta = np.arccos(np.clip(np.divide(zb, rb, out=np.zeros_like(rb), where=rb > 0), -1.0, 1.0))
            phi = np.arctan2(yb, xb) % (2.0 * np.pi)
            R[near] = R0 * (1.0 + amp * f(theta, phi))
        chi = 0.5 * (1.0 - np.tanh((r - R) / wid))
        Y = chi[..., None] * Yb + (1.0 - chi[..., None]) * Ya
        post = np.broadcast_to(g.xnode[sl][:, None, None] < shock_x * W, r.shape)
        Pc = np.where(post, P_post, P)
        Tc = np.where(post, T_post, T)
        Uc = np.where(post, U_post, 0.0)
        zero = np.zeros_like(Pc)
        cs = complete_state(mech, Pc, Tc, Uc, zero, zero, Y, fixed)
        for k, v in (("U", Uc), ("V", zero), ("W", zero), ("P", Pc), ("T", Tc), ("D", cs["D"]), ("H", cs["H"]),
                     ("Gamma", cs["Gamma"]), ("E", cs["E"]), ("C", cs["C"]), ("Yi", Y), ("CS", cs["CS"])):
            st[k][sl] = v
    return RsbiCase(g, st, shock_x * W, c, R0, dict(P=P_post, T=T_post, U=U_post))


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


__all__ = ["extrude_state", "STATE_FIELDS", "complete_state", "species_thermo", "odw_case", "setup_odw", "znd_case",
           "rsbi_case", "RsbiCase", "radial_perturbation", "real_sph_harm", "upload_primitive_state", "OdwCase", "ATM"]
