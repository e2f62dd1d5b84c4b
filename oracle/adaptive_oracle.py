"""CPU oracle of the adaptive closed-reactor chemistry (test infrastructure
only: the product never imports this file).

The integrator is new (no counterpart in the reference): substeps of the
species-diagonal implicit update rho_s += h CMS_s / (1 - h MD_s) with CMS and
MD from the oracle's Reaction::Diagonalized restatement (orc_diagonalized,
following src/Reaction.cpp:736-811) evaluated with Partion_T = 0 (the
composition part of the Jacobian), a decode (orc_update_after_cs, following
src/Flowfield.cpp:1246-1284) after each substep, the substep rule

    h = min(t_left, min_s rel (rho_s + 1e-9 rho) / |CMS_s|, min_{MD_s>0} amp / MD_s),
    h = min(max(h, dt / nmax), t_left), the last allowed substep takes t_left,

negative partial densities clipped to zero, then the mass-fraction change
projected to element conservation (least change in the metric
sum dY^2 / (Y + eps)).  Cells advance independently (each its own h).
"""
from __future__ import annotations

import numpy as np


def element_matrix(mech, atoms):
    return np.asarray(atoms, dtype=np.float64) / mech.mw


def project(Y, dY, A, eps):
    w = Y + eps
    r = dY @ A.T
    M = np.einsum("ek,nk,fk->nef", A, w, A)
    lam = np.linalg.solve(M, r[..., None])[..., 0]
    return dY - w * (lam @ A)


def _interior(o, name):
    b = o.bc
    return o.view(name)[b:-b, b:-b, b:-b]


def increment(o, dt, atoms, rel=0.02, amp=0.5, nmax=1024, proj_eps=1e-4):
    """Chemistry increment over dt of every interior cell of oracle field o
    (its current state): returns dY (ni, nj, nk, NS), Tchem (ni, nj, nk),
    substeps (ni, nj, nk).  The field's state is left as it was."""
    NS = o.NS
    keep = {n: o.view(n).copy() for n in ("CS", "T", "E", "D", "U", "V", "W", "P", "H", "Gamma", "Yi", "Mc",
                                          "Di", "Partion_T")}
    A = element_matrix(o.mech, atoms)
    # Di, Mc as the decode leaves them for the current CS (src/Flowfield.cpp:1254-1256)
    o.view("Di")[...] = o.view("CS")[..., :NS]
    o.view("Mc")[...] = o.view("Di") / o.mech.mw * 1000
    cs0 = _interior(o, "CS").copy()
    shape = cs0.shape[:3]
    trem = np.full(shape, dt)
    nsub = np.zeros(shape, dtype=np.int64)
    hmin = dt / nmax
    k = 0
    while (trem > 0).any() and k < nmax:
        o.view("Partion_T")[...] = 0.0
        o.lib().orc_diagonalized(*o._fm())
        c = _interior(o, "CS")
        w = _interior(o, "CMS")
        md = _interior(o, "MDd")[..., :NS]
        rho = c[..., :NS].copy()
        D = rho.sum(-1)
        with np.errstate(divide="ignore", invalid="ignore"):
            hr = np.where(np.abs(w) > 0, rel * (rho + 1e-9 * D[..., None]) / np.abs(w), np.inf)
            ha = np.where(md > 0, amp / md, np.inf)
        h = np.minimum(trem, np.minimum(hr.min(-1), ha.min(-1)))
        h = np.minimum(np.maximum(h, hmin), trem)
        if k == nmax - 1:
            h = trem.copy()
        act = trem > 0
        h = np.where(act, h, 0.0)
        new = np.maximum(rho + h[..., None] * w / (1.0 - h[..., None] * md), 0.0)
        T_before = _interior(o, "T").copy()
        c[..., :NS] = np.where(act[..., None], new, rho)
        o.update_after_cs()
        T = _interior(o, "T")
        T[...] = np.where(act, T, T_before)
        trem = trem - h
        nsub += act
        k += 1
    c = _interior(o, "CS")
    Y0 = cs0[..., :NS] / cs0[..., :NS].sum(-1)[..., None]
    dY = c[..., :NS] / c[..., :NS].sum(-1)[..., None] - Y0
    dY = project(Y0.reshape(-1, NS), dY.reshape(-1, NS), A, proj_eps).reshape(dY.shape)
    Tchem = _interior(o, "T").copy()
    for n, v in keep.items():
        o.view(n)[...] = v
    return dY, Tchem, nsub


def adaptive_step(o, dt, atoms, **kw):
    """The split cell update: CS += RHS and decode (Update_after_Adv,
    src/Flowfield.cpp:1140-1157), the increment at that state, CS_s = rho
    max(Y_s + dY_s, 0), decode from Tchem."""
    NS = o.NS
    o.update_after_adv()
    dY, Tchem, nsub = increment(o, dt, atoms, **kw)
    c = _interior(o, "CS")
    D = c[..., :NS].sum(-1)
    Y = c[..., :NS] / D[..., None]
    c[..., :NS] = np.maximum(D[..., None] * (Y + dY), 0.0)
    _interior(o, "T")[...] = Tchem
    o.update_after_cs()
    return nsub
