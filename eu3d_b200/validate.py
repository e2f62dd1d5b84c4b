"""Coupled validation of the learned chemistry surrogate: the oblique
detonation with the 3D benchmark case's cells -- in 2D, and in 3D with a
spanwise slice of the benchmark domain -- run with the surrogate, with the
FP64 adaptive integrator it was trained on and with the plain FP64 IMEX
integrator; peak temperature and detonation-front position compared."""
from __future__ import annotations

import numpy as np


def front_position(T, thr=1800.0):
    """Detonation-front position per line along x (axis 0) of a temperature
    field (ni, ...): the first x, in cells and linearly interpolated, where T
    exceeds thr; NaN where no cell does or the first cell already does."""
    T = np.asarray(T, dtype=np.float64)
    hot = T > thr
    k = np.argmax(hot, axis=0)
    f = np.full(k.shape, np.nan)
    ok = hot.any(axis=0) & (k > 0)
    idx = np.nonzero(ok)
    i = k[idx]
    a, b = T[(i - 1,) + idx], T[(i,) + idx]
    f[idx] = i - 1 + (thr - a) / (b - a)
    return f


def accuracy_2d(mech, model, steps, ni=512, nj=256, cfl=0.5):
    """Coupled 2D ODW (the 3D case's cells) with the surrogate, the FP64
    adaptive integrator (its teacher) and the plain FP64 IMEX integrator:
    peak T and detonation-front position (first x where T > 1800 K, per row)."""
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import odw_case, setup_odw
    res, stats = {}, {}
    for name, react in (("adaptive", gpu.REACT_ADAPTIVE), ("surrogate", gpu.REACT_SURROGATE), ("imex", gpu.REACT_IMEX)):
        c = odw_case(mech, ni, nj, 2)
        d = gpu.DeviceFlowfield(mech, c.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=32)
        setup_odw(d, c)
        d.set_elements(S.atoms_matrix(mech))
        if react == gpu.REACT_SURROGATE:
            model.attach(d, 97)
        d.run(steps, react=react, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=cfl, final_time=1.0)
        d.synchronize()
        res[name] = d.download("T")[2:-2, 2:-2, 2].copy()
        stats[name] = d.status()
        d.close()

    fa = front_position(res["adaptive"])
    out = {"case": f"2D ODW {ni}x{nj} (the 3D case's cells), SSP-RK2, CFL {cfl}, {steps} steps",
           "peak_T_adaptive": float(np.nanmax(res["adaptive"]))}
    for name in ("surrogate", "imex"):
        fx = front_position(res[name])
        both = np.isfinite(fa) & np.isfinite(fx)
        d = np.abs(fa - fx)[both]
        st = stats[name]
        out[name] = {"peak_T": float(np.nanmax(res[name])),
                     "peak_T_rel_err_vs_adaptive": float(abs(np.nanmax(res[name]) / np.nanmax(res["adaptive"]) - 1)),
                     "mean_abs_dT_K": float(np.nanmean(np.abs(res[name] - res["adaptive"]))),
                     "front_rows_both": int(both.sum()), "front_rows_one_only": int((np.isfinite(fa) ^ np.isfinite(fx)).sum()),
                     "front_abs_diff_cells_median": float(np.median(d)) if d.size else None,
                     "front_abs_diff_cells_max": float(d.max()) if d.size else None,
                     "nonfinite_cells": st["nonfinite_cells"]}
        if name == "surrogate":
            tot = st["surrogate_cells"] + st["surrogate_fallback"]
            out[name]["fallback_frac"] = st["surrogate_fallback"] / max(tot, 1)
            out[name]["audit_max_dT_K"] = st["surrogate_audit_max_dT"]
    return out


def accuracy_3d(mech, model, steps, ni=512, nj=256, nk=16, cfl=0.5):
    """The same comparison in 3D: the benchmark's x-y extent and cells with nk
    spanwise cells and the seeded spanwise inflow perturbation; fronts per
    (y, z) column."""
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import odw_case, setup_odw
    res, stats = {}, {}
    for name, react in (("adaptive", gpu.REACT_ADAPTIVE), ("surrogate", gpu.REACT_SURROGATE), ("imex", gpu.REACT_IMEX)):
        c = odw_case(mech, ni, nj, nk)
        d = gpu.DeviceFlowfield(mech, c.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=32)
        setup_odw(d, c)
        d.set_elements(S.atoms_matrix(mech))
        if react == gpu.REACT_SURROGATE:
            model.attach(d, 97)
        d.run(steps, react=react, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=cfl, final_time=1.0)
        d.synchronize()
        res[name] = d.download("T")[2:-2, 2:-2, 2:-2].copy()
        stats[name] = d.status()
        d.close()

    fa = front_position(res["adaptive"])
    extent = "the benchmark's full grid" if (ni, nj, nk) == (512, 256, 256) else "the benchmark's cells, spanwise slice"
    out = {"case": f"3D ODW {ni}x{nj}x{nk} ({extent}), SSP-RK2, CFL {cfl}, {steps} steps",
           "peak_T_adaptive": float(np.nanmax(res["adaptive"]))}
    for name in ("surrogate", "imex"):
        fx = front_position(res[name])
        both = np.isfinite(fa) & np.isfinite(fx)
        dd = np.abs(fa - fx)[both]
        st = stats[name]
        out[name] = {"peak_T": float(np.nanmax(res[name])),
                     "peak_T_rel_err_vs_adaptive": float(abs(np.nanmax(res[name]) / np.nanmax(res["adaptive"]) - 1)),
                     "mean_abs_dT_K": float(np.nanmean(np.abs(res[name] - res["adaptive"]))),
                     "front_columns_both": int(both.sum()),
                     "front_columns_one_only": int((np.isfinite(fa) ^ np.isfinite(fx)).sum()),
                     "front_abs_diff_cells_median": float(np.median(dd)) if dd.size else None,
                     "front_abs_diff_cells_p95": float(np.percentile(dd, 95)) if dd.size else None,
                     "front_abs_diff_cells_max": float(dd.max()) if dd.size else None,
                     "nonfinite_cells": st["nonfinite_cells"]}
        if name == "surrogate":
            tot = st["surrogate_cells"] + st["surrogate_fallback"]
            out[name]["fallback_frac"] = st["surrogate_fallback"] / max(tot, 1)
            out[name]["audit_max_dT_K"] = st["surrogate_audit_max_dT"]
    return out
