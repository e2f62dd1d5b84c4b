"""Coupled accuracy of the mixed-precision and learned-chemistry paths on
the oblique detonation, against the all-FP64 run.

The reference run is FP64 throughout: FP64 reconstruction, AUSM and flux
residual (flux_bits = 64), FP64 state, and the FP64 adaptive integrator --
the one FP64 chemistry integrator that stays finite through the ignition of
these cases, and the surrogate's teacher.  Against it, from the same initial
state and for the same steps:

  adaptive_fp32  FP32 reconstruction / AUSM / residual, FP64 state, the same
                 FP64 adaptive chemistry (the cost of the FP32 flux alone);
  surrogate      FP32 flux, learned chemistry with its FP64 fallback and the
                 frozen-chemistry gate (the benchmark's form);
  imex           FP32 flux, the reference's one-step FP64 IMEX (the plain
                 integrator the benchmark compares with).

Per run and quantity, on the fluid cells (the wedge's solid cells are not part
of the flow): rho, p and T by their pointwise relative error |x - x_ref| /
|x_ref|; each mass fraction Y_k by |Y_k - Y_k,ref| / max over the fluid cells
of Y_k,ref (each species against its own scale, so that radicals count as
much as N2); each as its maximum and 99th percentile.  Beside them the peak
temperature and the detonation-front position (first x where T > 1800 K, per
row in 2D and per (y, z) column in 3D) against the reference's."""
from __future__ import annotations

from typing import Optional

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


def fluid_mask(case):
    """(ni, nj, nk) True on the cells outside the case's wedge."""
    g = case.grid
    x = g.xnode[g.bc:-g.bc][:, None, None]
    y = g.ynode[g.bc:-g.bc][None, :, None]
    w = case.wedge
    solid = (x > w[0]) & ((y - w[1]) < (x - w[0]) * w[2])
    return np.broadcast_to(~solid, (g.ni, g.nj, g.nk))


RUNS = {
    # name: (chemistry, flux bits)
    "fp64": ("adaptive", 64),
    "adaptive_fp32": ("adaptive", 32),
    "surrogate": ("surrogate", 32),
    "imex": ("imex", 32),
}


def run_odw(mech, model, name, steps, ni, nj, nk, cfl, gate=None, audit=97):
    """One coupled ODW run from the fresh free stream: interior fields T, P, D
    and Yi (host FP64) and the final status."""
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import odw_case, setup_odw
    chem, bits = RUNS[name]
    react = {"adaptive": gpu.REACT_ADAPTIVE, "surrogate": gpu.REACT_SURROGATE, "imex": gpu.REACT_IMEX}[chem]
    c = odw_case(mech, ni, nj, nk)
    d = gpu.DeviceFlowfield(mech, c.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=bits)
    setup_odw(d, c)
    d.set_elements(S.atoms_matrix(mech))
    sur = model.attach(d, audit, gate=S.GATE if gate is None else gate) if react == gpu.REACT_SURROGATE else None
    d.run(steps, react=react, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=cfl, final_time=1.0)
    d.synchronize()
    b = c.grid.bc
    out = {n: d.download(n)[b:-b, b:-b, b:-b].copy() for n in ("T", "P", "D", "Yi")}
    st = d.status()
    if sur is not None:
        d.set_surrogate(None)
        sur.close()
    d.close()
    return out, st, c


def _stats(x):
    x = np.asarray(x, dtype=np.float64)
    return {"max": float(np.max(x)), "p99": float(np.percentile(x, 99))}


def field_errors(ref, run, fluid, species):
    """Pointwise errors of run against ref on the fluid cells (see the module
    docstring for the measures)."""
    out = {}
    for n, key in (("rho", "D"), ("p", "P"), ("T", "T")):
        r, x = ref[key][fluid], run[key][fluid]
        out[n] = _stats(np.abs(x - r) / np.abs(r))
    Yr, Yx = ref["Yi"][fluid], run["Yi"][fluid]
    for s, name in enumerate(species):
        scale = float(np.max(np.abs(Yr[:, s])))
        out[f"Y_{name}"] = _stats(np.abs(Yx[:, s] - Yr[:, s]) / max(scale, 1e-300))
    return out


def _front_stats(Tref, Tx, per):
    fa, fx = front_position(Tref), front_position(Tx)
    both = np.isfinite(fa) & np.isfinite(fx)
    d = np.abs(fa - fx)[both]
    return {f"front_{per}_both": int(both.sum()), f"front_{per}_one_only": int((np.isfinite(fa) ^ np.isfinite(fx)).sum()),
            "front_abs_diff_cells_median": float(np.median(d)) if d.size else None,
            "front_abs_diff_cells_p95": float(np.percentile(d, 95)) if d.size else None,
            "front_abs_diff_cells_max": float(d.max()) if d.size else None,
            f"front_{per}_over_1_cell": int((d > 1.0).sum())}


def accuracy(mech, model, steps, ni=512, nj=256, nk=16, cfl=0.5, runs=("adaptive_fp32", "surrogate", "imex"),
             gate: Optional[dict] = None):
    """The comparison table of the module docstring on an ni x nj x nk ODW
    (nk = 2: the 2D case, fronts per row; otherwise per (y, z) column)."""
    from eu3d_b200 import surrogate as S
    ref, st_ref, case = run_odw(mech, model, "fp64", steps, ni, nj, nk, cfl, gate)
    fluid = fluid_mask(case)
    two_d = nk == 2
    sl = (slice(None), slice(None), 0) if two_d else (slice(None), slice(None), slice(None))
    Tref = ref["T"][sl]
    peak_ref = float(np.nanmax(np.where(fluid[sl], Tref, np.nan)))
    if two_d:
        extent = "2D ODW (the 3D case's cells)"
    elif (ni, nj, nk) == (512, 256, 256):
        extent = "3D ODW, the benchmark's full grid"
    else:
        extent = "3D ODW, the benchmark's cells, spanwise slice"
    out = {"case": f"{extent} {ni}x{nj}x{nk}, SSP-RK2, CFL {cfl}, {steps} steps from the fresh free stream",
           "reference": "all-FP64 run: FP64 reconstruction, AUSM and residual, FP64 state, FP64 adaptive chemistry",
           "measures": "rho, p, T: pointwise |x - x_ref| / |x_ref|; Y_k: |Y_k - Y_k,ref| / max Y_k,ref; "
                       "max and p99 over the fluid cells",
           "peak_T_reference": peak_ref, "fluid_cells": int(fluid.sum()),
           "reference_nonfinite_cells": st_ref["nonfinite_cells"]}
    for name in runs:
        run, st, _ = run_odw(mech, model, name, steps, ni, nj, nk, cfl, gate)
        Tx = run["T"][sl]
        peak = float(np.nanmax(np.where(fluid[sl], Tx, np.nan)))
        r = {"peak_T": peak, "peak_T_rel_err": abs(peak / peak_ref - 1.0),
             "errors": field_errors(ref, run, fluid, mech.species),
             "mean_abs_dT_K": float(np.mean(np.abs(run["T"][fluid] - ref["T"][fluid]))),
             "nonfinite_cells": st["nonfinite_cells"]}
        r.update(_front_stats(Tref, Tx, "rows" if two_d else "columns"))
        if name == "surrogate":
            tot = st["surrogate_cells"] + st["surrogate_fallback"] + st["surrogate_audited"] + st["surrogate_frozen"]
            r["fallback_frac"] = st["surrogate_fallback"] / max(tot, 1)
            r["frozen_frac"] = st["surrogate_frozen"] / max(tot, 1)
            r["audit_max_dT_K"] = st["surrogate_audit_max_dT"]
            r["frozen_audit_max_dT_K"] = st["frozen_audit_max_dT"]
            r["gate"] = {k: (list(v) if isinstance(v, tuple) else v) for k, v in (gate or S.GATE).items()}
        out[name] = r
        del run
    return out


def accuracy_2d(mech, model, steps, ni=512, nj=256, cfl=0.5, **kw):
    """accuracy() on the 2D ODW with the 3D case's cells."""
    return accuracy(mech, model, steps, ni, nj, 2, cfl, **kw)


def accuracy_3d(mech, model, steps, ni=512, nj=256, nk=16, cfl=0.5, **kw):
    """accuracy() in 3D: the benchmark's x-y extent and cells with nk spanwise
    cells and the seeded spanwise inflow perturbation."""
    return accuracy(mech, model, steps, ni, nj, nk, cfl, **kw)


def main(argv=None):
    """python -m eu3d_b200.validate [--grid 512,256,256] [--steps 2000] --out result.json"""
    import argparse
    import json
    from eu3d_b200 import surrogate as S
    from eu3d_b200.readers import load_h2_ja919
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="512,256,256")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--cfl", type=float, default=0.5)
    ap.add_argument("--model", default=S.DEFAULT_MODEL)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    ni, nj, nk = (int(x) for x in a.grid.split(","))
    res = accuracy(load_h2_ja919(), S.SurrogateModel.load(a.model), a.steps, ni, nj, nk, a.cfl)
    txt = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)
    print(txt)


if __name__ == "__main__":
    main()
