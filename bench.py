#!/usr/bin/env python3
"""Headline benchmark of the EU3D B200 hot path.

Workload (one GPU): 3D oblique detonation, 512 x 256 x 256 interior cells
(33.5 M), stoichiometric H2-air at Mach 7, 0.1 atm, 300 K with a seeded 1 %
inflow density perturbation, 25 degree wedge from x = 0.1 L, L = 0.2 m.
MUSCL_2/minmod + AUSM with FP32 reconstruction and FP64 state, SSP-RK2 time
advance, CFL 0.5, every step one CUDA-graph replay of CFL -> ghost fill ->
flux sweeps -> chemistry + decode.  The timed state is a developed flow: the
2D case with the same cells advanced with the FP64 adaptive integrator and
extruded along z.  Inputs (~12 GB of state) are far larger than L2 (126 MB),
so no flush is needed between steps.

Metric: Mcell-steps/s = interior cells x steps / device time, with the
learned chemistry surrogate (value); the same steps with the plain FP64 IMEX
integrator and with the FP64 adaptive integrator (the surrogate's teacher)
are timed on the same GPU and state and reported beside it, with the
coupled accuracy of a 2D run (peak T, detonation front) against the FP64
runs.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

--gpus N (under torchrun, one rank per GPU): the same case split into N x
slabs (strong scaling), halos exchanged by NCCL send/recv and dt reduced by
an all-reduce MIN on each handle's stream (eu3d_b200.slabs); the time is the
max over ranks and the value counts the whole case's cells.

--impl reference times the reference's own CPU solver (oracle/_ref, the
reference sources compiled unmodified) on bounded samples of the same
workload on every host core and prints the same JSON line.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s, 3D ODW: NN chemistry vs FP64 integrator, same GPU, ≤1% T err"
UNIT = "Mcell-steps/s"
CFL = 0.5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", default="512,256,256")
    ap.add_argument("--flux-bits", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=2000)
    ap.add_argument("--accuracy-full", action="store_true",
                    help="also compare on the benchmark's full grid (about 2.5 more minutes)")
    ap.add_argument("--develop", type=int, default=1500, help="2D steps that develop the timed state")
    ap.add_argument("--model", default=os.path.join(ROOT, "eu3d_b200", "data", "sur_h2_ja919.npz"))
    return ap.parse_args()


# ------------------------------------------------------------ CPU baseline
def _ref_slab_worker(args):
    """One host process: the reference solver on a slab of the workload."""
    ni, nj, nk, steps, warm, use_ref = args
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    from eu3d_b200.cases import complete_state, odw_case
    from eu3d_b200.readers import load_h2_ja919
    import pyoracle

    mech = load_h2_ja919()
    case = odw_case(mech, ni, nj, nk, L=0.2 * (ni - 1) / 511.0)
    g = case.grid
    if use_ref:
        rc = pyoracle.RefCase(mech, g, fixed=False)
    else:
        rc = pyoracle.Oracle(mech, g, 0x1FF)
    NI, NJ, NK = g.ni + 4, g.nj + 4, g.nk + 4
    shp = (NI, NJ, NK)
    Y = np.broadcast_to(case.Y, shp + (mech.NS,))
    st = complete_state(mech, np.full(shp, case.P), np.full(shp, case.T), np.full(shp, case.U), np.zeros(shp),
                        np.zeros(shp), Y)
    for n, v in (("U", case.U), ("V", 0.0), ("W", 0.0), ("P", case.P), ("T", case.T)):
        rc.view(n)[...] = v
    for n in ("D", "H", "E", "Gamma", "C", "Rgas", "Cp"):
        rc.view(n)[...] = st[n]
    rc.view("Yi")[...] = Y
    rc.view("CS")[...] = st["CS"]
    rc.view("Di")[...] = st["CS"][..., :mech.NS]
    rc.view("Mc")[...] = st["CS"][..., :mech.NS] / mech.mw * 1000
    f = case.inflow
    for n, k in (("Uint", "U"), ("Vint", "V"), ("Wint", "W"), ("Pint", "P"), ("Dint", "D"), ("Tint", "T"),
                 ("Hint", "H"), ("Eint", "E"), ("Gint", "G")):
        rc.view(n)[...] = f[k]
    rc.view("Yint")[...] = f["Y"]
    rc.partial_t()

    def one():
        if use_ref:
            rc.cfl(CFL, 1.0)
            rc.boundary(1)
            rc.advection(0, 1)
            rc.imex()
        else:
            rc.step(1, 0, 0, 1, CFL, 1.0, 1)

    for _ in range(warm):
        one()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    t1 = time.perf_counter()
    return g.ni * g.nj * g.nk * steps, t1 - t0


def cpu_baseline(steps=3, warm=1, slab=(64, 32, 8), procs=None):
    """Reference CPU solver on `procs` concurrent slab processes (one per
    host core): the aggregate rate of an MPI run without halo cost."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    use_ref = pyoracle.RefCase.available()
    if not use_ref and not os.path.exists(pyoracle.ORACLE_SO):
        pyoracle.build_oracle()
    procs = procs or (os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_slab_worker, [(slab[0], slab[1], slab[2], steps, warm, use_ref)] * procs)
    cells = sum(r[0] for r in res)
    tmax = max(r[1] for r in res)
    value = cells / tmax / 1e6
    return {"value": value, "unit": UNIT, "cores": procs, "kind": "reference" if use_ref else "port",
            "sample": f"{procs} concurrent processes x {slab[0]}x{slab[1]}x{slab[2]}-cell slabs of the ODW inflow "
                      f"state, ODM ghost fill, EE + MUSCL_2/AUSM + IMEX, CFL {CFL}, {steps} timed steps after "
                      f"{warm} warm-up; {'reference sources built unmodified (oracle/_ref)' if use_ref else 'C restatement'}",
            "seconds": tmax}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.p = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                      stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.fh.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        load = [x for x in sm if x > 0.5 * (max(mx) if mx else 1)] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ------------------------------------------------------------------ ours
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def kernel_work(pb=4):
    """Algorithmic work per cell and launch of the kernels a roofline may be
    quoted for; pb = bytes of a primitive and of a residual value (4 with
    the FP32 flux path, 8 with the FP64 one)."""
    R = 13 * pb  # the flux residual of a cell
    return {
        # flux + residual: 16 primitives in, 13 residuals out
        "advection": ("hbm", 16 * pb + R),
        # decode after the flux update: 13 FP64 state + RHS in, state + T, E + 16 primitives out
        "cell_adv": ("hbm", 13 * 8 * 2 + R + 2 * 8 * 2 + 16 * pb),
        # surrogate apply: state + T, E + 10 FP32 outputs in; 9 species + T, E + 16 primitives out
        "sur_apply": ("hbm", 13 * 8 + 16 + 40 + 9 * 8 + 16 + 16 * pb),
        # MLP 12 -> 3 x 128 -> 10 forward: 2 (16 128 + 2 128 128 + 128 16) FLOP
        "sur_mlp": ("tensor", 2 * (16 * 128 + 2 * 128 * 128 + 128 * 16)),
        # the network and its apply in one kernel: the network's FLOPs
        "sur_mlp_apply": ("tensor", 2 * (16 * 128 + 2 * 128 * 128 + 128 * 16)),
        "cell_imex": ("hbm", 13 * 8 * 2 + R + 2 * 8 * 2 + 16 * pb),
        # stage 1: CS^n and RHS in, the stage state out (CS^n stays in place)
        "cell_rk1": ("hbm", 13 * 8 * 2 + R + 2 * 8 * 2 + 16 * pb),
        # stage 2: CS^n, the stage state and RHS in, CS out
        "cell_rk2": ("hbm", 13 * 8 * 3 + R + 2 * 8 * 2 + 16 * pb),
    }


KERNEL_WORK = kernel_work(4)  # the default FP32 flux path


def timed_steps(dev, step, K, W, torch, world, dist, clocks=False, local=0):
    """K steps timed with CUDA events on the handle's stream (max over ranks).
    step: a callable (one step) or eu3d_step's keyword arguments."""
    one = step if callable(step) else (lambda: dev.step(**step))
    for _ in range(W):
        one()
    dev.synchronize()
    stream = torch.cuda.ExternalStream(dev.stream)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local) if clocks else None
    if clk:
        clk.__enter__()
    ev0.record(stream)
    for _ in range(K):
        one()
    ev1.record(stream)
    dev.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, (clk.summary() if clk else None)


def profiled(dev, step, K):
    """Per-kernel CUDA-event durations over K steps (no graph)."""
    one = step if callable(step) else (lambda: dev.step(**step))
    dev.profile(True)
    for _ in range(K):
        one()
    prof = dev.profile_read()
    dev.profile(False)
    return prof


def roofline(prof, units, hbm, tflops, src, pb=4, kernel=None):
    """Roofline of one kernel -- by default the one with the largest share of
    the step among those with a stated algorithmic work (pb: bytes of a
    primitive / residual).  units: kernel -> cells whose work a launch must do
    (the fluid cells for the flux and cell kernels, which leave the wedge's
    solid cells out; the listed cells for the network)."""
    kw = kernel_work(pb)
    cand = [(k, v) for k, v in prof.items() if k in kw]
    k, v = (kernel, prof[kernel]) if kernel else max(cand, key=lambda kv: kv[1][0])
    avg_ms = v[0] / v[1]
    bound, work = kw[k]
    cells = units[k]
    if bound == "hbm":
        ach = work * cells / (avg_ms * 1e-3) / 1e9
        return {"bound": "hbm", "kernel": k, "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": TRAFFIC_PER_CELL[k] * cells if k in TRAFFIC_PER_CELL and pb == 4 else None,
                "traffic_note": TRAFFIC_NOTE.get(k),
                "per_cell": f"{work} B", "cells": cells, "avg_ms": avg_ms, "peak_source": src,
                "note": f"achieved = {work} B/cell x {cells} fluid cells / average launch of {k}; frac of {src} peak "
                        + ("(MEASURED_PEAKS.json hbm_gbs)" if src == "measured"
                           else "(MEASURED_PEAKS.json absent: the pool's earlier copy measurement, 6650 GB/s)")}
    ach = work * cells / (avg_ms * 1e-3) / 1e12
    return {"bound": "tensor", "kernel": k, "achieved": ach, "peak": tflops, "unit": "TFLOP/s", "frac": ach / tflops,
            "traffic": TRAFFIC_PER_CELL[k] * cells if k in TRAFFIC_PER_CELL and pb == 4 else None,
            "per_cell": f"{work} FLOP", "cells": cells, "avg_ms": avg_ms, "peak_source": src,
            "note": f"achieved = {work} FLOP/cell x {cells} network cells / average launch of {k}; frac of {src} "
                    "peak " + ("(MEASURED_PEAKS.json bf16_tflops)" if src == "measured"
                               else "(MEASURED_PEAKS.json absent: the pool's earlier cuBLAS measurement, 1590 TFLOP/s)")}


# DRAM bytes per cell of a launch (ncu dram__bytes_read.sum + dram__bytes_write.sum
# of one launch on the 256 x 128 x 64 ODW, 2.10 M cells, with the benchmark's 64
# z planes per block: the full 33.5 M-cell case is too large to capture under
# the profiling rule), scaled to a launch by cells; the flux kernel's traffic
# grows with cells (one pass; the tile halos add 3 % of reads)
TRAFFIC_PER_CELL = {"advection": (168.854016e6 + 81.255936e6) / 2097152}
TRAFFIC_NOTE = {"advection": "ncu DRAM bytes of one launch on a 2.10 M-cell case, per cell, times the fluid cells"}


def fluid_cells(case, i0=0, n_loc=None):
    """Interior cells of the case (or of the x slab i0 .. i0 + n_loc) outside its wedge."""
    g = case.grid
    x = g.xnode[g.bc:-g.bc][i0:i0 + (n_loc or g.ni)][:, None]
    y = g.ynode[g.bc:-g.bc][None, :]
    w = case.wedge
    solid = (x > w[0]) & ((y - w[1]) < (x - w[0]) * w[2])
    return int((~solid).sum()) * g.nk


# kernels of the step that make up its chemistry (the rest: ghost fills, CFL,
# flux sweeps and stage updates)
CHEM_KERNELS = {"cell_imex", "cell_adapt", "sur_gate", "sur_mlp", "sur_apply", "sur_fallback", "sur_mlp_apply"}


def developed_state(mech, ni, nj, nk, steps2d, seed):
    """A developed 3D ODW state: the 2D case (same cells) advanced steps2d
    SSP-RK2 steps with the FP64 adaptive integrator, extruded along z, with
    the 3D case's seeded inflow perturbation."""
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import extrude_state, odw_case, setup_odw
    c2 = odw_case(mech, ni, nj, 2, seed=seed)
    d2 = gpu.DeviceFlowfield(mech, c2.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=32)
    setup_odw(d2, c2)
    d2.set_elements(S.atoms_matrix(mech))
    d2.run(steps2d, react=gpu.REACT_ADAPTIVE, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=CFL, final_time=1.0)
    d2.synchronize()
    c3 = odw_case(mech, ni, nj, nk, seed=seed)
    return d2, c3


def run_ours(a, rank, world, local):
    import torch
    import torch.distributed as dist

    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import extrude_state, setup_odw
    from eu3d_b200.readers import load_h2_ja919

    from eu3d_b200.slabs import DeviceSlab, SlabRun, StepSpec, TorchTransport, slab_extents, slab_grid

    torch.cuda.set_device(local)
    ni, nj, nk = (int(x) for x in a.grid.split(","))
    mech = load_h2_ja919()
    cells = ni * nj * nk  # the whole case; N > 1 splits it into x slabs
    model = S.SurrogateModel.load(a.model)
    d2, case = developed_state(mech, ni, nj, nk, a.develop, seed=0)
    i0, n_loc = slab_extents(ni, world)[rank] if world > 1 else (0, ni)
    grid = slab_grid(case.grid, i0, n_loc) if world > 1 else case.grid
    dev = gpu.DeviceFlowfield(mech, grid, quirks=gpu.QUIRKS_FIXED, flux_bits=a.flux_bits, device=local)
    setup_odw(dev, case)
    dev.set_elements(S.atoms_matrix(mech))
    model.attach(dev, 4099, gate=S.GATE)
    fluid = fluid_cells(case, i0, n_loc) if world > 1 else fluid_cells(case)

    def reset():
        extrude_state(d2, dev, i0=i0)
        dev.set_time(0.0)
        dev.reset_status()

    base = dict(type_=0, timeadv=gpu.ADV_SSPRK2, diff=gpu.DIFF_MUSCL2, bc_kind=gpu.BC_ODM, cfl=CFL, final_time=1.0)
    forms = {"surrogate": gpu.REACT_SURROGATE, "imex": gpu.REACT_IMEX, "adaptive": gpu.REACT_ADAPTIVE}
    # N > 1: the slab of this rank, halos by NCCL send/recv and dt by an
    # all-reduce MIN on the handle's stream (eu3d_b200.slabs); N = 1: eu3d_step
    run = SlabRun([DeviceSlab(dev, rank, world, wedge=True)], TorchTransport()) if world > 1 else None

    def stepper(step):
        if run is None:
            return step
        spec = StepSpec(**step)
        return lambda: run.step(spec)

    W = max(a.warmup, 3)
    timing, profs, statuses, clocks = {}, {}, {}, None
    for name, react in forms.items():
        reset()
        step = stepper(dict(base, react=react))
        ms, clk = timed_steps(dev, step, a.steps, W, torch, world, dist, clocks=(name == "surrogate"), local=local)
        if clk:
            clocks = clk
        statuses[name] = dev.status()
        timing[name] = ms
        profs[name] = profiled(dev, step, a.steps)
    hbm, tfl, src = peaks()
    prof = profs["surrogate"]
    st = statuses["surrogate"]
    # cells one launch must process: the fluid cells of this rank; the network
    # takes the cells the frozen-chemistry gate listed, per step
    steps_run = a.steps + W
    net_cells = (st["surrogate_cells"] + st["surrogate_fallback"] + st["surrogate_audited"]) // max(steps_run, 1)
    units = {k: fluid for k in kernel_work(4)}
    units["sur_mlp"] = units["sur_mlp_apply"] = net_cells
    pb = 4 if a.flux_bits == 32 else 8
    rf = roofline(prof, units, hbm, tfl, src, pb=pb)
    rf_more = {k: {f: r[f] for f in ("achieved", "unit", "frac", "avg_ms", "cells", "per_cell")}
               for k, r in ((k, roofline(prof, units, hbm, tfl, src, pb=pb, kernel=k))
                            for k in ("advection", "cell_rk1", "cell_rk2", "sur_mlp", "sur_apply") if k in prof)}
    ms = timing["surrogate"]
    value = cells * a.steps / (ms * 1e-3) / 1e6
    integ = {k: cells * a.steps / (timing[k] * 1e-3) / 1e6 for k in ("imex", "adaptive")}
    tot = st["surrogate_cells"] + st["surrogate_fallback"] + st["surrogate_audited"] + st["surrogate_frozen"]
    # per-step split from the per-kernel events: chemistry and the rest
    split = {}
    for f, pr in profs.items():
        chem = sum(v[0] for k, v in pr.items() if k in CHEM_KERNELS) / a.steps
        rest = sum(v[0] for k, v in pr.items() if k not in CHEM_KERNELS) / a.steps
        split[f] = {"chemistry_ms": chem, "non_chemistry_ms": rest}
    nc = split["imex"]["non_chemistry_ms"]
    amdahl = (nc + split["imex"]["chemistry_ms"]) / nc
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": W,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "bf16 (network) + f64 (state, decode, fallback integrator)", "data": "synthetic",
        "config": {"workload": workload_name(ni, nj, nk),
                   "cells": cells, "cells_per_gpu": n_loc * nj * nk,
                   "fluid_cells_per_gpu": fluid,
                   "cell_count_note": "value counts every interior cell of the grid, the wedge's solid ones "
                                      "included; the kernels skip solid cells (and the flux kernel all-solid "
                                      "tiles), so per fluid cell the rate is value x cells / fluid cells",
                   "chemistry": "learned surrogate (BF16 tcgen05 MLP) with FP64 adaptive fallback; frozen-chemistry "
                                "gate: cells below 600 K with radicals <= 1e-6 skip the network",
                   "flux": f"MUSCL_2/minmod + AUSM, FP{a.flux_bits} reconstruction, FP64 state",
                   "time": f"SSP-RK2, CFL {CFL}",
                   "state": f"developed: 2D case advanced {a.develop} steps with the FP64 adaptive integrator, "
                            f"extruded along z",
                   "parallelism": (f"{world} x slabs of {n_loc} cells (NCCL halo send/recv, all-reduce MIN of dt)"
                                   if world > 1 else "1 GPU"),
                   "l2": "state ~12 GB per GPU >> 126 MB L2 (no flush needed)",
                   "graph": "one CUDA graph per step" if world == 1 else "per-op launches (halo exchanges between)"},
        "integrator": {"imex_value": integ["imex"], "adaptive_value": integ["adaptive"],
                       "ratio_vs_imex": value / integ["imex"], "ratio_vs_adaptive": value / integ["adaptive"],
                       "ms_per_step": {k: timing[k] / a.steps for k in timing},
                       "split_ms_per_step": split,
                       "amdahl_bound_vs_imex": amdahl,
                       "amdahl_note": "the IMEX step over its non-chemistry part: the ratio a free chemistry would "
                                      "reach against plain IMEX with the same flux, stage and boundary kernels",
                       "note": "same GPU, same state and step; imex = the reference's one-step FP64 IMEX, "
                               "adaptive = FP64 adaptive integrator (the surrogate's teacher and fallback)"},
        "surrogate": {"fallback_frac": st["surrogate_fallback"] / max(tot, 1),
                      "frozen_frac": st["surrogate_frozen"] / max(tot, 1), "rejects": st["surrogate_rejects"],
                      "audited": st["surrogate_audited"], "audit_max_dT_K": st["surrogate_audit_max_dT"],
                      "frozen_audited": st["frozen_audited"], "frozen_audit_max_dT_K": st["frozen_audit_max_dT"],
                      "model": os.path.relpath(a.model, ROOT)},
        "gpu_launches": int(sum(v[1] for v in prof.values())),
        "kernels": {f: {k: {"ms_avg": v[0] / v[1], "share": v[0] / sum(x[0] for x in profs[f].values()),
                            "launches": v[1]} for k, v in sorted(profs[f].items(), key=lambda kv: -kv[1][0])}
                    for f in profs},
        "roofline": rf,
        "roofline_other_kernels": rf_more,
        "status": {k: st[k] for k in ("nonfinite_cells", "newton_capped", "dt", "time")},
    }
    if clocks:
        out["clocks"] = clocks
    if not a.no_accuracy and rank == 0:
        # errors of the FP32-flux, surrogate and IMEX forms against the all-FP64 run
        from eu3d_b200.validate import accuracy_2d, accuracy_3d
        out["accuracy"] = accuracy_2d(mech, model, a.accuracy_steps, cfl=CFL)
        out["accuracy_3d"] = accuracy_3d(mech, model, a.accuracy_steps, nk=16, cfl=CFL)
        if a.accuracy_full:
            out["accuracy_full_grid"] = accuracy_3d(mech, model, a.accuracy_steps, ni, nj, nk, cfl=CFL)
        else:
            out["accuracy_full_grid"] = ("not run by default (about five minutes): python -m eu3d_b200.validate "
                                         "--grid 512,256,256, or bench.py --accuracy-full")
    if not a.no_e2e:
        reset()
        out["e2e"] = run_e2e(dev, stepper(dict(base, react=gpu.REACT_SURROGATE)), a.steps, cells, torch, world, dist)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    dev.close()
    d2.close()
    return out


def run_e2e(dev, step, K, cells, torch, world=1, dist=None):
    """The same metric through the C ABI with host buffers: upload CS, T, E
    from pinned host memory, decode, K steps each followed by a status read,
    download CS and T -- all inside the timed region (N > 1: each rank its
    slab, the time the max over ranks)."""
    one = step if callable(step) else (lambda: dev.step(**step))
    shapes = {n: dev.shape(n) for n in ("CS", "T", "E")}
    host = {n: torch.empty(s, dtype=torch.float64, pin_memory=True).numpy() for n, s in shapes.items()}
    for n in host:
        dev.download(n, host[n])
    stream = torch.cuda.ExternalStream(dev.stream)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for n in ("CS", "T", "E"):
        dev.upload(n, host[n])
    dev.update_after_cs()
    for _ in range(K):
        one()
        dev.status()
    dev.download("CS", host["CS"])
    dev.download("T", host["T"])
    ev1.record(stream)
    dev.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    h2d = sum(host[n].nbytes for n in ("CS", "T", "E"))
    d2h = host["CS"].nbytes + host["T"].nbytes + K * 96
    return {"value": cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": h2d // K,
            "d2h_bytes_per_step": d2h // K, "ms": ms,
            "protocol": "upload CS,T,E (pinned) + decode, K eu3d_step calls (surrogate chemistry) each with a status "
                        "read, download CS,T; the state stays on the device between steps (the drop-in's design), "
                        "so the host copies are amortised over the K steps and the value depends on K"}


def workload_name(ni, nj, nk):
    return (f"3D oblique detonation {ni}x{nj}x{nk} (ODW, Mach 7 H2-air 0.1 atm 300 K, 25 deg wedge, "
            f"1 % seeded inflow density perturbation)")


def run_reference(a, rank, world):
    if rank != 0:
        return None
    ni, nj, nk = (int(x) for x in a.grid.split(","))
    vals = []
    for _ in range(max(a.warmup, 0)):
        cpu_baseline(steps=1, warm=0)
    for _ in range(a.steps):
        vals.append(cpu_baseline(steps=2, warm=1))
    v = float(np.median([x["value"] for x in vals]))
    cb = dict(vals[0])
    cb["value"] = v
    return {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": workload_name(ni, nj, nk), "cells": ni * nj * nk,
                       "chemistry": "the reference's own FP64 IMEX (Euler::IMEX), no learned chemistry",
                       "flux": "the reference's MUSCL_2/minmod + AUSM, FP64", "time": "TimeAdv::EE",
                       "measured_on": "bounded host samples of the workload (cpu_baseline.sample), per cell-step"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        out = run_reference(a, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    out = run_ours(a, rank, world, local)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
