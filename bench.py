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
learned chemistry surrogate (value; its frozen-chemistry gate on, launch
settings from the project's autotuner); the same steps with the plain FP64
IMEX integrator and with the FP64 adaptive integrator (the surrogate's
teacher) are timed on the same GPU and state and reported beside it, with
the per-step split of chemistry and the rest; so is the all-FP64 GPU path
(FP64 reconstruction, AUSM and residual with FP64 IMEX, on a handle of its
own, `all_fp64_imex`); and the coupled accuracy of
the FP32-flux, surrogate and IMEX forms against the all-FP64 run (errors in
rho, p, T and each Y_k, peak T, detonation front) on the 2D case and a
spanwise slice of the 3D one.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
    python bench.py --config {znd,odw2d,rsbi,surrogate}   (the other configurations, one GPU)

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
    ap.add_argument("--no-all-fp64", action="store_true", help="skip the all-FP64 IMEX arm of the headline")
    ap.add_argument("--tuning", default="",
                    help="fixed launch settings instead of the autotuner, e.g. flux_kz=64,cell_blocks=4")
    ap.add_argument("--accuracy-steps", type=int, default=2000)
    ap.add_argument("--accuracy-full", action="store_true",
                    help="also compare on the benchmark's full grid (about 2.5 more minutes)")
    ap.add_argument("--develop", type=int, default=1500, help="2D steps that develop the timed state")
    ap.add_argument("--model", default=os.path.join(ROOT, "eu3d_b200", "data", "sur_h2_ja919.npz"))
    ap.add_argument("--dlb", action="store_true",
                    help="N > 1: balance the learned chemistry's FP64 fallback across the slabs (off by default)")
    ap.add_argument("--config", choices=list(CONFIGS), default="odw3d",
                    help="odw3d: the headline (3D ODW 512x256x256); znd, odw2d, rsbi, surrogate: the other "
                         "benchmark configurations, one GPU")
    return ap.parse_args()


CONFIGS = {
    "odw3d": "3D oblique detonation 512x256x256, surrogate chemistry vs the FP64 integrators",
    "znd": "1D ZND detonation 4000x2x2, FP64",
    "odw2d": "2D oblique detonation 1024x512, FP64 vs FP32 flux; adaptive chemistry queue vs one thread per cell",
    "rsbi": "3D reactive shock-bubble interaction 256^3, FP32 flux vs FP64",
    "surrogate": "chemistry surrogate: FP64 labels, training and inference on 2^22 states",
}


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
    # the chemistry kernels are FP64-bound: their rooflines are chem_roofline's
    cand = [(k, v) for k, v in prof.items() if k in kw and k not in ("cell_imex", "cell_adapt")]
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


# DRAM bytes of a flux launch per fluid cell (ncu dram__bytes_read.sum +
# dram__bytes_write.sum of one launch of k_flux_ring on the 512 x 256 x 64 ODW
# at 64 planes per block, the benchmark's cross-section and tile depth,
# 8.39 M cells of which 5.22 M fluid, all-solid tiles skipped; the full
# 33.5 M-cell case is too large to capture under the profiling rule, and the
# kernel's traffic grows with the fluid cells): 535.2 MB read + 275.4 MB written
TRAFFIC_PER_CELL = {"advection": (535170560 + 275366912) / 5217088}
TRAFFIC_NOTE = {"advection": "ncu DRAM bytes of one launch on the 512x256x64 case (5.22 M fluid cells), per fluid "
                             "cell, times the fluid cells"}


def step_roofline(ms, cells, fluid, hbm, src, stages=2):
    """The flux-and-update part of a step against the HBM roofline, by the
    per-step definition of the algorithmic bytes: per cell and RK stage the
    conserved state read and written (13 x 8 B each) and T read and written
    (2 x 8 B), 224 B; ms the step's non-chemistry time (flux, stage updates,
    ghost fills, CFL)."""
    per = 224 * stages
    out = {"bound": "hbm", "per_cell": f"224 B x {stages} stages", "ms": ms, "peak": hbm, "unit": "GB/s",
           "peak_source": src}
    for name, n in (("all_cells", cells), ("fluid_cells", fluid)):
        ach = per * n / (ms * 1e-3) / 1e9
        out[name] = {"cells": n, "achieved": ach, "frac": ach / hbm}
    return out


def fluid_cells(case, i0=0, n_loc=None):
    """Interior cells of the case (or of the x slab i0 .. i0 + n_loc) outside its wedge."""
    g = case.grid
    x = g.xnode[g.bc:-g.bc][i0:i0 + (n_loc or g.ni)][:, None]
    y = g.ynode[g.bc:-g.bc][None, :]
    w = case.wedge
    solid = (x > w[0]) & ((y - w[1]) < (x - w[0]) * w[2])
    return int((~solid).sum()) * g.nk


# FP64 operations of the reference's per-cell chemistry, counted by running
# its arithmetic on an operation-counting type (oracle/opcount.py,
# reference_counts: 64 states of the surrogate's standalone set, the decode
# at 3 Newton iterations): add, sub, mul, div 1 FLOP each; exp and log 20,
# a non-integer pow 40, sqrt 1 FLOP-equivalents in the "equiv" figures.
# tests/test_opcount.py recomputes them.
CHEM_FLOP = {"imex_cell": 8277.0, "imex_cell_equiv": 10159.0,
             "adaptive_substep": 7923.2, "adaptive_substep_equiv": 9625.2}
# nominal FP64 peak of one B200 (no measured FP64 figure exists on this pool)
FP64_PEAK_TFLOPS = 37.0


def chem_roofline(profs, stats, fluid, steps_run, K):
    """FP64 rooflines of the chemistry kernels: IMEX (CHEM_FLOP per fluid cell
    a launch) and the adaptive integrator (CHEM_FLOP per substep taken)."""
    out = {}
    if "cell_imex" in profs.get("imex", {}):
        ms, n = profs["imex"]["cell_imex"]
        for key in ("imex_cell", "imex_cell_equiv"):
            ach = CHEM_FLOP[key] * fluid / (ms / n * 1e-3) / 1e12
            out.setdefault("cell_imex", {})[key.replace("imex_cell", "flop")] = {
                "achieved": ach, "unit": "TFLOP/s", "peak": FP64_PEAK_TFLOPS, "frac": ach / FP64_PEAK_TFLOPS}
        out["cell_imex"]["flop_per_cell"] = CHEM_FLOP["imex_cell"]
        out["cell_imex"]["avg_ms"] = ms / n
    ad = profs.get("adaptive", {})
    key_k = "cell_adapt" if "cell_adapt" in ad else ("adapt_queue" if "adapt_queue" in ad else None)
    if key_k and stats.get("adaptive"):
        ms, n = ad[key_k]
        sub = stats["adaptive"]["substeps"] / max(steps_run, 1)  # per launch
        for key in ("adaptive_substep", "adaptive_substep_equiv"):
            ach = CHEM_FLOP[key] * sub / (ms / n * 1e-3) / 1e12
            out.setdefault(key_k, {})[key.replace("adaptive_substep", "flop")] = {
                "achieved": ach, "unit": "TFLOP/s", "peak": FP64_PEAK_TFLOPS, "frac": ach / FP64_PEAK_TFLOPS}
        out[key_k]["substeps_per_launch"] = sub
        out[key_k]["avg_ms"] = ms / n
    out["note"] = ("algorithmic FP64 work of the reference's arithmetic (oracle/opcount.py) / CUDA-event launch time, "
                   "against a nominal 37 TFLOP/s FP64 peak; the device code evaluates the same chemistry with fewer "
                   "operations (powers by multiplication, mixture polynomials summed once, zero stoichiometric "
                   "factors dropped), so this is work done per second, not pipe occupancy")
    return out


# kernels of the step that make up its chemistry (the rest: ghost fills, CFL,
# flux sweeps and stage updates)
CHEM_KERNELS = {"cell_imex", "cell_adapt", "sur_gate", "sur_mlp", "sur_apply", "sur_fallback", "sur_fallback_finish",
                "sur_mlp_apply"}


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
        # --dlb: the surrogate form balances its fallback list across the
        # slabs (the other forms have nothing to balance in this protocol)
        spec = StepSpec(**step, dlb=a.dlb and step["react"] == gpu.REACT_SURROGATE)
        return lambda: run.step(spec)

    W = max(a.warmup, 3)
    tuned = None
    if a.tuning:
        # fixed launch settings instead of the autotuner (a profiler's
        # serialised launches would mislead the autotuner's timing)
        fixed = {k: int(v) for k, v in (kv.split("=") for kv in a.tuning.split(","))}
        dev.set_tuning(**fixed)
        tuned = {"setting": dev.tuning(), "fixed": True}
    elif world == 1:
        # the project's autotuner picks the flux tile depth and kernel on this
        # state (restored after every trial), outside the timed region
        reset()
        best, best_ms = dev.autotune(steps=2, **dict(base, react=gpu.REACT_SURROGATE))
        tuned = {"setting": best, "ms_per_step": best_ms}
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
    all64 = None
    if world == 1 and a.flux_bits == 32 and not a.no_all_fp64:
        # the all-FP64 GPU path (FP64 reconstruction and residual, FP64 IMEX)
        # on a handle of its own, from the same developed state
        d64 = gpu.DeviceFlowfield(mech, grid, quirks=gpu.QUIRKS_FIXED, flux_bits=64, device=local)
        setup_odw(d64, case)
        extrude_state(d2, d64)
        d64.set_time(0.0)
        step64 = dict(base, react=gpu.REACT_IMEX)
        ms64, _ = timed_steps(d64, step64, a.steps, W, torch, world, dist, local=local)
        p64 = profiled(d64, step64, a.steps)
        chem64 = sum(v[0] for k, v in p64.items() if k in CHEM_KERNELS) / a.steps
        all64 = {"value": cells * a.steps / (ms64 * 1e-3) / 1e6, "ms_per_step": ms64 / a.steps,
                 "split_ms_per_step": {"chemistry_ms": chem64,
                                       "non_chemistry_ms": sum(v[0] for v in p64.values()) / a.steps - chem64},
                 "status": {k: d64.status()[k] for k in ("nonfinite_cells", "newton_capped")}}
        d64.close()
    hbm, tfl, src = peaks()
    prof = profs["surrogate"]
    st = statuses["surrogate"]
    # cells one launch must process: the fluid cells of this rank; the network
    # takes the cells the frozen-chemistry gate listed, per step
    steps_run = a.steps + W
    net_cells = (st["surrogate_cells"] + st["surrogate_fallback"] + st["surrogate_audited"]) // max(steps_run, 1)
    units = {k: fluid for k in kernel_work(4)}
    units["sur_mlp"] = units["sur_mlp_apply"] = units["sur_apply"] = net_cells
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
                                "gate: cells below 600 K with radicals <= 1e-6 skip the network (the gate runs "
                                "inside the SSP-RK2 stage 2 kernel, so its time is in the non-chemistry split)",
                   "flux": f"MUSCL_2/minmod + AUSM, FP{a.flux_bits} reconstruction, FP64 state",
                   "time": f"SSP-RK2, CFL {CFL}",
                   "state": f"developed: 2D case advanced {a.develop} steps with the FP64 adaptive integrator, "
                            f"extruded along z",
                   "parallelism": (f"{world} x slabs of {n_loc} cells (NCCL halo send/recv, all-reduce MIN of dt"
                                   + (", the surrogate's FP64 fallback balanced across the slabs)" if a.dlb else ")")
                                   if world > 1 else "1 GPU"),
                   "l2": "state ~12 GB per GPU >> 126 MB L2 (no flush needed)",
                   "graph": "one CUDA graph per step" if world == 1 else "per-op launches (halo exchanges between)",
                   "autotuned": tuned},
        "integrator": {"imex_value": integ["imex"], "adaptive_value": integ["adaptive"],
                       "ratio_vs_imex": value / integ["imex"], "ratio_vs_adaptive": value / integ["adaptive"],
                       "ms_per_step": {k: timing[k] / a.steps for k in timing},
                       "split_ms_per_step": split,
                       "amdahl_bound_vs_imex": amdahl,
                       "amdahl_note": "the IMEX step over its non-chemistry part: the ratio a free chemistry would "
                                      "reach against plain IMEX with the same flux, stage and boundary kernels",
                       "note": "same GPU, same state and step; imex = the reference's one-step FP64 IMEX, "
                               "adaptive = FP64 adaptive integrator (the surrogate's teacher and fallback)"},
        "all_fp64_imex": (dict(all64, ratio=value / all64["value"],
                               note="the all-FP64 GPU path: FP64 reconstruction, AUSM and residual with the "
                                    "reference's FP64 IMEX, same state and step (the imex arm above keeps the "
                                    "FP32 flux of the timed form)")
                          if all64 else None),
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
        "roofline_chemistry": chem_roofline(profs, statuses, fluid, a.steps + W, a.steps),
        "roofline_step": step_roofline(split["surrogate"]["non_chemistry_ms"], n_loc * nj * nk, fluid, hbm, src),
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
        if world == 1:
            reset()
            out["e2e_state_through_host"] = run_e2e_host_state(dev, dict(base, react=gpu.REACT_SURROGATE),
                                                               max(a.steps // 2, 2), cells, torch)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    dev.close()
    d2.close()
    return out


def run_e2e(dev, step, K, cells, torch, world=1, dist=None, chemistry="surrogate chemistry"):
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
            "protocol": f"upload CS,T,E (pinned) + decode, K eu3d_step calls ({chemistry}) each with a status "
                        "read, download CS,T; the state stays on the device between steps (the drop-in's design), "
                        "so the host copies are amortised over the K steps and the value depends on K"}


def run_e2e_host_state(dev, step, K, cells, torch):
    """The host-array calling convention of the reference (its state lives in
    host arrays between calls): every step uploads CS, T, E from pinned host
    memory, decodes, steps and downloads CS and T.  Reported beside e2e."""
    one = step if callable(step) else (lambda: dev.step(**step))
    shapes = {n: dev.shape(n) for n in ("CS", "T", "E")}
    host = {n: torch.empty(s, dtype=torch.float64, pin_memory=True).numpy() for n, s in shapes.items()}
    for n in host:
        dev.download(n, host[n])
    stream = torch.cuda.ExternalStream(dev.stream)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(K):
        for n in ("CS", "T", "E"):
            dev.upload(n, host[n])
        dev.update_after_cs()
        one()
        dev.download("CS", host["CS"])
        dev.download("T", host["T"])
    ev1.record(stream)
    dev.synchronize()
    ms = ev0.elapsed_time(ev1)
    h2d = sum(host[n].nbytes for n in ("CS", "T", "E"))
    d2h = host["CS"].nbytes + host["T"].nbytes
    return {"value": cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms": ms,
            "protocol": "every step: upload CS,T,E (pinned), decode, one eu3d_step, download CS,T"}


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


# ------------------------------------------------- the other configurations
def _line(metric, value, unit, K, W, ms, dtype, config, **extra):
    out = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": K, "warmup": W,
           "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
           "data": "synthetic", "config": config}
    out.update(extra)
    return out


def _case_run(dev, forms, K, W, torch, cells, units, pb, value_form, clocks_form=None):
    """Times each form (eu3d_step keyword sets) K steps after W warm-up from
    the state `reset` puts back; per-kernel profile, roofline of the value
    form's top kernel, clocks during the value form's timed steps."""
    hbm, tfl, src = peaks()
    timing, profs, stats, clocks = {}, {}, {}, None
    for name, (reset, step) in forms.items():
        reset()
        ms, clk = timed_steps(dev, step, K, W, torch, 1, None, clocks=(name == (clocks_form or value_form)))
        if clk:
            clocks = clk
        timing[name] = ms
        stats[name] = dev.status()
        reset()
        profs[name] = profiled(dev, step, K)
    prof = profs[value_form]
    rf = roofline(prof, units, hbm, tfl, src, pb=pb)
    if "cell_imex" in prof:
        fluid = units.get("cell_rk1", cells)
        rf["chemistry"] = chem_roofline({"imex": prof}, {}, fluid, 1, K).get("cell_imex")
    rates = {k: cells * K / (v * 1e-3) / 1e6 for k, v in timing.items()}
    return timing, profs, stats, clocks, rf, rates


def _kernel_table(profs):
    return {f: {k: {"ms_avg": v[0] / v[1], "share": v[0] / sum(x[0] for x in pr.values()), "launches": v[1]}
                for k, v in sorted(pr.items(), key=lambda kv: -kv[1][0])} for f, pr in profs.items()}


def _port_baseline(make, step, steps, label):
    """The oracle (the C restatement of the reference's path) on one host
    core: `make()` builds it, `step(o)` advances it one step."""
    o, cells = make()
    step(o)
    t0 = time.perf_counter()
    for _ in range(steps):
        step(o)
    dt = time.perf_counter() - t0
    return {"value": cells * steps / dt / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{label}: {steps} steps after one warm-up step on one host core", "seconds": dt}


def run_znd(a):
    """C1: the 1D ZND detonation at its full size, FP64 throughout, SSP-RK2,
    CFL 0.3 (at 0.5 the reference's own arithmetic goes non-finite in the
    first step at the driver interface).  Value: the reference's one-step
    IMEX; beside it the FP64 adaptive chemistry.  The fixed-policy adaptive
    trapezoid (the configuration's chemistry) goes non-finite at its 12th step
    in the reference's arithmetic, so it is not timed."""
    import torch
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import upload_primitive_state, znd_case
    from eu3d_b200.readers import load_h2_ja919
    mech = load_h2_ja919()
    g, st = znd_case(mech)
    dev = gpu.DeviceFlowfield(mech, g, quirks=gpu.QUIRKS_FIXED, flux_bits=64)
    dev.set_elements(S.atoms_matrix(mech))

    def reset():
        upload_primitive_state(dev, st)
        dev.set_time(0.0)
        dev.reset_status()

    base = dict(timeadv=gpu.ADV_SSPRK2, diff=gpu.DIFF_MUSCL2, bc_kind=gpu.BC_TRANSMISSIVE, cfl=0.3, final_time=1.0)
    forms = {"imex": (reset, dict(base, react=gpu.REACT_IMEX)), "adaptive": (reset, dict(base, react=gpu.REACT_ADAPTIVE))}
    K, W = max(a.steps, 500), max(a.warmup, 20)
    cells = g.ni * g.nj * g.nk
    units = {k: cells for k in kernel_work(8)}
    timing, profs, stats, clocks, rf, rates = _case_run(dev, forms, K, W, torch, cells, units, 8, "imex")
    reset()
    e2e = run_e2e(dev, forms["imex"][1], K, cells, torch, chemistry="FP64 IMEX")
    dev.close()

    def make():
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from pyoracle import Oracle
        o = Oracle(mech, g, gpu.QUIRKS_FIXED)
        for n in ("U", "V", "W", "P", "T", "Yi"):
            o.view(n)[...] = st[n]
        o.prims_from_state()
        return o, cells

    cb = _port_baseline(make, lambda o: o.step(gpu.REACT_IMEX, 0, gpu.ADV_SSPRK2, gpu.DIFF_MUSCL2, 0.3, 1.0,
                                                gpu.BC_TRANSMISSIVE), 20,
                        "the oracle on the whole 4000x2x2 case, SSP-RK2 + IMEX, CFL 0.3")
    return _line("Mcell-steps/s, 1D ZND detonation 4000x2x2, FP64", rates["imex"], UNIT, K, W, timing["imex"], "f64",
                 {"workload": "1D ZND detonation 4000x2x2 cells on 0.1 m: stoichiometric H2-air 300 K 1 atm, "
                              "H2O/N2 driver 3000 K 30 atm for x < 5 mm, transmissive ends",
                  "cells": cells, "chemistry": "FP64 IMEX (the reference's); adaptive FP64 beside",
                  "flux": "MUSCL_2/minmod + AUSM, FP64", "time": "SSP-RK2, CFL 0.3", "graph": "one CUDA graph per step",
                  "l2": "the whole state fits L2: steps are latency- and launch-bound"},
                 rates={k: v for k, v in rates.items()}, ms_per_step_forms={k: v / K for k, v in timing.items()},
                 kernels=_kernel_table(profs), roofline=rf, clocks=clocks, e2e=e2e, cpu_baseline=cb,
                 gpu_launches=int(sum(v[1] for v in profs["imex"].values())),
                 status={k: stats["imex"][k] for k in ("nonfinite_cells", "newton_capped", "dt", "time")})


def run_odw2d(a):
    """C2: the 2D oblique detonation 1024x512 from a developed state (1000
    SSP-RK2 steps of FP64 adaptive chemistry): IMEX with FP64 and with FP32
    reconstruction/AUSM (FP64 state); the FP64 adaptive chemistry with one
    thread per cell and on the persistent queue (one cell per lane, refill).
    The reference's IMEX has the same work in every cell, so the queue is
    measured on the integrator whose substep counts vary from cell to cell."""
    import torch
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import extrude_state, odw_case, setup_odw
    from eu3d_b200.readers import load_h2_ja919
    mech = load_h2_ja919()
    ni, nj = 1024, 512
    case = odw_case(mech, ni, nj, 2)
    src = gpu.DeviceFlowfield(mech, case.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=32)
    setup_odw(src, case)
    src.set_elements(S.atoms_matrix(mech))
    src.run(1000, react=gpu.REACT_ADAPTIVE, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=CFL, final_time=1.0)
    src.synchronize()
    cells = ni * nj * 2
    fluid = fluid_cells(case)
    out_forms, profs_all, timing_all, rates_all = {}, {}, {}, {}
    K, W = max(a.steps, 50), max(a.warmup, 5)
    base = dict(timeadv=gpu.ADV_SSPRK2, diff=gpu.DIFF_MUSCL2, bc_kind=gpu.BC_ODM, cfl=CFL, final_time=1.0)
    results = {}
    for bits in (64, 32):
        dev = gpu.DeviceFlowfield(mech, case.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=bits)
        setup_odw(dev, case)
        dev.set_elements(S.atoms_matrix(mech))

        def reset(q=None, dev=dev):
            extrude_state(src, dev)
            dev.set_time(0.0)
            dev.reset_status()
            if q is not None:
                dev.set_tuning(adapt_queue=q)

        forms = {f"imex_fp{bits}": (lambda dev=dev: reset(0, dev), dict(base, react=gpu.REACT_IMEX))}
        if bits == 32:
            forms["adaptive_thread_per_cell"] = (lambda dev=dev: reset(0, dev), dict(base, react=gpu.REACT_ADAPTIVE))
            forms["adaptive_queue"] = (lambda dev=dev: reset(1, dev), dict(base, react=gpu.REACT_ADAPTIVE))
        units = {k: fluid for k in kernel_work(bits // 8)}
        timing, profs, stats, clocks, rf, rates = _case_run(dev, forms, K, W, torch, cells, units, bits // 8,
                                                            f"imex_fp{bits}")
        results[bits] = (rf, clocks, stats)
        timing_all.update(timing)
        profs_all.update(profs)
        rates_all.update(rates)
        if bits == 32:
            reset(0)
            e2e = run_e2e(dev, forms["imex_fp32"][1], K, cells, torch, chemistry="FP64 IMEX, FP32 flux")
        dev.close()
    src.close()
    rf, clocks, stats = results[32]
    chem = {f: sum(v[0] for k, v in profs_all[f].items() if k in CHEM_KERNELS | {"adapt_list", "adapt_queue", "adapt_finish"}) / K
            for f in ("adaptive_thread_per_cell", "adaptive_queue")}
    cb = cpu_baseline(slab=(64, 32, 2))
    return _line("Mcell-steps/s, 2D ODW 1024x512, FP32 flux / FP64 state, IMEX", rates_all["imex_fp32"], UNIT, K, W,
                 timing_all["imex_fp32"], "f32 (reconstruction, AUSM, residual) + f64 (state, decode, chemistry)",
                 {"workload": "2D oblique detonation 1024x512x2 (L = 0.2 m, Mach 7 H2-air 0.1 atm 300 K, 25 deg "
                              "wedge), developed by 1000 steps of FP64 adaptive chemistry",
                  "cells": cells, "fluid_cells": fluid, "time": f"SSP-RK2, CFL {CFL}", "graph": "one CUDA graph per step",
                  "l2": "state ~0.4 GB > 126 MB L2"},
                 rates=rates_all, ms_per_step_forms={k: v / K for k, v in timing_all.items()},
                 fp64_vs_fp32_speedup=rates_all["imex_fp32"] / rates_all["imex_fp64"],
                 adaptive_chemistry_ms_per_step={"thread_per_cell": chem["adaptive_thread_per_cell"],
                                                 "persistent_queue": chem["adaptive_queue"]},
                 kernels=_kernel_table(profs_all), roofline=rf, clocks=clocks, e2e=e2e, cpu_baseline=cb,
                 gpu_launches=int(sum(v[1] for v in profs_all["imex_fp32"].values())),
                 status={k: stats["imex_fp32"][k] for k in ("nonfinite_cells", "newton_capped", "dt", "time")})


def run_rsbi(a):
    """C3: the 3D reactive shock-bubble interaction at 256^3, SSP-RK2, IMEX,
    RSBI (mirror) ghost fill, CFL 0.5, one CUDA graph per step; FP32
    reconstruction/AUSM/residual (value) and FP64 beside, and the FP32 run's
    errors against the FP64 one after `--accuracy-steps`/20 steps from the same
    initial state (pointwise rho, p, T; Y_k against each species' scale)."""
    import torch
    from eu3d_b200 import gpu
    from eu3d_b200.cases import rsbi_case, upload_primitive_state
    from eu3d_b200.readers import load_h2_ja919
    from eu3d_b200.validate import field_errors
    mech = load_h2_ja919()
    t0 = time.time()
    case = rsbi_case(mech, n=256)
    setup_s = time.time() - t0
    g = case.grid
    cells = g.ni * g.nj * g.nk
    base = dict(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK2, diff=gpu.DIFF_MUSCL2, bc_kind=gpu.BC_RSBI, cfl=CFL,
                final_time=1.0)
    K, W = max(a.steps, 10), max(a.warmup, 3)
    nerr = max(a.accuracy_steps // 20, 10)
    rates, timing_all, profs_all, fields = {}, {}, {}, {}
    rf = clocks = e2e = stats32 = None
    for bits in (64, 32):
        dev = gpu.DeviceFlowfield(mech, g, quirks=gpu.QUIRKS_FIXED, flux_bits=bits)

        def reset(dev=dev):
            upload_primitive_state(dev, case.state)
            dev.set_time(0.0)
            dev.reset_status()

        units = {k: cells for k in kernel_work(bits // 8)}
        timing, profs, stats, clk, r, rt = _case_run(dev, {f"fp{bits}": (reset, base)}, K, W, torch, cells, units,
                                                     bits // 8, f"fp{bits}")
        rates.update(rt)
        timing_all.update(timing)
        profs_all.update(profs)
        reset()
        dev.run(nerr, **base)
        dev.synchronize()
        b = g.bc
        fields[bits] = {n: dev.download(n)[b:-b, b:-b, b:-b].copy() for n in ("T", "P", "D", "Yi")}
        fields[bits]["nonfinite"] = dev.status()["nonfinite_cells"]
        if bits == 32:
            rf, clocks, stats32 = r, clk, stats["fp32"]
            reset()
            e2e = run_e2e(dev, base, K, cells, torch, chemistry="FP64 IMEX, FP32 flux")
        dev.close()
    finite = np.isfinite(fields[64]["T"]) & np.isfinite(fields[32]["T"])
    err = field_errors(fields[64], fields[32], finite, mech.species)
    err["cells_compared"] = int(finite.sum())
    err["nonfinite_cells"] = {"fp64": fields[64]["nonfinite"], "fp32": fields[32]["nonfinite"]}
    cb = cpu_baseline(slab=(32, 32, 8))
    return _line("Mcell-steps/s, 3D reactive shock-bubble 256^3, FP32 flux / FP64 state, IMEX", rates["fp32"], UNIT, K,
                 W, timing_all["fp32"], "f32 (reconstruction, AUSM, residual) + f64 (state, decode, chemistry)",
                 {"workload": "3D reactive shock-bubble interaction 256^3 on a 0.1 m cube: Mach 2 shock in air "
                              "(300 K, 1 atm) from x = 0.01 m into a stoichiometric H2-O2 bubble of radius 25 mm at "
                              "the centre, tanh interface 2 cells wide, seeded radial perturbation 0.02 R on "
                              "spherical harmonics l <= 8",
                  "cells": cells, "time": f"SSP-RK2, CFL {CFL}", "chemistry": "FP64 IMEX", "boundary": "RSBI (mirror)",
                  "graph": "one CUDA graph per step", "l2": "state ~6 GB >> 126 MB L2", "setup_s": setup_s},
                 rates=rates, fp32_vs_fp64_speedup=rates["fp32"] / rates["fp64"],
                 fp32_flux_errors_vs_fp64={"steps": nerr, "errors": err,
                                           "measures": "rho, p, T: pointwise relative; Y_k: |dY_k| / max Y_k"},
                 kernels=_kernel_table(profs_all), roofline=rf, clocks=clocks, e2e=e2e, cpu_baseline=cb,
                 gpu_launches=int(sum(v[1] for v in profs_all["fp32"].values())),
                 status={k: stats32[k] for k in ("nonfinite_cells", "newton_capped", "dt", "time")})


def run_surrogate(a):
    """C4: the learned chemistry standalone on 2^22 states (T 300-3500 K, log p
    in [0.05, 50] atm, compositions at the element ratios of stoichiometric
    H2-air, dt log-uniform in [1e-9, 1e-7] s): FP64 labels from the adaptive
    integrator, Adam training steps (batch 8192) on the tensor-core kernels,
    and inference of all states with the fused tensor-core kernel.  Value:
    inference, in million states per second; the roofline is the inference
    kernel's (71 168 FLOP a state)."""
    import torch
    from eu3d_b200 import gpu
    from eu3d_b200 import surrogate as S
    from eu3d_b200.readers import load_h2_ja919
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    mech = load_h2_ja919()
    n = 1 << 22
    from eu3d_b200.readers import make_grid
    grid = make_grid(8, 0, 1, 8, 0, 1, 2, 0, 1, 2, fixed_ghosts=True)
    dev = gpu.DeviceFlowfield(mech, grid, quirks=gpu.QUIRKS_FIXED, flux_bits=32)
    sur = gpu.DeviceSurrogate(dev, n, S.atoms_matrix(mech))
    env = (300.0, 3500.0, np.log(0.05), np.log(50.0), np.log(1e-9), np.log(1e-7))
    sur.add_random(n, env, S.species_index(mech), 7)
    # labels and training are synchronous calls on the surrogate's own stream:
    # timed on the host around them, the device idle on both sides
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nv = sur.label(gpu.REACT_ADAPTIVE, cap=4096)
    label_ms = (time.perf_counter() - t0) * 1e3
    X, Lb = sur.dataset()
    model = S.SurrogateModel.load(a.model)
    sur.set_norm(model.norm)
    sur.set_params(model.params)
    batch, steps = 8192, max(a.steps, 200)
    sur.train(20, batch, 1e-4, 1e-5, 1, 3)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sur.train(steps, batch, 1e-4, 1e-5, 1, 5)
    torch.cuda.synchronize()
    train_ms = (time.perf_counter() - t0) * 1e3
    feats = torch.from_numpy(np.ascontiguousarray(S.features(X, model.norm), dtype=np.float32)).cuda()
    out = torch.empty((n, 16), dtype=torch.float32, device="cuda")
    # a stream of its own (the legacy default stream's handle is 0, which the
    # library reads as "the surrogate's stream", where these events would
    # not see the kernels)
    cur = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(max(a.warmup, 3)):
        sur.infer_device(feats.data_ptr(), n, out.data_ptr(), cur.cuda_stream)
    K = max(a.steps, 10)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    clk = ClockSampler(0)
    clk.__enter__()
    ev[0].record(cur)
    for _ in range(K):
        sur.infer_device(feats.data_ptr(), n, out.data_ptr(), cur.cuda_stream)
    ev[1].record(cur)
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    infer_ms = ev[0].elapsed_time(ev[1]) / K
    hbm, tfl, src = peaks()
    flop = kernel_work(4)["sur_mlp"][1]
    ach = flop * n / (infer_ms * 1e-3) / 1e12
    rf = {"bound": "tensor", "kernel": "sur_mlp (array source)", "achieved": ach, "peak": tfl, "unit": "TFLOP/s",
          "frac": ach / tfl, "traffic": None, "per_cell": f"{flop} FLOP", "cells": n, "avg_ms": infer_ms,
          "peak_source": src}
    train_flop = 3 * flop * batch * steps
    # host baseline: the oracle's FP64 forward pass (numpy) on a bounded sample
    from mlp_oracle import forward
    m = 1 << 16
    f64 = S.features(X[:m], model.norm).astype(np.float64)
    t0 = time.perf_counter()
    forward(model.params.astype(np.float64), f64, quantize=False)
    cpu_s = time.perf_counter() - t0
    cb = {"value": m / cpu_s / 1e6, "unit": "Mstates/s", "cores": os.cpu_count() or 1, "kind": "port",
          "sample": f"the oracle's FP64 forward pass (numpy, BLAS threads) on {m} of the states", "seconds": cpu_s}
    # e2e: host features in, host outputs back, every pass
    host_in = torch.from_numpy(np.ascontiguousarray(S.features(X, model.norm), dtype=np.float32)).pin_memory()
    host_out = torch.empty((n, 16), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(cur):
        e0.record(cur)
        for _ in range(3):
            feats.copy_(host_in, non_blocking=True)
            sur.infer_device(feats.data_ptr(), n, out.data_ptr(), cur.cuda_stream)
            host_out.copy_(out, non_blocking=True)
        e1.record(cur)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / 3
    sur.close()
    dev.close()
    return _line("Mstates/s, chemistry surrogate inference on 2^22 states", n / (infer_ms * 1e-3) / 1e6, "Mstates/s",
                 K, max(a.warmup, 3), infer_ms * K, "bf16 (weights, activations) + f32 (accumulation)",
                 {"workload": "2^22 random thermochemical states (T 300-3500 K, p 0.05-50 atm, stoichiometric H2-air "
                              "element ratios, dt 1e-9-1e-7 s); MLP 12 -> 3x128 GELU -> 10",
                  "states": n, "labels": "FP64 adaptive integrator (cap 4096 substeps)",
                  "training": f"Adam, batch {batch}, {steps} steps", "l2": "inputs 268 MB > 126 MB L2"},
                 labels={"valid": nv, "ms": label_ms, "Mstates_per_s": n / (label_ms * 1e-3) / 1e6},
                 training={"steps": steps, "batch": batch, "ms": train_ms,
                           "samples_per_s": batch * steps / (train_ms * 1e-3),
                           "tflops_forward_backward": train_flop / (train_ms * 1e-3) / 1e12,
                           "flop_note": "3 x 71 168 FLOP per sample (forward and the two backward GEMMs)"},
                 roofline=rf, clocks=clocks, cpu_baseline=cb,
                 e2e={"value": n / (e2e_ms * 1e-3) / 1e6, "unit": "Mstates/s", "h2d_bytes_per_step": n * 64,
                      "d2h_bytes_per_step": n * 64, "ms": e2e_ms,
                      "protocol": "pinned host features -> device, inference, outputs -> pinned host, per pass"},
                 gpu_launches=K)


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
    if a.config != "odw3d":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            fn = {"znd": run_znd, "odw2d": run_odw2d, "rsbi": run_rsbi, "surrogate": run_surrogate}[a.config]
            print(json.dumps(fn(a)), flush=True)
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
