#!/usr/bin/env python3
"""Headline benchmark of the EU3D B200 hot path.

Workload (one GPU): 3D oblique detonation, 512 x 256 x 256 interior cells
(33.5 M), stoichiometric H2-air at Mach 7, 0.1 atm, 300 K with a seeded 1 %
inflow density perturbation, 25 degree wedge from x = 0.1 L, L = 0.2 m.
MUSCL_2/minmod + AUSM with FP32 reconstruction and FP64 state, EE time
advance, CFL 0.5, FP64 IMEX chemistry (9 species, 19 reactions), every step
one CUDA-graph replay of CFL -> ghost fill -> flux sweeps -> chemistry+decode.
Inputs (~11 GB of state) are far larger than L2 (126 MB), so no flush is
needed between steps.

Metric: Mcell-steps/s = interior cells x steps / device time.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

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
BYTES_PER_CELL_STEP = 224  # algorithmic HBM bytes per cell-step of the fused step (13 FP64 in/out + T in/out)
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
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def run_ours(a, rank, world, local):
    import torch
    import torch.distributed as dist

    from eu3d_b200 import gpu
    from eu3d_b200.cases import odw_case, setup_odw
    from eu3d_b200.readers import load_h2_ja919

    torch.cuda.set_device(local)
    ni, nj, nk = (int(x) for x in a.grid.split(","))
    mech = load_h2_ja919()
    case = odw_case(mech, ni, nj, nk, seed=rank)
    cells = ni * nj * nk
    dev = gpu.DeviceFlowfield(mech, case.grid, quirks=gpu.QUIRKS_FIXED, flux_bits=a.flux_bits, device=local)
    setup_odw(dev, case)
    step = dict(react=gpu.REACT_IMEX, type_=0, timeadv=gpu.ADV_EE, diff=gpu.DIFF_MUSCL2, bc_kind=gpu.BC_ODM,
                cfl=CFL, final_time=1.0)
    stream = torch.cuda.ExternalStream(dev.stream)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(a.warmup, 3)):
        dev.step(**step)
    dev.synchronize()

    # timed region: K graph replays, CUDA events on the handle's stream
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            dev.step(**step)
        ev1.record(stream)
        dev.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clocks = clk.summary()

    # per-kernel CUDA-event durations over K more steps (no graph)
    dev.profile(True)
    for _ in range(a.steps):
        dev.step(**step)
    prof = dev.profile_read()
    dev.profile(False)
    prof_total = sum(v[0] for v in prof.values())
    launches = sum(v[1] for v in prof.values())
    top = max(prof.items(), key=lambda kv: kv[1][0])
    top_avg_ms = top[1][0] / top[1][1]
    hbm, src = peaks()
    achieved = BYTES_PER_CELL_STEP * cells / (top_avg_ms * 1e-3) / 1e9
    st = dev.status()

    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(dev, step, a.steps, cells, torch)

    value = cells * a.steps * world / (ms * 1e-3) / 1e6
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": max(a.warmup, 3),
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3D oblique detonation {ni}x{nj}x{nk} (ODW, Mach 7 H2-air 0.1 atm 300 K, 25 deg wedge)",
                   "cells_per_gpu": cells, "chemistry": "FP64 IMEX integrator (surrogate path not in this line)",
                   "flux": f"MUSCL_2/minmod + AUSM, FP{a.flux_bits} reconstruction, FP64 state", "time": "EE, CFL 0.5",
                   "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU",
                   "l2": "state ~11 GB per GPU >> 126 MB L2 (no flush needed)", "graph": "one CUDA graph per step"},
        "gpu_launches": int(launches),
        "kernels": {k: {"ms_avg": v[0] / v[1], "share": v[0] / prof_total, "launches": v[1]} for k, v in
                    sorted(prof.items(), key=lambda kv: -kv[1][0])},
        "roofline": {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "note": f"achieved = {BYTES_PER_CELL_STEP} B/cell-step x {cells} cells / avg launch of {top[0]}; "
                             f"peak {src} (MEASURED_PEAKS.json hbm_gbs)"},
        "status": {k: st[k] for k in ("nonfinite_cells", "newton_capped", "dt", "time")},
    }
    if clocks:
        out["clocks"] = clocks
    if e2e:
        out["e2e"] = e2e
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    dev.close()
    return out


def run_e2e(dev, step, K, cells, torch):
    """The same metric through the C ABI with host buffers: upload CS, T, E
    from pinned host memory, decode, K steps each followed by a status read,
    download CS and T -- all inside the timed region."""
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
        dev.step(**step)
        dev.status()
    dev.download("CS", host["CS"])
    dev.download("T", host["T"])
    ev1.record(stream)
    dev.synchronize()
    ms = ev0.elapsed_time(ev1)
    h2d = sum(host[n].nbytes for n in ("CS", "T", "E"))
    d2h = host["CS"].nbytes + host["T"].nbytes + K * 72
    return {"value": cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": h2d // K,
            "d2h_bytes_per_step": d2h // K, "ms": ms,
            "protocol": "upload CS,T,E (pinned) + decode, K eu3d_step calls each with a status read, download CS,T"}


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
            "warmup": a.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"3D oblique detonation {ni}x{nj}x{nk} (ODW), bounded host samples"},
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
