"""Generate the golden fixtures under tests/golden/ from the reference itself.

    python tests/golden/make_golden.py

1. ref_steps.npz -- outputs of the compiled reference (oracle/_ref, built by
   `make -C oracle all` from an EU3D checkout) run through Euler::Computing's
   loop body on small seeded states (tests/_cases.py), for the shipped policy
   and for the corrected one.  The oracle tests replay the same inputs and
   must reproduce these outputs bit for bit, so the oracle stays pinned to the
   reference where the reference library is absent.
2. rsbi_t0.npz -- the reference's own published t = 0 field of the shipped 3D
   RSBI case (output_8/resultsIMEX0_{rank}.dat of an EU3D checkout; 8 ranks,
   4 x 2 x 1 blocks, 6 significant digits), columns X Y T D P U V Y1..Y7, for
   ranks 0 and 5.
3. rsbi_t0_text.npz -- the whole text of output_8/resultsIMEX0_0.dat (the
   reference's Euler::Output file of rank 0), zlib-compressed, to pin the
   result-file writer's format.

4. dlb_plans.npz -- transfer plans of the reference's load-balancing planner
   (DynamicLoadBalancer::DLBPriorityQueue, compiled into oracle/_ref) for
   seeded per-rank loads on 1 to 12 ranks and a few edge cases.

    python tests/golden/make_golden.py --text    (3. only)
    python tests/golden/make_golden.py --dlb     (4. only)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

from _cases import QUIRKS_FIXED, QUIRKS_REF, make_oracle  # noqa: E402
from eu3d_b200.readers import load_h2_ja919  # noqa: E402
from pyoracle import RefCase, copy_state  # noqa: E402

REF_DIR = os.environ.get("EU3D_REF", "/root/reference")

# (name, quirks, react, type, cfl, dt, steps, bc_kind, (seed, tlo, thi, radicals))
HOT = (11, 1100.0, 2600.0, 1e-3)
COOL = (7, 450.0, 980.0, 1e-3)
# the adaptive trapezoid needs substep counts beyond int range (and the
# reference aborts) on far-from-equilibrium hot states; this case takes up to
# five hundred substeps per cell
MILD = (13, 1300.0, 1900.0, 1e-4)
WARM = (11, 800.0, 1200.0, 1e-6)
CASES = [
    ("ref_imex", QUIRKS_REF, 1, 0, 0.0, 2e-8, 3, 0, COOL),
    ("ref_trap0", QUIRKS_REF, 0, 0, 0.0, 2e-8, 1, 0, COOL),
    ("ref_trap1", QUIRKS_REF, 0, 1, 0.0, 2e-8, 2, 0, COOL),
    ("ref_imex_cfl", QUIRKS_REF, 1, 0, 0.3, 0.0, 2, 0, COOL),
    ("fixed_imex", QUIRKS_FIXED, 1, 0, 0.0, 2e-8, 3, 0, HOT),
    ("fixed_trap0", QUIRKS_FIXED, 0, 0, 0.0, 2e-8, 4, 0, WARM),
    ("fixed_trap1", QUIRKS_FIXED, 0, 1, 0.0, 1e-8, 2, 0, MILD),
    ("fixed_imex_cfl_odm", QUIRKS_FIXED, 1, 0, 0.3, 0.0, 2, 1, HOT),
]
OUT_FIELDS = ["CS", "T"]  # interior cells only


def case_state(mech, quirks, st):
    seed, tlo, thi, rad = st
    return make_oracle(mech, seed=seed, quirks=quirks, tlo=tlo, thi=thi, radicals=rad)


def set_inflow(o):
    """ODM inflow planes from the first interior column of the state."""
    bc = o.bc
    for name, src in (("Uint", "U"), ("Vint", "V"), ("Wint", "W"), ("Pint", "P"), ("Dint", "D"), ("Tint", "T"),
                      ("Hint", "H"), ("Eint", "E"), ("Gint", "Gamma")):
        o.view(name)[...] = o.view(src)[bc, bc:-bc, bc:-bc]
    o.view("Yint")[...] = o.view("Yi")[bc, bc:-bc, bc:-bc, :]


def run_reference(mech, name, quirks, react, typ, cfl, dt, steps, bc_kind, st):
    o, g = case_state(mech, quirks, st)
    if bc_kind == 1:
        set_inflow(o)
    rc = RefCase(mech, g, fixed=(quirks == QUIRKS_FIXED))
    copy_state(o, rc)
    if bc_kind == 1:
        for n in ("Uint", "Vint", "Wint", "Pint", "Dint", "Tint", "Hint", "Eint", "Gint", "Yint"):
            rc.view(n)[...] = o.view(n)
    for _ in range(steps):
        if cfl != 0:
            rc.cfl(cfl, 1.0)
        else:
            rc.dt = dt
        rc.boundary(bc_kind)
        rc.advection(0, 1)
        if react == 1:
            rc.imex()
        else:
            rc.trapezoid(typ)
    b = o.bc
    res = {f: np.array(rc.view(f)[b:-b, b:-b, b:-b]) for f in OUT_FIELDS}
    if react == 0 and typ == 1:
        res["Nchem"] = np.array(rc.view("R.Nchem")[b:-b, b:-b, b:-b], dtype=np.float64)
    return res, rc.dt, rc.time


def text_fixture():
    import zlib
    path = os.path.join(REF_DIR, "output_8", "resultsIMEX0_0.dat")
    with open(path, "rb") as fh:
        raw = fh.read()
    np.savez_compressed(os.path.join(HERE, "rsbi_t0_text.npz"),
                        rank0=np.frombuffer(zlib.compress(raw, 9), dtype=np.uint8))
    print("wrote", os.path.join(HERE, "rsbi_t0_text.npz"), len(raw), "bytes of text")


def dlb_cases():
    """Per-rank load vectors: seeded random ones (spread and skewed) and edge cases."""
    rng = np.random.default_rng(2024)
    cases = [[7], [0, 0], [5, 5, 5, 5], [100, 0, 0, 0], [0, 0, 0, 100], [1, 2], [3, 0, 1],
             [100, 0, 0, 50, 1, 80, 3, 2], [2 ** 20, 3, 2 ** 19, 7, 11, 2 ** 18]]
    for n in range(1, 13):
        for _ in range(6):
            cases.append([int(v) for v in rng.integers(0, 5000, n)])
            cases.append([int(v) for v in (rng.pareto(1.2, n) * 300).astype(np.int64)])
    return cases


def dlb_fixture():
    import ctypes as C
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libeu3d_ref.so"))
    out = {}
    for t, loads in enumerate(dlb_cases()):
        a = (C.c_int * len(loads))(*loads)
        buf = (C.c_int * (3 * 200))()
        m = L.ref_dlb_plan(a, len(loads), buf, 200)
        out[f"loads{t}"] = np.array(loads, dtype=np.int64)
        out[f"plan{t}"] = np.array(buf[:3 * m], dtype=np.int64).reshape(m, 3)
    np.savez_compressed(os.path.join(HERE, "dlb_plans.npz"), **out)
    print("wrote", os.path.join(HERE, "dlb_plans.npz"), len(out) // 2, "plans")


def main():
    text_fixture()
    dlb_fixture()
    mech = load_h2_ja919()
    out = {}
    for c in CASES:
        res, dt, t = run_reference(mech, *c)
        for f, v in res.items():
            out[f"{c[0]}/{f}"] = v
        out[f"{c[0]}/dt_time"] = np.array([dt, t])
    np.savez_compressed(os.path.join(HERE, "ref_steps.npz"), **out)

    rs = {}
    for rank in (0, 5):
        path = os.path.join(REF_DIR, "output_8", f"resultsIMEX0_{rank}.dat")
        with open(path) as fh:
            lines = fh.read().split("\n")
        zone = lines[1].replace("\t", " ").split()
        ni, nj, nk = (int(z.split("=")[1]) for z in zone[1:4])
        vals = np.array([float(v) for v in lines[3:] if v.strip()])
        n = ni * nj * nk
        cols = vals.reshape(-1, n)  # X Y Z T D P U V Ma Y1..Y7 L WaitTime
        keep = np.concatenate([cols[0:2], cols[3:8], cols[9:16]])  # X Y T D P U V Y1..Y7
        rs[f"rank{rank}"] = keep.astype(np.float64)
        rs[f"rank{rank}_shape"] = np.array([ni, nj, nk])
    np.savez_compressed(os.path.join(HERE, "rsbi_t0.npz"), **rs)
    print("wrote", os.path.join(HERE, "ref_steps.npz"), os.path.join(HERE, "rsbi_t0.npz"))


if __name__ == "__main__":
    if "--text" in sys.argv:
        text_fixture()
    elif "--dlb" in sys.argv:
        dlb_fixture()
    else:
        main()
