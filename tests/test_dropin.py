"""The compiled C++ caller of the C ABI (eu3d_b200/host): Euler::Computing's
loop body through the shim class on reference-layout host buffers.

CPU: the header compiles from C++, the driver links against the in-tree
library, and the struct layouts of include/eu3d_gpu.h (sizes and every
field offset, as a C++ compiler lays them out) equal the ctypes mirror in
eu3d_b200/gpu.py.  GPU: the driver's result after N steps -- member by
member as src/Euler.cpp:266-333 calls them, and as one eu3d_step per step --
equals the oracle's to 1e-10 per variable."""
import os
import struct
import subprocess
import sys

import ctypes as C
import numpy as np
import pytest

from _cases import QUIRKS_FIXED, interior, make_oracle, rel_err, small_grid
from eu3d_b200 import gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "eu3d_b200", "host")
EXE = os.path.join(HOST, "eu3d_dropin")


def build_driver():
    """Links the driver against the in-tree library (built by
    __graft_entry__.build / python -m eu3d_b200.build)."""
    from eu3d_b200 import build as b
    assert os.path.exists(b.LIB), "libeu3d_gpu.so missing: python -m eu3d_b200.build"
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    return EXE


LAYOUT_SRC = r"""
#include <cstddef>
#include <cstdio>
#include "eu3d_gpu.h"
#define F(S, m) std::printf("%s.%s %zu\n", #S, #m, offsetof(S, m));
int main() {
  std::printf("eu3d_desc %zu\n", sizeof(eu3d_desc));
  std::printf("eu3d_step_desc %zu\n", sizeof(eu3d_step_desc));
  std::printf("eu3d_status %zu\n", sizeof(eu3d_status));
  std::printf("eu3d_tuning %zu\n", sizeof(eu3d_tuning));
  %FIELDS%
  return 0;
}
"""


def test_abi_struct_layouts_match_ctypes_mirror(tmp_path):
    """Every field offset and the size of the four ABI structs as g++ lays
    them out equal those of the ctypes mirror."""
    mirrors = {"eu3d_desc": gpu.Desc, "eu3d_step_desc": gpu.StepDesc, "eu3d_status": gpu.Status,
               "eu3d_tuning": gpu.Tuning}
    lines = [f"F({s}, {f})" for s, cls in mirrors.items() for f, _ in cls._fields_]
    src = tmp_path / "layout.cpp"
    src.write_text(LAYOUT_SRC.replace("%FIELDS%", "\n  ".join(lines)))
    exe = tmp_path / "layout"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                        text=True).stdout.splitlines())
    for s, cls in mirrors.items():
        assert int(out[s]) == C.sizeof(cls), s
        for f, _ in cls._fields_:
            assert int(out[f"{s}.{f}"]) == getattr(cls, f).offset, (s, f)


def test_driver_builds_and_links():
    exe = build_driver()
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def write_case(path, o, grid, mech, steps, react, type_, timeadv, diff, bc_kind, cfl, final_time, dt, whole_step,
               inflow=None):
    NI, NJ, NK = grid.ni + 2 * grid.bc, grid.nj + 2 * grid.bc, grid.nk + 2 * grid.bc
    hd = [0x44335545, 1, grid.ni, grid.nj, grid.nk, grid.bc, mech.NS, mech.NR, steps, react, type_, timeadv, diff,
          bc_kind, QUIRKS_FIXED, 64, whole_step, 1 if inflow is not None else 0]
    with open(path, "wb") as f:
        f.write(struct.pack("<18i", *hd))
        f.write(struct.pack("<3d", cfl, final_time, dt))
        for a in (grid.xnode, grid.ynode, grid.znode, mech.stoi_f, mech.stoi_b, mech.react_tb, mech.af, mech.bf,
                  mech.eaf, mech.c0, mech.c1, mech.mw):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        for n in ("U", "V", "W", "P", "D", "T", "H", "Gamma", "E", "Yi", "CS"):
            f.write(np.ascontiguousarray(o.view(n), dtype="<f8").tobytes())
        if inflow is not None:
            for a in inflow:
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return NI, NJ, NK


def read_result(path, NI, NJ, NK, NS):
    n3 = NI * NJ * NK
    raw = open(path, "rb").read()
    d = np.frombuffer(raw[:8 * (n3 * (NS + 4) + 3 * n3 + 2)], dtype="<f8")
    CS = d[:n3 * (NS + 4)].reshape(NI, NJ, NK, NS + 4)
    T, P, D = (d[n3 * (NS + 4) + i * n3:n3 * (NS + 4) + (i + 1) * n3].reshape(NI, NJ, NK) for i in range(3))
    dt, time = d[-2:]
    tail = np.frombuffer(raw[8 * (n3 * (NS + 4) + 3 * n3 + 2):], dtype="<i8")
    return dict(CS=CS, T=T, P=P, D=D, dt=dt, time=time, nonfinite=int(tail[0]), newton_capped=int(tail[1]),
                nan_step=int(tail[2]))


@pytest.mark.gpu
@pytest.mark.parametrize("whole_step", [0, 1], ids=["members", "eu3d_step"])
@pytest.mark.parametrize("react,type_", [(gpu.REACT_IMEX, 0), (gpu.REACT_TRAPEZOID, 1)], ids=["imex", "trap1"])
def test_cpp_driver_matches_oracle(mech, tmp_path, whole_step, react, type_):
    """Four steps of the reference's loop (CFL 0.3, RSBI ghost fill, EE +
    MUSCL_2/AUSM, IMEX or the adaptive trapezoid) on a 37 x 5 x 2 grid,
    driven by the compiled C++ caller: CS, T, P, D within 1e-10 per variable
    of the oracle; dt and time alike; no NaN step."""
    exe = build_driver()
    g = small_grid(ni=37, nj=5, nk=2, lx=0.037, ly=0.005, lz=0.001)
    st = dict(tlo=1100.0, thi=2600.0) if react == gpu.REACT_IMEX else dict(tlo=1500.0, thi=2200.0, radicals=1e-5)
    o, g = make_oracle(mech, seed=41, quirks=QUIRKS_FIXED, grid=g, **st)
    cfl, dt = (0.3, 0.0) if react == gpu.REACT_IMEX else (0.0, 5e-9)
    case = tmp_path / "case.bin"
    res = tmp_path / "result.bin"
    NI, NJ, NK = write_case(case, o, g, mech, 4, react, type_, gpu.ADV_EE, gpu.DIFF_MUSCL2, gpu.BC_RSBI, cfl, 1.0,
                            dt, whole_step)
    subprocess.run([exe, str(case), str(res)], check=True, timeout=300)
    r = read_result(res, NI, NJ, NK, mech.NS)
    if cfl == 0.0:
        o.dt = dt
    for _ in range(4):
        o.step(react, type_, gpu.ADV_EE, gpu.DIFF_MUSCL2, cfl, 1.0, gpu.BC_RSBI)
    assert np.isfinite(interior(o.view("T"))).all()
    assert r["nan_step"] == -1 and r["nonfinite"] == 0
    for n in ("CS", "T", "P", "D"):
        e = rel_err(interior(r[n]), interior(o.view(n)))
        assert e < 1e-10, (n, e)
    if cfl != 0.0:
        assert abs(r["time"] - o.time) <= 1e-12 * o.time
        assert abs(r["dt"] - o.dt) <= 1e-12 * o.dt


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-v"]))
