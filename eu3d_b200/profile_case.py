"""A small oblique-detonation run for kernel profiling (ncu captures must
stay small): the 3D ODW at the benchmark's cell size on a reduced grid,
a few steps of each chemistry form.

    python -m eu3d_b200.profile_case [--ni 256 --nj 128 --nk 64 --L 0.1]
        [--imex 3] [--surrogate 2] [--adaptive 0] [--flux-stage 2] [--kz 0]

--flux-stage picks the FP32 flux kernel: 2 the TMA ring (default), 1 the
load-staged kernel, 0 reads through L1; --kz sets the z planes per flux
block (0: the handle's default for the grid).
"""
from __future__ import annotations

import argparse

from . import gpu
from . import surrogate as S
from .cases import odw_case, setup_odw
from .readers import load_h2_ja919


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ni", type=int, default=256)
    ap.add_argument("--nj", type=int, default=128)
    ap.add_argument("--nk", type=int, default=64)
    ap.add_argument("--L", type=float, default=0.1)
    ap.add_argument("--imex", type=int, default=3)
    ap.add_argument("--surrogate", type=int, default=2)
    ap.add_argument("--adaptive", type=int, default=0)
    ap.add_argument("--flux-stage", type=int, default=2)
    ap.add_argument("--kz", type=int, default=0)
    a = ap.parse_args(argv)
    mech = load_h2_ja919()
    case = odw_case(mech, a.ni, a.nj, a.nk, L=a.L)
    d = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=32)
    setup_odw(d, case)
    d.set_tuning(flux_stage=a.flux_stage)
    if a.kz:
        d.set_tuning(flux_kz=a.kz)
    S.SurrogateModel.load(S.DEFAULT_MODEL).attach(d, 0, gate=S.GATE)
    kw = dict(timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.5, final_time=1.0)
    for react, n in ((gpu.REACT_IMEX, a.imex), (gpu.REACT_SURROGATE, a.surrogate), (gpu.REACT_ADAPTIVE, a.adaptive)):
        if n:
            d.run(n, react=react, **kw)
    d.synchronize()
    print(d.status())


if __name__ == "__main__":
    main()
