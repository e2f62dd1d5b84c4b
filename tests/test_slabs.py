"""x-slab decomposition (Flowfield::Mpi_Boundary and the dt reduction of
CFLcondition, src/Flowfield.cpp:775-1083, :242-272): slabs stepped through
eu3d_b200.slabs give the single-domain result bit for bit.  CPU: the oracle
as the slab state, in one process (loopback transport) and as two gloo
ranks (torch.distributed transport)."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from _slab_cases import assert_slabs_equal_full, cut, full_oracle
from _slab_oracle import OracleSlab
from eu3d_b200 import gpu
from eu3d_b200.slabs import LoopbackTransport, SlabRun, StepSpec, slab_extents

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_extents():
    assert slab_extents(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert slab_extents(64, 2) == [(0, 32), (32, 32)]
    # reference blocks share their end node (src/Mesh.cpp:77-93)
    assert slab_extents(25, 3, "reference") == [(0, 9), (8, 9), (16, 9)]
    with pytest.raises(ValueError):
        slab_extents(24, 5, "reference")
    with pytest.raises(ValueError):
        slab_extents(5, 3)


def _full_run(full, spec, steps):
    for _ in range(steps):
        full.step(spec.react, spec.type_, spec.timeadv, spec.diff, spec.cfl, spec.final_time, spec.bc_kind)


@pytest.mark.parametrize("nranks,layout,react,timeadv,cfl,bc", [
    (3, "partition", gpu.REACT_IMEX, gpu.ADV_EE, 0.5, gpu.BC_RSBI),
    (2, "partition", gpu.REACT_IMEX, gpu.ADV_SSPRK2, 0.5, gpu.BC_RSBI),
    (3, "reference", gpu.REACT_IMEX, gpu.ADV_SSPRK3, 0.5, gpu.BC_RSBI),
    (3, "reference", gpu.REACT_IMEX, gpu.ADV_EE, 0.0, gpu.BC_RSBI),
    (4, "partition", gpu.REACT_NONE, gpu.ADV_EE, 0.3, gpu.BC_TRANSMISSIVE),
])
def test_loopback_slabs_equal_single_domain(mech, nranks, layout, react, timeadv, cfl, bc):
    dims = (25, 6, 4) if layout == "reference" else (24, 6, 4)
    full = full_oracle(mech, dims)
    pieces = cut(mech, full, nranks, layout)
    slabs = [OracleSlab(o, r, nranks, overlap=1 if layout == "reference" else 0) for r, (_, _, o) in enumerate(pieces)]
    spec = StepSpec(react=react, timeadv=timeadv, bc_kind=bc, cfl=cfl, final_time=1.0)
    steps = 3
    SlabRun(slabs, LoopbackTransport()).run(steps, spec)
    _full_run(full, spec, steps)
    assert_slabs_equal_full(full, pieces)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("layout,timeadv", [("partition", gpu.ADV_EE), ("partition", gpu.ADV_SSPRK2),
                                            ("partition", gpu.ADV_SSPRK3)])
def test_two_gloo_ranks_equal_single_domain(mech, tmp_path, layout, timeadv):
    port, world, steps, cfl = _free_port(), 2, 3, 0.5
    outs = [str(tmp_path / f"rank{r}.npz") for r in range(world)]
    procs = [subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "slab_worker.py"), str(r), str(world),
                               str(port), outs[r], str(gpu.REACT_IMEX), str(timeadv), str(cfl), str(steps), layout],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(world)]
    for p in procs:
        out, _ = p.communicate(timeout=240)
        assert p.returncode == 0, out.decode(errors="replace")[-2000:]
    full = full_oracle(mech, (24, 6, 4))
    _full_run(full, StepSpec(react=gpu.REACT_IMEX, timeadv=timeadv, bc_kind=gpu.BC_RSBI, cfl=cfl, final_time=1.0),
              steps)
    b = full.bc
    for o in outs:
        d = np.load(o)
        i0, n = int(d["i0"]), int(d["n"])
        for f in ("CS", "T", "P", "Yi"):
            ref = full.view(f)[b:full.ni + b, b:full.nj + b, b:full.nk + b][i0:i0 + n]
            assert np.array_equal(d[f], ref), f
        assert float(d["time"]) == full.time and float(d["dt"]) == full.dt


def test_loopback_slabs_weno_rk3_equal_single_domain(mech):
    """The WENO reconstruction reads the same two cells on each side as
    MUSCL_2, so the two-plane halo suffices: slabs equal the single domain."""
    full = full_oracle(mech, (24, 6, 4))
    pieces = cut(mech, full, 3, "partition")
    slabs = [OracleSlab(o, r, 3, overlap=0) for r, (_, _, o) in enumerate(pieces)]
    spec = StepSpec(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK3, diff=gpu.DIFF_WENO, bc_kind=gpu.BC_RSBI, cfl=0.5,
                    final_time=1.0)
    SlabRun(slabs, LoopbackTransport()).run(3, spec)
    _full_run(full, spec, 3)
    assert_slabs_equal_full(full, pieces)
