"""One rank of the two-process x-slab test: the oracle slab of this rank is
stepped through eu3d_b200.slabs.SlabRun with torch.distributed (gloo) as the
transport; its interior state is written to an .npz for the parent test.

    python tests/slab_worker.py RANK WORLD PORT OUT REACT TIMEADV CFL STEPS LAYOUT"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402
from datetime import timedelta  # noqa: E402

from _slab_cases import cut, full_oracle, interior  # noqa: E402
from _slab_oracle import OracleSlab  # noqa: E402
from eu3d_b200 import gpu  # noqa: E402
from eu3d_b200.readers import load_h2_ja919  # noqa: E402
from eu3d_b200.slabs import SlabRun, StepSpec, TorchTransport  # noqa: E402


def main():
    rank, world, port, out = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
    react, timeadv, cfl, steps, layout = int(sys.argv[5]), int(sys.argv[6]), float(sys.argv[7]), int(sys.argv[8]), sys.argv[9]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    mech = load_h2_ja919()
    full = full_oracle(mech, (24, 6, 4))
    i0, n, o = cut(mech, full, world, layout)[rank]
    slab = OracleSlab(o, rank, world, overlap=1 if layout == "reference" else 0)
    spec = StepSpec(react=react, timeadv=timeadv, bc_kind=gpu.BC_RSBI, cfl=cfl, final_time=1.0)
    SlabRun([slab], TorchTransport()).run(steps, spec)
    np.savez(out, i0=i0, n=n, CS=interior(o, "CS"), T=interior(o, "T"), P=interior(o, "P"), Yi=interior(o, "Yi"),
             time=o.time, dt=o.dt)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
