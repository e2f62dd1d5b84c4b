"""One rank of the multi-process load-balancing test: a host slab
(tests/_dlb_host.py) stepped through SlabRun with torch.distributed (gloo);
its values and the plan are written to an .npz for the parent test.

    python tests/dlb_worker.py RANK WORLD PORT OUT STEPS [KIND]

KIND "trap" (default): the adaptive trapezoid's rows (HostSlab); "sur": the
learned chemistry's fallback list (HostListSlab)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

from datetime import timedelta  # noqa: E402

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

from _dlb_host import HostListSlab, HostSlab, make_slabs  # noqa: E402
from eu3d_b200 import gpu  # noqa: E402
from eu3d_b200.slabs import SlabRun, StepSpec, TorchTransport  # noqa: E402


def main():
    rank, world, port, out, steps = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4], int(sys.argv[5])
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    kind = sys.argv[6] if len(sys.argv) > 6 else "trap"
    vals, solid = make_slabs(world)[rank]
    if kind == "sur":
        slab = HostListSlab(vals, solid, rank, world)
        spec = StepSpec(react=gpu.REACT_SURROGATE, dlb=True)
    else:
        slab = HostSlab(vals, solid, rank, world)
        spec = StepSpec(react=gpu.REACT_TRAPEZOID, type_=1, dlb=True)
    SlabRun([slab], TorchTransport()).run(steps, spec)
    plan = np.array(slab.last_plan, dtype=np.int64).reshape(-1, 3)
    np.savez(out, vals=slab.vals, plan=plan, loads=np.array(slab.loads))
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
