"""eu3d_cfl_noalloc: the CFL step for callers that cannot allocate device
memory (a framework owns the memory pool, or cudaMalloc/cudaFree would
synchronise the device under their feet).  The entry point must give the
same dt and time as the handle-based eu3d_cfl, call after call, while the
only scratch it uses is the library's fixed device array.

This file is collected last so that a stop-at-first-failure run has already
run every other test before it; it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

from _cases import QUIRKS_FIXED, make_oracle
from eu3d_b200 import gpu

pytestmark = pytest.mark.gpu

TOL = 1e-14  # both paths take the same minimum; only dt's clip arithmetic can round


def _device_fields(d, torch):
    """FP64 copies of the decoded primitives on the device, x fastest."""
    out = {}
    for n in ("D", "U", "V", "W", "P", "Gamma"):
        a = d.download(n)                      # (NI, NJ, NK), k fastest
        x_fastest = np.ascontiguousarray(np.transpose(a, (2, 1, 0)))  # (NK, NJ, NI)
        out[n] = torch.from_numpy(x_fastest).to("cuda")
    return out


@pytest.mark.parametrize("nblocks", [0, 1, 1024], ids=["default", "one-block", "full-scratch"])
def test_noalloc_cfl_matches_handle_cfl_twice(mech, nblocks):
    """nblocks 0 (592 blocks), 1 (one block walks the whole grid) and 1024
    (every entry of the scratch array filled)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    o, g = make_oracle(mech, seed=31, quirks=QUIRKS_FIXED, tlo=1100.0, thi=2600.0)
    d = gpu.DeviceFlowfield(mech, g, quirks=QUIRKS_FIXED, flux_bits=64)
    d.upload_state(o)
    d.update_after_cs()
    d.set_time(0.0)
    f = _device_fields(d, torch)
    NI, NJ, NK = d.NI, d.NJ, d.NK
    dx = g.xnode[1] - g.xnode[0]
    dy = g.ynode[1] - g.ynode[0]
    dz = g.znode[1] - g.znode[0]
    t_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = gpu.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    cfl, final = 0.5, 1.0
    for call in range(2):
        dt_ref = d.cfl(cfl, final)              # existing entry point: dt and time += dt on the handle
        t_ref = d.status()["time"]
        rc = L.eu3d_cfl_noalloc(*[f[n].data_ptr() for n in ("D", "U", "V", "W", "P", "Gamma")],
                                g.ni, g.nj, g.nk, g.bc, NI, NI * NJ, dx, dy, dz, 1, cfl, final,
                                t_dev.data_ptr(), dt_dev.data_ptr(), nblocks, stream)
        assert rc == 0, L.eu3d_last_error()
        torch.cuda.synchronize()
        dt_new, t_new = float(dt_dev.item()), float(t_dev.item())
        assert abs(dt_new - dt_ref) <= TOL * dt_ref, (call, dt_new, dt_ref)
        assert abs(t_new - t_ref) <= TOL * t_ref, (call, t_new, t_ref)
    d.close()


def test_noalloc_cfl_rejects_scratch_overflow(mech):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    buf = torch.ones(4 * 4 * 4, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    L = gpu.load_library()
    rc = L.eu3d_cfl_noalloc(p, p, p, p, p, p, 1, 1, 1, 0, 4, 16, 1.0, 1.0, 1.0, 1, 0.5, 1.0, p, p, 1025, None)
    assert rc == -1
    assert b"1024" in L.eu3d_last_error()
    # a bad layout is refused before any launch
    rc = L.eu3d_cfl_noalloc(p, p, p, p, p, p, 4, 4, 4, 0, 3, 16, 1.0, 1.0, 1.0, 1, 0.5, 1.0, p, p, 0, None)
    assert rc == -1
