"""Persistent work queue of the adaptive trapezoid and the launch-setting
autotuner, through the C ABI."""
import numpy as np
import pytest

from pyoracle import Oracle

from _cases import QUIRKS_FIXED, QUIRKS_REF, fill_state, interior, small_grid
from eu3d_b200 import gpu

pytestmark = pytest.mark.gpu


def _pair(mech, grid, dt, tlo=1300.0, thi=1900.0):
    o = Oracle(mech, grid, QUIRKS_FIXED)
    fill_state(o, 13, tlo, thi, radicals=1e-4)
    devs = []
    for _ in range(2):
        d = gpu.DeviceFlowfield(mech, grid, QUIRKS_FIXED, flux_bits=64)
        d.upload_state(o)
        d.upload("RHS", np.zeros(d.shape("RHS")))
        d.dt = dt
        devs.append(d)
    return devs


@pytest.mark.parametrize("dims", [(10, 6, 4), (37, 5, 2)])
def test_trap1_queue_matches_thread_per_cell(mech, dims):
    a, b = _pair(mech, small_grid(*dims), 5e-8)
    a.set_tuning(chem_queue=0)
    b.set_tuning(chem_queue=1, queue_blocks=2)
    a.trapezoid(1)
    b.trapezoid(1)
    sa, sb = a.status(), b.status()
    assert sa["substeps"] == sb["substeps"] and sa["nchem_max"] == sb["nchem_max"]
    if dims == (10, 6, 4):
        assert sb["nchem_max"] > 1  # stiff enough to substep unevenly
    assert np.array_equal(interior(a.download("Nchem")), interior(b.download("Nchem")))
    for f in ("CS", "T", "P", "Yi", "E"):
        x, y = interior(a.download(f)), interior(b.download(f))
        assert np.max(np.abs(x - y)) <= 1e-13 * np.max(np.abs(x)), f


def test_autotune_restores_state_and_sets_best(mech):
    a, _ = _pair(mech, small_grid(24, 12, 20), 2e-9)
    cs0 = a.download("CS").copy()
    T0 = a.download("T").copy()
    best, ms = a.autotune(steps=2, react=gpu.REACT_TRAPEZOID, type_=1, bc_kind=gpu.BC_RSBI)
    assert ms > 0
    assert best["flux_kz"] in (4, 8, 16, 32) and best["chem_queue"] in (0, 1)
    assert a.tuning() == best
    assert np.array_equal(a.download("CS"), cs0) and np.array_equal(a.download("T"), T0)
    st = a.status()
    assert st["substeps"] == 0  # status restored too
    with pytest.raises(gpu.Eu3dError):
        a.set_tuning(flux_kz=0)


@pytest.mark.parametrize("dims,kz,diff,quirks", [((70, 19, 9), 4, gpu.DIFF_MUSCL2, QUIRKS_FIXED),
                                                 ((33, 9, 4), 4, gpu.DIFF_MUSCL2, QUIRKS_FIXED),
                                                 ((70, 19, 9), 1, gpu.DIFF_MUSCL2, QUIRKS_REF),
                                                 ((40, 17, 7), 16, gpu.DIFF_MUSCL1, QUIRKS_REF),
                                                 ((96, 24, 12), 5, gpu.DIFF_MUSCL2, QUIRKS_FIXED),
                                                 ((70, 19, 9), 4, gpu.DIFF_WENO, QUIRKS_FIXED),
                                                 ((40, 17, 7), 16, gpu.DIFF_WENO, QUIRKS_REF)])
def test_flux_staged_equals_l1_path(mech, dims, kz, diff, quirks):
    """The three FP32 flux kernels -- primitives read through L1 (0), staged
    into shared memory by loads (1), brought into a shared-memory ring by
    TMA (2) -- give the same residual bit for bit, over ragged tiles, blocks
    of one to many z planes, the three reconstructions and the species-face quirk."""
    g = small_grid(*dims)
    o = Oracle(mech, g, quirks)
    fill_state(o, 5, 1100.0, 2600.0)
    out = []
    for stage in (0, 1, 2):
        d = gpu.DeviceFlowfield(mech, g, quirks, flux_bits=32)
        d.upload_state(o)
        d.set_tuning(flux_stage=stage, flux_kz=kz)
        assert d.tuning()["flux_stage"] == stage
        d.boundary(gpu.BC_RSBI)
        d.dt = 2e-8
        d.advection(gpu.ADV_EE, diff)
        out.append(interior(d.download("RHS")))
        assert d.status()["wait_timeouts"] == 0
        d.close()
    assert np.all(np.isfinite(out[0]))
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[0], out[2])
