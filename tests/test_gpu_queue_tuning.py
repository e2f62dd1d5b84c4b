"""Persistent work queues (the adaptive trapezoid's, and the FP64 adaptive
chemistry's on the surrogate's fallback workers), the launch-setting
autotuner and the FP32 flux kernels' agreement, through the C ABI."""
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
    assert best["flux_kz"] in (4, 8, 16, 32, 64) and best["chem_queue"] in (0, 1) and best["cell_blocks"] == 3
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


def test_adaptive_queue_matches_thread_per_cell(mech):
    """The FP64 adaptive chemistry on the persistent queue (every fluid cell
    listed, one cell per lane with refill) against one thread per cell: the
    same substeps, and the same state to rounding (the two kernels inline the
    same substep arithmetic; contraction may differ in the last bit)."""
    from eu3d_b200 import surrogate as S
    a, b = _pair(mech, small_grid(10, 6, 4), 3e-8, tlo=1100.0, thi=2600.0)
    for d, q in ((a, 0), (b, 1)):
        d.set_elements(S.atoms_matrix(mech))
        d.set_tuning(adapt_queue=q)
        assert d.tuning()["adapt_queue"] == q
        d.react_adaptive()
    sa, sb = a.status(), b.status()
    assert sa["substeps"] == sb["substeps"] > 240  # more than one substep per cell on average
    for f in ("CS", "T", "P", "Yi", "E"):
        x, y = interior(a.download(f)), interior(b.download(f))
        assert np.max(np.abs(x - y)) <= 1e-12 * np.max(np.abs(x)), f


def test_adaptive_queue_in_the_odw_step(mech):
    """Both adaptive forms through eu3d_step on a small ODW with its wedge
    (SSP-RK2: the chemistry finds the state decoded)."""
    from eu3d_b200 import surrogate as S
    from eu3d_b200.cases import odw_case, setup_odw
    case = odw_case(mech, 96, 48, 4, L=0.2 * 95 / 511.0)
    out = []
    for q in (0, 1):
        d = gpu.DeviceFlowfield(mech, case.grid, QUIRKS_FIXED, flux_bits=32)
        setup_odw(d, case)
        d.set_elements(S.atoms_matrix(mech))
        d.set_tuning(adapt_queue=q)
        d.run(30, react=gpu.REACT_ADAPTIVE, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.5)
        d.synchronize()
        out.append(({f: interior(d.download(f)) for f in ("CS", "T")}, d.status()))
        d.close()
    (a, sa), (b, sb) = out
    assert sa["substeps"] == sb["substeps"] and sa["nonfinite_cells"] == sb["nonfinite_cells"] == 0
    for f in ("CS", "T"):
        assert np.max(np.abs(a[f] - b[f])) <= 1e-10 * np.max(np.abs(a[f])), f


@pytest.mark.parametrize("stage", [0, 1, 2])
def test_flux_kernels_with_wedge_match_oracle(mech, stage):
    """With the wedge on, the flux kernels skip the tiles with no fluid cell:
    every fluid cell's residual is still formed -- FP64 against the oracle
    to 1e-12 of the flux scale, the three FP32 kernels bit for bit alike."""
    g = small_grid(72, 40, 6, lx=0.072, ly=0.04, lz=0.006)
    o = Oracle(mech, g, QUIRKS_FIXED)
    fill_state(o, 7, 1100.0, 2600.0)
    wedge = np.array([0.012, 0.0, np.tan(np.radians(25.0))])
    x = g.xnode[2:-2][:, None, None]
    y = g.ynode[2:-2][None, :, None]
    fluid = np.broadcast_to(~((x > wedge[0]) & (y - wedge[1] < (x - wedge[0]) * wedge[2])), (g.ni, g.nj, g.nk))
    assert (~fluid).sum() > 0.25 * fluid.size
    o.boundary(gpu.BC_RSBI, wedge)
    o.dt = 2e-8
    o.advection(0, gpu.DIFF_MUSCL2)
    ref = interior(o.view("RHS"))
    res = {}
    for bits, st in ((64, 0), (32, stage)):
        d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=bits)
        d.upload_state(o)
        d.set_wedge(*wedge)
        d.set_tuning(flux_stage=st)
        d.boundary(gpu.BC_RSBI)
        d.dt = 2e-8
        d.advection(gpu.ADV_EE, gpu.DIFF_MUSCL2)
        res[bits] = interior(d.download("RHS"))
        d.close()
    cs = interior(o.view("CS"))
    for v in range(ref.shape[-1]):
        scale = np.max(np.abs(cs[..., v][fluid])) * 1e-3 + np.max(np.abs(ref[..., v][fluid]))
        assert np.max(np.abs(res[64][..., v][fluid] - ref[..., v][fluid])) / scale < 1e-12, v
        assert np.max(np.abs(res[32][..., v][fluid] - ref[..., v][fluid])) / scale < 1e-4, v
    if stage == 2:
        # the kernels of one precision agree with each other: the FP32 result
        # of this stage equals the others' (checked pairwise by the three
        # parametrised runs against the FP64 reference above and here exactly)
        d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=32)
        d.upload_state(o)
        d.set_wedge(*wedge)
        d.set_tuning(flux_stage=0)
        d.boundary(gpu.BC_RSBI)
        d.dt = 2e-8
        d.advection(gpu.ADV_EE, gpu.DIFF_MUSCL2)
        assert np.array_equal(interior(d.download("RHS"))[fluid], res[32][fluid])
        d.close()


def test_stage_update_occupancy_gives_the_same_bits(mech):
    """The SSP-RK2 stage updates compiled for 3 and 4 resident blocks per SM
    (tuning cell_blocks) are the same arithmetic: identical state after a
    few steps of the ODW with its wedge."""
    from eu3d_b200.cases import odw_case, setup_odw
    case = odw_case(mech, 96, 48, 4, L=0.2 * 95 / 511.0)
    out = []
    for cb in (3, 4):
        d = gpu.DeviceFlowfield(mech, case.grid, QUIRKS_FIXED, flux_bits=32)
        setup_odw(d, case)
        d.set_tuning(cell_blocks=cb)
        assert d.tuning()["cell_blocks"] == cb
        d.run(8, react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.5)
        d.synchronize()
        out.append({f: d.download(f) for f in ("CS", "T", "P")})
        d.close()
    for f in ("CS", "T", "P"):
        assert np.array_equal(out[0][f], out[1][f]), f
    with pytest.raises(gpu.Eu3dError):
        d2 = gpu.DeviceFlowfield(mech, case.grid, QUIRKS_FIXED, flux_bits=32)
        try:
            d2.set_tuning(cell_blocks=6)
        finally:
            d2.close()
