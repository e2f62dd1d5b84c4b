"""x-slab decomposition on the GPU: slabs of one flowfield, each its own
handle, stepped through eu3d_b200.slabs (halo pack/unpack kernels, local CFL
and time update, the parts of eu3d_step) with the in-process loopback
transport give the single-domain CUDA-graph step's result bit for bit.
Flowfield::Mpi_Boundary, src/Flowfield.cpp:775-1083."""
import numpy as np
import pytest

from _slab_cases import dyadic_grid
from eu3d_b200 import gpu
from eu3d_b200 import surrogate as S
from eu3d_b200.cases import STATE_FIELDS, odw_case, setup_odw
from eu3d_b200.slabs import DeviceSlab, LoopbackTransport, SlabRun, StepSpec, slab_extents, slab_grid

pytestmark = pytest.mark.gpu


def _cut(full, mech, grid, nranks, layout, flux_bits, setup=None):
    out = []
    for i0, n in slab_extents(grid.ni, nranks, layout):
        d = gpu.DeviceFlowfield(mech, slab_grid(grid, i0, n), gpu.QUIRKS_FIXED, flux_bits=flux_bits)
        if setup:
            setup(d)
        for f in STATE_FIELDS:
            d.upload(f, full.download(f)[i0:i0 + n + 2 * grid.bc])
        d.dt = full.dt
        d.set_time(full.time)
        d.synchronize()
        out.append((i0, n, d))
    return out


def _compare(full, pieces, bc=2, names=("CS", "T", "P", "Yi")):
    ref = {f: full.download(f) for f in names}
    for i0, n, d in pieces:
        for f in names:
            a = d.download(f)[bc:-bc, bc:-bc, bc:-bc]
            b = ref[f][bc:-bc, bc:-bc, bc:-bc][i0:i0 + n]
            assert np.all(np.isfinite(b)), f
            assert np.array_equal(a, b), (f, i0, n, float(np.max(np.abs(a - b))))
        assert d.dt == full.dt and d.time == full.time
        assert d.status()["wait_timeouts"] == 0


@pytest.mark.parametrize("nranks,layout,flux_bits,timeadv", [
    (3, "partition", 64, gpu.ADV_EE),
    (2, "partition", 32, gpu.ADV_SSPRK2),
    (3, "reference", 32, gpu.ADV_SSPRK2),
    (2, "partition", 64, gpu.ADV_SSPRK3),
    (3, "reference", 32, gpu.ADV_SSPRK3),
])
def test_rsbi_slabs_equal_single_domain(mech, nranks, layout, flux_bits, timeadv):
    from _cases import fill_state
    from pyoracle import Oracle
    ni = 97 if layout == "reference" else 96
    g = dyadic_grid(ni, 20, 9)
    o = Oracle(mech, g, gpu.QUIRKS_FIXED)
    fill_state(o, 7, 1100.0, 2600.0)
    full = gpu.DeviceFlowfield(mech, g, gpu.QUIRKS_FIXED, flux_bits=flux_bits)
    full.upload_state(o)
    full.dt = 1e-8
    pieces = _cut(full, mech, g, nranks, layout, flux_bits)
    spec = StepSpec(react=gpu.REACT_IMEX, timeadv=timeadv, bc_kind=gpu.BC_RSBI, cfl=0.5, final_time=1.0)
    slabs = [DeviceSlab(d, r, nranks, overlap=1 if layout == "reference" else 0) for r, (_, _, d) in enumerate(pieces)]
    run = SlabRun(slabs, LoopbackTransport())
    for _ in range(3):
        full.step(**spec.kw())
        run.step(spec)
    full.synchronize()
    for _, _, d in pieces:
        d.synchronize()
    _compare(full, pieces)


@pytest.mark.parametrize("react", [gpu.REACT_IMEX, gpu.REACT_SURROGATE])
def test_odw_wedge_slabs_equal_single_domain(mech, react):
    """Inflow / wall x faces on the end slabs only, the immersed wedge across
    every slab face (band refilled after the exchange), SSP-RK2, FP32 flux;
    with the learned chemistry and its FP64 fallback as well."""
    case = odw_case(mech, 128, 48, 6, L=0.05)
    model = S.SurrogateModel.load(S.DEFAULT_MODEL) if react == gpu.REACT_SURROGATE else None

    def setup(d):
        setup_odw(d, case)
        if model is not None:
            d._model_sur = model.attach(d, 0)

    full = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=32)
    setup(full)
    spec = StepSpec(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0, final_time=1.0)
    full.dt = 4e-8
    # develop a flow with the wedge shock first (one domain), then split it
    for _ in range(30):
        full.step(**spec.kw())
    full.synchronize()
    pieces = _cut(full, mech, case.grid, 3, "partition", 32, setup)
    spec.react = react
    slabs = [DeviceSlab(d, r, 3, wedge=True) for r, (_, _, d) in enumerate(pieces)]
    run = SlabRun(slabs, LoopbackTransport())
    for _ in range(4):
        full.step(**spec.kw())
        run.step(spec)
    full.synchronize()
    for _, _, d in pieces:
        d.synchronize()
    _compare(full, pieces)
    if react == gpu.REACT_SURROGATE:
        assert sum(d.status()["surrogate_cells"] for _, _, d in pieces) == full.status()["surrogate_cells"]


def test_halo_pack_unpack_roundtrip(mech):
    """pack(side) of one slab unpacked into the other side's ghosts of a copy
    puts exactly the planes next to the face there (all fields, ghost rows
    included); overlap 1 skips the shared end plane."""
    from _cases import fill_state
    from pyoracle import Oracle
    g = dyadic_grid(12, 6, 5)
    o = Oracle(mech, g, gpu.QUIRKS_FIXED)
    fill_state(o, 11, 900.0, 2000.0)
    import torch
    for bits in (32, 64):
        a = gpu.DeviceFlowfield(mech, g, gpu.QUIRKS_FIXED, flux_bits=bits)
        a.upload_state(o)
        buf = torch.empty(a.halo_bytes(), dtype=torch.uint8, device="cuda")
        for overlap in (0, 1):
            for side in (0, 1):
                a.halo_pack(side, buf.data_ptr(), overlap)
                b = gpu.DeviceFlowfield(mech, g, gpu.QUIRKS_FIXED, flux_bits=bits)
                b.upload_state(o)
                b.halo_unpack(1 - side, buf.data_ptr())
                b.synchronize()
                src = slice(2 + overlap, 4 + overlap) if side == 0 else slice(g.ni - overlap, g.ni + 2 - overlap)
                dst = slice(g.ni + 2, g.ni + 4) if side == 0 else slice(0, 2)
                for f in ("D", "U", "P", "T", "E", "H", "Gamma", "Yi"):
                    assert np.array_equal(b.download(f)[dst], a.download(f)[src]), (bits, overlap, side, f)
                b.close()
        a.close()
    with pytest.raises(gpu.Eu3dError):
        gpu.DeviceFlowfield(mech, g, gpu.QUIRKS_FIXED).halo_pack(2, buf.data_ptr())


def _dlb_run(full, pieces, spec, steps, wedge=False):
    slabs = [DeviceSlab(d, r, len(pieces), wedge=wedge) for r, (_, _, d) in enumerate(pieces)]
    run = SlabRun(slabs, LoopbackTransport())
    plans = []
    for _ in range(steps):
        full.step(**spec.kw())
        run.step(spec)
        plans.append(slabs[0].last_plan)
    full.synchronize()
    for _, _, d in pieces:
        d.synchronize()
    return slabs, plans


@pytest.mark.parametrize("flux_bits", [64, 32])
def test_dlb_trapezoid_slabs_equal_single_domain(mech, flux_bits):
    """The adaptive trapezoid balanced across three slabs (the most loaded
    slab hands rows to the others: packets out, substeps on the receivers,
    results back) gives the unbalanced single domain bit for bit, counts
    included; the substeps counted over the slabs equal the single domain's.
    (The state stays finite under this trapezoid form for the two steps, as
    the oracle shows; hotter ones do not.)"""
    from _cases import fill_state
    from pyoracle import Oracle
    g = dyadic_grid(96, 20, 9)
    o = Oracle(mech, g, gpu.QUIRKS_FIXED)
    fill_state(o, 7, 1200.0, 1800.0, radicals=1e-5)
    o.view("T")[:36] += 200.0  # more substeps in the first slab
    o.prims_from_state()
    full = gpu.DeviceFlowfield(mech, g, gpu.QUIRKS_FIXED, flux_bits=flux_bits)
    full.upload_state(o)
    full.dt = 1e-8
    pieces = _cut(full, mech, g, 3, "partition", flux_bits)
    spec = StepSpec(react=gpu.REACT_TRAPEZOID, type_=1, bc_kind=gpu.BC_RSBI, cfl=0.0, final_time=1.0, dlb=True)
    full.reset_status()
    for _, _, d in pieces:
        d.reset_status()
    slabs, plans = _dlb_run(full, pieces, spec, 2)
    _compare(full, pieces, names=("CS", "T", "P", "Yi", "Nchem", "E"))
    # step 1 predicts one substep everywhere (balanced); step 2 balances
    assert plans[0] == [] and plans[1] and plans[1][0][0] == 0, plans
    assert sum(slabs[0].counts[t] for t in slabs[0].mine) > 0
    assert sum(d.status()["substeps"] for _, _, d in pieces) == full.status()["substeps"]
    assert all(d.status()["wait_timeouts"] == 0 for _, _, d in pieces)


def test_dlb_odw_wedge_slabs_equal_single_domain(mech):
    """Balancing with the immersed wedge: solid cells travel in the packets
    unintegrated and are left untouched on return."""
    case = odw_case(mech, 128, 48, 6, L=0.05)
    full = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=32)
    setup_odw(full, case)
    full.dt = 4e-8
    warm = StepSpec(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0, final_time=1.0)
    for _ in range(30):
        full.step(**warm.kw())
    full.synchronize()
    pieces = _cut(full, mech, case.grid, 3, "partition", 32, lambda d: setup_odw(d, case))
    spec = StepSpec(react=gpu.REACT_TRAPEZOID, type_=1, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0,
                    final_time=1.0, dlb=True)
    _, plans = _dlb_run(full, pieces, spec, 2, wedge=True)
    _compare(full, pieces, names=("CS", "T", "P", "Yi", "Nchem"))
    assert any(plans), plans


@pytest.mark.parametrize("flux_bits", [32, 64])
def test_dlb_surrogate_fallback_slabs_equal_single_domain(mech, flux_bits):
    """The learned chemistry's FP64 fallback balanced across three slabs with
    the immersed wedge: every accepted cell is audited (audit stride 1, the
    same cells on the slabs as on the single domain), so each slab's fallback
    list holds its fluid cells and the slabs the wedge takes cells from carry
    less.  The loaded slab hands the last cells of its list to the others,
    which integrate them and send them back -- bit for bit the unbalanced
    single domain; the fallback, audit and substep counts summed over the
    slabs equal the single domain's, and so does the largest audit
    difference."""
    case = odw_case(mech, 128, 48, 6, L=0.05)
    model = S.SurrogateModel.load(S.DEFAULT_MODEL)

    def setup(d):
        setup_odw(d, case)
        d._model_sur = model.attach(d, 1)

    full = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=flux_bits)
    setup(full)
    warm = StepSpec(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0, final_time=1.0)
    full.dt = 4e-8
    for _ in range(30):
        full.step(**warm.kw())
    full.synchronize()
    pieces = _cut(full, mech, case.grid, 3, "partition", flux_bits, setup)
    spec = StepSpec(react=gpu.REACT_SURROGATE, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0, final_time=1.0,
                    dlb=True)
    full.reset_status()
    for _, _, d in pieces:
        d.reset_status()
    slabs, plans = _dlb_run(full, pieces, spec, 2, wedge=True)
    _compare(full, pieces, names=("CS", "T", "P", "Yi", "E"))
    assert all(plans), plans
    assert plans[0][0][0] == 0, plans  # the inflow slab has no wedge cells: the most fallback
    assert sum(slabs[0].counts[t] for t in slabs[0].mine) > 0
    st = [d.status() for _, _, d in pieces]
    sf = full.status()
    for key in ("surrogate_fallback", "surrogate_audited", "surrogate_cells", "substeps", "newton_capped"):
        assert sum(x[key] for x in st) == sf[key], key
    assert max(x["surrogate_audit_max_dT"] for x in st) == sf["surrogate_audit_max_dT"]
    assert sf["surrogate_audited"] > 0


@pytest.mark.parametrize("flux_bits", [64, 32])
def test_weno_rk3_slabs_equal_single_domain(mech, flux_bits):
    """WENO + SSP-RK3 on three device slabs equal the single domain bit for bit."""
    from _cases import fill_state
    from pyoracle import Oracle
    g = dyadic_grid(96, 20, 9)
    o = Oracle(mech, g, gpu.QUIRKS_FIXED)
    fill_state(o, 7, 1100.0, 2600.0)
    full = gpu.DeviceFlowfield(mech, g, gpu.QUIRKS_FIXED, flux_bits=flux_bits)
    full.upload_state(o)
    full.dt = 1e-8
    pieces = _cut(full, mech, g, 3, "partition", flux_bits)
    spec = StepSpec(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK3, diff=gpu.DIFF_WENO, bc_kind=gpu.BC_RSBI, cfl=0.5,
                    final_time=1.0)
    slabs = [DeviceSlab(d, r, 3) for r, (_, _, d) in enumerate(pieces)]
    run = SlabRun(slabs, LoopbackTransport())
    for _ in range(3):
        full.step(**spec.kw())
        run.step(spec)
    full.synchronize()
    for _, _, d in pieces:
        d.synchronize()
    _compare(full, pieces)


def test_sdlb_entry_points_reject_misuse(mech):
    """The fallback balancing calls refuse what they cannot do: a fallback
    list length without a list, a selection before the list's length was
    read, a guest without an attached network; packing and unpacking with
    nothing selected are no-ops."""
    case = odw_case(mech, 32, 16, 4, L=0.05 * 31 / 127)
    d = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=32)
    setup_odw(d, case)
    with pytest.raises(gpu.Eu3dError):
        d.sur_load()
    with pytest.raises(gpu.Eu3dError):
        d.sdlb_select([-1])
    with pytest.raises(gpu.Eu3dError):
        d.sdlb_select([])  # no eu3d_sur_load yet
    with pytest.raises(gpu.Eu3dError):
        d.sdlb_guest([4], 0, 0)
    d.sdlb_pack(0)    # nothing selected: no packet, no pointer needed
    d.sdlb_unpack(0)
    d.close()
