"""Frozen-chemistry gate of the learned surrogate step on the GPU, through the
C ABI: with the gate on, only the listed (active) cells go through the
network and its apply.

* a gate that freezes nothing gives the ungated step's decisions, counters
  and conserved state;
* with the coupled runs' gate (600 K, radicals <= 1e-6) the frozen cells keep
  the state of the step's flux stages alone, bit for bit, while the audit
  shows that the FP64 integrator would have changed their temperature by far
  less than a millikelvin;
* every fluid cell is counted once: accepted, fallen back, audited or frozen.
"""
import numpy as np
import pytest

from eu3d_b200 import gpu
from eu3d_b200 import surrogate as S
from eu3d_b200.cases import odw_case, setup_odw

pytestmark = pytest.mark.gpu

KW = dict(timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.0, final_time=1.0)


def _developed(mech, case, flux_bits):
    d = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=flux_bits)
    setup_odw(d, case)
    d.set_elements(S.atoms_matrix(mech))
    d.dt = 4e-8
    d.run(40, react=gpu.REACT_IMEX, **KW)
    d.synchronize()
    return d


def _fluid(case):
    g = case.grid
    x = g.xnode[2:-2][:, None, None]
    y = g.ynode[2:-2][None, :, None]
    w = case.wedge
    solid = (x > w[0]) & ((y - w[1]) < (x - w[0]) * w[2])
    return np.broadcast_to(~solid, (g.ni, g.nj, g.nk))


@pytest.mark.parametrize("flux_bits", [32, 64])
def test_gate_that_freezes_nothing_equals_ungated_step(mech, flux_bits):
    case = odw_case(mech, 160, 64, 3, L=0.05)
    m0 = S.SurrogateModel.load(S.DEFAULT_MODEL)
    norm = m0.norm.copy()
    norm[S.N_ENV + 0] = 320.0  # the 300 K free stream leaves the envelope: it falls back
    model = S.SurrogateModel(m0.params, norm, m0.meta)
    out = []
    for gate in (None, dict(t_frozen=1.0)):
        d = _developed(mech, case, flux_bits)
        s = model.attach(d, 7, gate=gate)
        d.run(3, react=gpu.REACT_SURROGATE, **KW)
        d.synchronize()
        out.append(({f: d.download(f) for f in ("CS", "T", "E", "P", "Yi")}, d.status()))
        d.set_surrogate(None)
        s.close()
        d.close()
    (a, sa), (b, sb) = out
    assert sa["surrogate_cells"] > 0 and sa["surrogate_fallback"] > 0, sa
    assert sb["surrogate_frozen"] == 0
    for k in ("surrogate_cells", "surrogate_fallback", "surrogate_rejects", "surrogate_audited", "nonfinite_cells"):
        assert sa[k] == sb[k], k
    # the list kernels inline the same per-cell apply; FP32 primitives round a
    # decode's last-bit contraction difference away before the next flux
    for f in ("CS", "Yi"):
        if flux_bits == 32:
            assert np.array_equal(a[f], b[f]), f
        else:
            assert np.max(np.abs(a[f] - b[f])) <= 1e-10 * np.max(np.abs(a[f])), f
    for f in ("T", "E", "P"):
        assert np.max(np.abs(a[f] - b[f]) / np.maximum(np.abs(a[f]), 1e-300)) <= 1e-8, f


def test_frozen_cells_keep_the_flux_update_and_are_audited(mech):
    case = odw_case(mech, 160, 64, 3, L=0.05)
    model = S.SurrogateModel.load(S.DEFAULT_MODEL)
    gate = dict(S.GATE, audit_stride=7)
    res = {}
    for name in ("gated", "stages"):
        d = _developed(mech, case, 32)
        T0 = d.download("T")[2:-2, 2:-2, 2:-2].copy()
        if name == "gated":
            s = model.attach(d, 0, gate=gate)
            d.reset_status()
            d.step(react=gpu.REACT_SURROGATE, **KW)
        else:
            # the same step's ghost fills and SSP-RK2 stages, without its chemistry
            spec = dict(react=gpu.REACT_IMEX, **KW)  # the stages do not depend on the chemistry
            d.boundary(gpu.BC_ODM)
            d.step_part(gpu.PART_STAGE1, **spec)
            d.boundary(gpu.BC_ODM)
            d.step_part(gpu.PART_STAGE2, **spec)
        d.synchronize()
        res[name] = ({f: d.download(f)[2:-2, 2:-2, 2:-2].copy() for f in ("CS", "T", "Yi")}, d.status(), T0)
        if name == "gated":
            d.set_surrogate(None)
            s.close()
        d.close()
    (g, st, T0), (n, _, _) = res["gated"], res["stages"]
    fluid = _fluid(case)
    # the gate's decision from the state the stages leave: T below 600 K and
    # the radicals' mass fractions (FP32 primitives, summed in FP32 in species
    # order) <= 1e-6
    rad = sorted(mech.species.index(r) for r in gate["species"])
    yr = np.zeros(n["T"].shape, np.float32)
    for r in rad:
        yr = yr + np.maximum(n["Yi"][..., r].astype(np.float32), np.float32(0))
    frozen = fluid & (n["T"] < gate["t_frozen"]) & (yr <= np.float32(gate["y_max"]))
    assert frozen.sum() > 0.2 * fluid.sum()
    assert st["surrogate_frozen"] == frozen.sum(), (st["surrogate_frozen"], frozen.sum())
    # every fluid cell counted once
    assert st["surrogate_cells"] + st["surrogate_fallback"] + st["surrogate_audited"] + st["surrogate_frozen"] \
        == fluid.sum(), st
    assert st["frozen_audited"] > 0
    assert st["frozen_audit_max_dT"] < 1e-3, st["frozen_audit_max_dT"]
    # frozen cells keep the stages' state bit for bit (audited ones are
    # integrated by the fallback, which keeps its result)
    ni, nj, nk = case.grid.ni, case.grid.nj, case.grid.nk
    idx = np.arange(ni * nj * nk, dtype=np.uint64).reshape(nk, nj, ni).transpose(2, 1, 0)
    sampled = ((idx * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) < np.uint64(0xFFFFFFFF // gate["audit_stride"])
    assert st["frozen_audited"] == (frozen & sampled).sum()
    keep = frozen & ~sampled
    for f in ("CS", "T"):
        assert np.array_equal(g[f][keep], n[f][keep]), f
    assert st["nonfinite_cells"] == 0
    del T0


def test_gate_argument_errors(mech):
    case = odw_case(mech, 32, 16, 2, L=0.02)
    d = gpu.DeviceFlowfield(mech, case.grid, gpu.QUIRKS_FIXED, flux_bits=32)
    with pytest.raises(gpu.Eu3dError):
        d.set_surrogate_gate(-1.0)
    with pytest.raises(gpu.Eu3dError):
        d.set_surrogate_gate(600.0, -1e-6)
    with pytest.raises(gpu.Eu3dError):
        d.set_surrogate_gate(600.0, 1e-6, audit_stride=-1)
    d.close()


@pytest.mark.parametrize("flux_bits", [32, 64])
def test_gate_fused_into_stage2_equals_gate_kernel(mech, flux_bits):
    """The gate inside SSP-RK2's stage 2 (tuning gate_fused 1, the default)
    takes the separate gate kernel's decisions on the state the stage has
    just decoded: the same counts (accepted, fallen back, rejected, audited,
    frozen) and the same state after three coupled steps."""
    case = odw_case(mech, 160, 64, 3, L=0.05)
    model = S.SurrogateModel.load(S.DEFAULT_MODEL)
    gate = dict(S.GATE, audit_stride=7)
    out = []
    for fused in (0, 1):
        d = _developed(mech, case, flux_bits)
        d.set_tuning(gate_fused=fused)
        assert d.tuning()["gate_fused"] == fused
        s = model.attach(d, 0, gate=gate)
        d.reset_status()
        d.run(3, react=gpu.REACT_SURROGATE, **KW)
        d.synchronize()
        out.append(({f: d.download(f) for f in ("CS", "T", "E", "P", "Yi")}, d.status()))
        d.set_surrogate(None)
        s.close()
        d.close()
    (a, sa), (b, sb) = out
    assert sa["surrogate_frozen"] > 0 and sa["frozen_audited"] > 0 and sa["surrogate_cells"] > 0, sa
    for k in ("surrogate_cells", "surrogate_fallback", "surrogate_rejects", "surrogate_audited", "surrogate_frozen",
              "frozen_audited", "frozen_audit_max_dT", "nonfinite_cells", "newton_capped"):
        assert sa[k] == sb[k], k
    for f in a:
        assert np.array_equal(a[f], b[f]), f
