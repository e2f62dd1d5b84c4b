"""Failure detection on the GPU without a GPU fault, through the C ABI.

The reference aborts when its state goes NaN (src/Euler.cpp:319-331) or a
substep count is not positive (src/Reaction.cpp:664-668), and its Newton
temperature inversion silently returns the tenth iterate
(src/Flowfield.cpp:1542-1566).  Here every such event is a status counter
the host reads after the step; kernels never trap.  Each test provokes its
event from the host: a state whose energy the Newton inversion cannot reach
in ten iterations, a substep cap of one, and a wait bound of zero on the
TMA-fed flux kernel, which must then count the timeout, let its copies land
and return, leaving the context usable."""
import numpy as np
import pytest

from _cases import QUIRKS_FIXED, interior, make_oracle, rel_err
from eu3d_b200 import gpu
from eu3d_b200 import surrogate as S
from eu3d_b200.cases import complete_state, odw_case, setup_odw

pytestmark = pytest.mark.gpu

HOT = dict(tlo=1100.0, thi=2600.0)


def test_newton_cap_is_counted_and_matches_the_reference_iterate(mech):
    """Cells of stoichiometric H2-air at rest whose internal energy belongs to
    9500 K, decoded from a 300 K start: beyond the polynomials' range the
    Newton inversion overshoots, is still moving by thousands of kelvin at
    its tenth iteration and keeps that iterate, as Get_temp does (the host
    restatement of the iteration, oracle/opcount.py, shows the same for
    starts 0.1 K either side, so the count is not a rounding accident).  The
    status counts every such cell, nothing goes non-finite, and the iterate
    agrees with the oracle's."""
    from eu3d_b200.readers import stoichiometric_h2_air
    o, g = make_oracle(mech, seed=31, quirks=QUIRKS_FIXED, **HOT)
    sl = (slice(3, 6), slice(2, 5), slice(2, 4))  # 18 interior cells
    Y = np.broadcast_to(stoichiometric_h2_air(mech), o.view("Yi")[sl].shape)
    z = np.zeros(Y.shape[:-1])
    hot = complete_state(mech, z + 101325.0, z + 9500.0, z, z, z, Y)
    o.view("CS")[sl] = hot["CS"]
    o.view("T")[sl] = 300.0
    d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=64)
    d.upload_state(o)
    d.reset_status()
    d.update_after_cs()
    o.update_after_cs()
    st = d.status()
    assert st["newton_capped"] == 18, st
    assert st["nonfinite_cells"] == 0
    T = d.download("T")[sl]
    assert np.all(np.isfinite(T)) and np.all(T > 20000.0)  # far from 9500 K: not converged
    assert np.max(np.abs(T / o.view("T")[sl] - 1.0)) < 1e-8
    d.close()


def test_adaptive_substep_cap_is_counted(mech):
    """The adaptive chemistry with at most one substep on reacting states:
    every cell whose controller wanted a shorter step is counted in
    substep_capped; with the default cap of 1024 none is."""
    o, g = make_oracle(mech, seed=32, quirks=QUIRKS_FIXED, radicals=1e-3, **HOT)
    counts = {}
    for nmax in (1024, 1):
        d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=64)
        d.upload_state(o)
        d.upload("RHS", np.zeros(d.shape("RHS")))
        d.set_elements(S.atoms_matrix(mech))
        d.set_adaptive(nmax=nmax)
        d.dt = 3e-8
        d.reset_status()
        d.react_adaptive()
        st = d.status()
        counts[nmax] = st
        assert st["nonfinite_cells"] == 0
        assert np.all(np.isfinite(interior(d.download("T"))))
        d.close()
    n = g.ni * g.nj * g.nk
    assert counts[1024]["substep_capped"] == 0
    assert counts[1024]["substeps"] > n  # the controller subdivides these states
    assert 0 < counts[1]["substep_capped"] <= n
    assert counts[1]["substeps"] == n


def test_flux_wait_timeout_returns_and_context_stays_usable(mech):
    """Wait bound 0 on the TMA-fed flux kernel: every block gives up at its
    first wait, counts it, waits (with the full bound) for its copies in
    flight and returns.  The status shows the timeouts and no failed drain;
    with the bound restored the same handle computes the residual of a fresh
    handle bit for bit."""
    case = odw_case(mech, 96, 48, 16, L=0.2 * 95 / 511.0)
    ds = []
    for _ in range(2):
        d = gpu.DeviceFlowfield(mech, case.grid, QUIRKS_FIXED, flux_bits=32)
        setup_odw(d, case)
        assert d.tuning()["flux_stage"] == 2  # the TMA ring kernel
        d.boundary(gpu.BC_ODM)
        d.dt = 5e-8
        ds.append(d)
    a, b = ds
    a.set_wait_limit(0)
    a.reset_status()
    a.advection(gpu.ADV_EE, gpu.DIFF_MUSCL2)
    a.synchronize()
    st = a.status()
    assert st["wait_timeouts"] > 0, st
    assert st["drain_timeouts"] == 0, st
    assert st["nonfinite_cells"] == 0
    a.set_wait_limit()
    a.reset_status()
    a.advection(gpu.ADV_EE, gpu.DIFF_MUSCL2)
    b.advection(gpu.ADV_EE, gpu.DIFF_MUSCL2)
    assert a.status()["wait_timeouts"] == 0
    assert np.array_equal(interior(a.download("RHS")), interior(b.download("RHS")))
    # a whole step after the timeout: finite and counted clean
    a.step(react=gpu.REACT_IMEX, timeadv=gpu.ADV_SSPRK2, bc_kind=gpu.BC_ODM, cfl=0.5)
    a.synchronize()
    st = a.status()
    assert st["wait_timeouts"] == 0 and st["nonfinite_cells"] == 0
    for d in ds:
        d.close()


def test_wait_limit_argument_errors(mech):
    o, g = make_oracle(mech, seed=33, quirks=QUIRKS_FIXED, **HOT)
    d = gpu.DeviceFlowfield(mech, g, QUIRKS_FIXED, flux_bits=32)
    with pytest.raises(gpu.Eu3dError):
        d.set_wait_limit(-1)
    with pytest.raises(gpu.Eu3dError):
        d.set_wait_limit(1 << 25)
    d.close()
