"""Pins the oracle (the C restatement in oracle/) to the reference.

* against the reference's own published t = 0 RSBI fields (output_8, the only
  golden data the reference ships);
* against fixtures produced by running the compiled reference
  (tests/golden/ref_steps.npz, made by tests/golden/make_golden.py) -- the
  oracle must reproduce them bit for bit;
* live against the compiled reference (oracle/_ref) when it is present.
"""
import os

import numpy as np
import pytest

from _cases import QUIRKS_FIXED, QUIRKS_REF, interior, make_oracle
from eu3d_b200.readers import make_grid, read_mechanism
from pyoracle import Oracle, RefCase, copy_state

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
import golden.make_golden as mg  # noqa: E402

REF_INPUT = os.path.join(mg.REF_DIR, "input")  # the reference's input tables, when its tree is present


@pytest.mark.parametrize("case", mg.CASES, ids=[c[0] for c in mg.CASES])
def test_oracle_reproduces_reference_fixture(mech, case):
    name, quirks, react, typ, cfl, dt, steps, bc_kind, st = case
    gold = np.load(os.path.join(GOLD, "ref_steps.npz"))
    o, g = mg.case_state(mech, quirks, st)
    if bc_kind == 1:
        mg.set_inflow(o)
    for _ in range(steps):
        if cfl == 0:
            o.dt = dt
        o.step(react, typ, 0, 1, cfl, 1.0, bc_kind)
    for f in mg.OUT_FIELDS:
        assert np.array_equal(interior(o.view(f)), gold[f"{name}/{f}"], equal_nan=True), f
    assert np.array_equal(np.array([o.dt, o.time]), gold[f"{name}/dt_time"])
    if react == 0 and typ == 1:
        assert np.array_equal(interior(o.view("Nchem")).astype(np.float64), gold[f"{name}/Nchem"])


@pytest.mark.parametrize("rank", [0, 5])
def test_rsbi_initial_field_matches_published_output(mech, rank):
    """FieldInitial/ReactionInitial/Mesh of the shipped case vs the reference's
    output_8/resultsIMEX0_<rank>.dat (6 significant digits)."""
    gold = np.load(os.path.join(GOLD, "rsbi_t0.npz"))
    ref = gold[f"rank{rank}"]
    ni, nj, nk = gold[f"rank{rank}_shape"]
    g = make_grid(241, 0.0, 0.17, 81, 0.0, 0.08, 2, 0.0, 0.02, 2, blocks=(4, 2, 1), rank=(rank % 4, rank // 4, 0))
    assert (g.ni, g.nj, g.nk) == (ni, nj, nk)
    o = Oracle(mech, g, QUIRKS_REF)
    o.rsbi_initial(101325.0, 1000.0, 3.0)
    b = g.bc

    def block(a):  # interior, written k-outer, j, i-inner
        return np.transpose(a[b:-b, b:-b, b:-b], (2, 1, 0)).reshape(-1)

    X = np.broadcast_to(g.xnode[:, None, None], (o.NI, o.NJ, o.NK))
    Y = np.broadcast_to(g.ynode[None, :, None], (o.NI, o.NJ, o.NK))
    cols = [block(X), block(Y)] + [block(o.view(n)) for n in ("T", "D", "P", "U", "V")] + \
           [block(o.view("Yi")[..., s]) for s in range(7)]
    mine = np.stack(cols)
    np.testing.assert_allclose(mine, ref, rtol=6e-6, atol=1e-12)


def test_mechanism_reader_matches_reference():
    if not RefCase.available() or not os.path.isdir(REF_INPUT):
        pytest.skip("compiled reference or its input files absent")
    m = read_mechanism(REF_INPUT + "/H2_JA919.txt", REF_INPUT + "/thermo.dat")
    r = RefCase.read_mechanism(REF_INPUT + "/H2_JA919.txt", REF_INPUT + "/thermo.dat")
    assert (m.NS, m.NR, m.TB) == (r["NS"], r["NR"], r["TB"])
    for k in ("stoi_f", "stoi_b", "react_tb", "af", "bf", "eaf", "c0", "c1", "mw"):
        assert np.array_equal(getattr(m, k), r[k]), k


def test_packaged_mechanism_matches_input_files(mech):
    if not os.path.isdir(REF_INPUT):
        pytest.skip("reference input files absent")
    m = read_mechanism(REF_INPUT + "/H2_JA919.txt", REF_INPUT + "/thermo.dat")
    for k in ("stoi_f", "stoi_b", "react_tb", "af", "bf", "eaf", "c0", "c1", "mw"):
        assert np.array_equal(getattr(m, k), getattr(mech, k)), k


@pytest.mark.parametrize("fixed", [False, True])
def test_oracle_matches_reference_live(mech, fixed):
    """Longer live runs against the compiled reference: IMEX with CFL, five
    steps, and the thermo polynomials at both ranges."""
    if not RefCase.available(fixed):
        pytest.skip("compiled reference absent")
    quirks = QUIRKS_FIXED if fixed else QUIRKS_REF
    tl, th = (900.0, 2400.0) if fixed else (400.0, 990.0)
    o, g = make_oracle(mech, seed=23, quirks=quirks, tlo=tl, thi=th)
    rc = RefCase(mech, g, fixed=fixed)
    copy_state(o, rc)
    for _ in range(5):
        o.step(1, 0, 0, 1, 0.4, 1.0, 0)
        rc.cfl(0.4, 1.0)
        rc.boundary(0)
        rc.advection(0, 1)
        rc.imex()
    for n in ("CS", "T", "U", "V", "W", "P", "D", "H", "Gamma", "E", "Yi", "RHS"):
        assert np.array_equal(o.view(n), rc.view(n), equal_nan=True), n
    for T in (300.0, 999.9, 1000.0, 2500.0):
        for sp in range(mech.NS):
            assert o.getcpi(T, 1.0, sp) == rc.thermo(0, T, 1.0, sp)
            assert o.gethi(T, 8.31434, sp) == rc.thermo(1, T, 8.31434, sp)
            assert o.getsi(T, 8.31434, sp) == rc.thermo(2, T, 8.31434, sp)


def test_oracle_ref_policy_shipped_case_goes_nonfinite(mech):
    """The shipped RSBI case with the reference's own arithmetic (high-range
    b1/b2 defect) loses finiteness in the first step; the corrected policy
    stays finite.  This is the documented behaviour the policies encode."""
    g_ref = make_grid(41, 0.0, 0.17 * 40 / 240, 21, 0.0, 0.02, 2, 0.0, 0.02, 2)
    g_fix = make_grid(41, 0.0, 0.17 * 40 / 240, 21, 0.0, 0.02, 2, 0.0, 0.02, 2, fixed_ghosts=True)
    res = {}
    for q, g in ((QUIRKS_REF, g_ref), (QUIRKS_FIXED, g_fix)):
        o = Oracle(mech, g, q)
        o.rsbi_initial(101325.0, 1000.0, 3.0)
        for _ in range(2):
            o.step(1, 0, 0, 1, 0.1, 1.0, 0)
        res[q] = np.isfinite(interior(o.view("T"))).all()
    assert not res[QUIRKS_REF]
    assert res[QUIRKS_FIXED]
