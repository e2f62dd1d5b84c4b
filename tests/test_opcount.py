"""The operation-counting restatement of the per-cell chemistry
(oracle/opcount.py) against the C oracle: with plain floats it reproduces
Diagonalized's source and Jacobian diagonal, the IMEX update and the decode
of the oracle bit for bit, so its counts are those of the reference's
arithmetic; and the counts themselves are stable and plausible."""
import numpy as np

import opcount as oc
from _cases import QUIRKS_FIXED, make_oracle


def _cells(o, n=6):
    b = o.bc
    return [(b + i, b + 1, b + 1) for i in range(n)]


def test_restatement_reproduces_the_oracle(mech):
    o, g = make_oracle(mech, seed=51, quirks=QUIRKS_FIXED, tlo=900.0, thi=2600.0, radicals=1e-3)
    o.update_after_cs()
    o.partial_t()
    o.view("RHS")[...] = 1e-6 * o.view("CS")
    o.dt = 2e-8
    before = {n: o.view(n).copy() for n in ("CS", "RHS", "T", "Partion_T", "Di", "Mc")}
    o.lib().orc_diagonalized(*o._fm())
    CMS_o, MD_o = o.view("CMS").copy(), o.view("MDd").copy()
    o.lib().orc_update_imex(*o._fm())
    m = oc.Mech(mech)
    NS = mech.NS
    for c in _cells(o):
        cms, md = oc.diagonalized(m, before["Di"][c].tolist(), before["Mc"][c].tolist(), float(before["T"][c]),
                                  before["Partion_T"][c][:NS].tolist())
        assert np.array_equal(np.array(cms), CMS_o[c]), c
        assert np.array_equal(np.array(md), MD_o[c][:NS]), c
        out, st, pt, it = oc.imex_cell(m, before["CS"][c].tolist(), before["RHS"][c].tolist(), float(before["T"][c]),
                                       before["Partion_T"][c][:NS].tolist(), 2e-8)
        assert np.array_equal(np.array(out), o.view("CS")[c]), c
        assert st["T"] == o.view("T")[c] and 1 <= it <= 10
        assert np.array_equal(np.array(pt), o.view("Partion_T")[c][:NS]), c


def test_counts(mech):
    o, g = make_oracle(mech, seed=52, quirks=QUIRKS_FIXED, tlo=1100.0, thi=2600.0, radicals=1e-3)
    o.update_after_cs()
    o.partial_t()
    c = _cells(o, 1)[0]
    NS = mech.NS
    t = oc.count_imex(mech, o.view("CS")[c].tolist(), [0.0] * (NS + 4), float(o.view("T")[c]),
                      o.view("Partion_T")[c][:NS].tolist(), 2e-8)
    # 19 reactions x 9 species of rate products, the Jacobian's 171 terms,
    # the thermo polynomials: thousands of FLOPs, a few hundred transcendentals
    assert 3000 < t.flops < 20000, t
    # exp of the Arrhenius factor and of the equilibrium constant per reaction;
    # pow only where the temperature exponent is not an integer
    assert t["exp"] == 2 * mech.NR
    assert t["pow"] == sum(1 for b in mech.bf if b != int(b))
    assert t["log"] >= 2 * NS
    s = oc.count_adaptive_substep(mech, o.view("CS")[c].tolist(), float(o.view("T")[c]), 2e-8)
    assert 2000 < s.flops < 20000
    assert t.flops_with_transcendentals() > t.flops


def test_bench_constants_match_the_count(mech):
    """bench.py's CHEM_FLOP figures are reference_counts' averages."""
    import bench
    r = oc.reference_counts(mech, n=64, seed=0, newton=2)
    assert abs(r["imex_cell"]["flops"] - bench.CHEM_FLOP["imex_cell"]) < 0.5
    assert abs(r["imex_cell"]["flops_equiv"] - bench.CHEM_FLOP["imex_cell_equiv"]) < 0.5
    assert abs(r["adaptive_substep"]["flops"] - bench.CHEM_FLOP["adaptive_substep"]) < 0.5
    assert abs(r["adaptive_substep"]["flops_equiv"] - bench.CHEM_FLOP["adaptive_substep_equiv"]) < 0.5
