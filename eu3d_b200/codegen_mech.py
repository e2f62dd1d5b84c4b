"""Generate mechanism-specialised device code (eu3d_b200/csrc/mech_h2_ja919.cuh).

    python -m eu3d_b200.codegen_mech

The generic kernels read the stoichiometric and Arrhenius tables from constant
memory and loop densely over 9 species x 19 reactions.  For the compiled-in
mechanism this script writes straight-line code instead: every coefficient is
a literal (hexadecimal, exact), each reaction touches only the species it
involves, and zero terms are dropped.  The arithmetic of each surviving term
is the reference's (src/Reaction.cpp:744-810, :416-482):

    KF  = A T^b exp(-Ea / (Ru T))
    Kp  = exp(-sum_s nu_s G_s / (R T)) (P0 1e-6)^Xr,  Kc = Kp (R T)^-Xr,  KB = KF / Kc
    RRF = prod_s Mc_s^nu'_s,  RRB = prod_s Mc_s^nu''_s,  R_TB = sum_s alpha_s Mc_s
    RR  = KF RRF - KB RRB

eu3d_create compares the handle's tables with the ones compiled in and uses
the specialised kernels only when they are identical.
"""
from __future__ import annotations

import os

import numpy as np

from .readers import load_h2_ja919

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "mech_h2_ja919.cuh")


def lit(x: float) -> str:
    """Exact C literal of a double (hexadecimal floating constant)."""
    x = float(x)
    if x == 0.0:
        return "0.0"
    return f"({x.hex()})" if x < 0 else x.hex()


def gen(mech) -> str:
    NS, NR = mech.NS, mech.NR
    sf, sb, tb = mech.stoi_f, mech.stoi_b, mech.react_tb
    L = []
    w = L.append
    w("// Generated by eu3d_b200/codegen_mech.py from the H2_JA919 mechanism and")
    w("// thermo.dat tables (do not edit).  Specialised rate evaluation for that")
    w("// mechanism; see the generator's docstring for the formulas.")
    w("#pragma once")
    w("")
    w('#include "common.cuh"')
    w("")
    w("namespace eu3d {")
    w("namespace h2ja919 {")
    w("")
    # table fingerprint for the run-time check
    w("// tables this code was generated from (compared at handle creation)")
    def arr(name, a):
        a = np.asarray(a, dtype=np.float64).reshape(-1)
        w(f"constexpr double {name}[{a.size}] = {{" + ", ".join(lit(x) for x in a) + "};")
    arr("K_STOI_F", sf)
    arr("K_STOI_B", sb)
    arr("K_TB", tb)
    arr("K_AF", mech.af)
    arr("K_BF", mech.bf)
    arr("K_EAF", mech.eaf)
    arr("K_C0", mech.c0)
    arr("K_C1", mech.c1)
    arr("K_MW", mech.mw)
    w("")

    # thermo: per-species H/R and S/R, Cp/R with literal coefficients
    w("// H/R, S/R of species s at p (both NASA-9 ranges as literals)")
    for kind in ("h", "s", "cp"):
        w(f"template <int S> __device__ __forceinline__ double {kind}_r_spec(const TPow &p);")
    for s in range(NS):
        for kind in ("h", "s", "cp"):
            def poly(c, b):
                c = [lit(v) for v in c]
                if kind == "h":
                    return (f"-{c[0]} * p.tm1 + {c[1]} * p.lnT + {c[2]} * p.T + {c[3]} * p.t2 * 0.5 + "
                            f"{c[4]} * p.t3 * (1.0 / 3.0) + {c[5]} * p.t4 * 0.25 + {c[6]} * p.t5 * 0.2 + {b}")
                if kind == "s":
                    return (f"-{c[0]} * p.tm2 * 0.5 - {c[1]} * p.tm1 + {c[2]} * p.lnT + {c[3]} * p.T + "
                            f"{c[4]} * p.t2 * 0.5 + {c[5]} * p.t3 * (1.0 / 3.0) + {c[6]} * p.t4 * 0.25 + {b}")
                return (f"{c[0]} * p.tm2 + {c[1]} * p.tm1 + {c[2]} + {c[3]} * p.T + {c[4]} * p.t2 + "
                        f"{c[5]} * p.t3 + {c[6]} * p.t4")
            bi = 7 if kind == "h" else 8
            lo = poly(mech.c0[:7, s], lit(mech.c0[bi, s]))
            hi_b = f"(p.rb ? {lit(mech.c1[bi, s])} : {lit(mech.c0[bi, s])})"
            hi = poly(mech.c1[:7, s], hi_b)
            w(f"template <> __device__ __forceinline__ double {kind}_r_spec<{s}>(const TPow &p)")
            w("{")
            w(f"    return p.hi ? ({hi}) : ({lo});")
            w("}")
    w("")
    w("// Gibbs energies G_s = R (H_s/R - T S_s/R) in J/mol")
    w("__device__ __forceinline__ void gibbs_spec(const TPow &p, double G[NS])")
    w("{")
    for s in range(NS):
        w(f"    G[{s}] = R_GAS * h_r_spec<{s}>(p) - (R_GAS * s_r_spec<{s}>(p)) * p.T;")
    w("}")
    w("")
    w("// H/R, S/R and Cp/R of every species at one temperature")
    w("__device__ __forceinline__ void thermo_spec(const TPow &p, double h[NS], double sr[NS], double cp[NS])")
    w("{")
    for s in range(NS):
        w(f"    h[{s}] = h_r_spec<{s}>(p);")
        w(f"    sr[{s}] = s_r_spec<{s}>(p);")
        w(f"    cp[{s}] = cp_r_spec<{s}>(p);")
    w("}")
    w("")

    # one reaction's rate block
    def reaction(r, rtb_expr):
        xr = float(np.sum(sb[:, r] - sf[:, r]))
        b = float(mech.bf[r])
        if b == 0.0:
            powt = "1.0"
        elif b == 1.0:
            powt = "p.T"
        elif b == -1.0:
            powt = "p.tm1"
        elif b == -2.0:
            powt = "p.tm2"
        else:
            powt = f"exp({lit(b)} * p.lnT)"
        o = []
        o.append(f"        // reaction {r + 1}")
        if mech.eaf[r] == 0.0:
            o.append(f"        const double kf = {lit(mech.af[r])} * {powt};")
        else:
            o.append(f"        const double kf = {lit(mech.af[r])} * {powt} * exp(-{lit(mech.eaf[r])} / (RU_CAL * p.T));")
        terms = []
        for s in range(NS):
            nu = sb[s, r] - sf[s, r]
            if nu != 0:
                terms.append(f"{lit(nu)} * G[{s}]")
        dg = " + ".join(terms) if terms else "0.0"
        o.append(f"        const double dg = {dg};")

        def prod(st):
            fs = []
            for s in range(NS):
                n = st[s, r]
                if n == 1:
                    fs.append(f"Mc[{s}]")
                elif n == 2:
                    fs.append(f"(Mc[{s}] * Mc[{s}])")
                elif n != 0:
                    fs.append(f"pow(Mc[{s}], {lit(n)})")
            return " * ".join(fs) if fs else "1.0"
        o.append(f"        const double rf = {prod(sf)};")
        o.append(f"        const double rb = {prod(sb)};")
        tbt = [f"Mc[{s}] * {lit(tb[s, r])}" if tb[s, r] != 1.0 else f"Mc[{s}]" for s in range(NS) if tb[s, r] != 0]
        has_tb = bool(tbt)
        p0 = (101325.0 * 1e-6) ** xr
        if xr == 0:
            kc = f"kp"
        elif xr == 1:
            kc = f"kp * (1.0 / (R_GAS * p.T))"
        elif xr == -1:
            kc = f"kp * (R_GAS * p.T)"
        else:
            kc = f"kp * pow(R_GAS * p.T, {lit(-xr)})"
        o.append(f"        const double kp = exp(-dg / (R_GAS * p.T)) * {lit(p0)};")
        o.append(f"        const double kb = kf / ({kc});")
        if has_tb:
            o.append(f"        double tb = {' + '.join(tbt)};")
        else:
            o.append(f"        double tb = 0.0;")
        o.append(f"        {rtb_expr}")
        o.append(f"        const double rr = kf * rf - kb * rb;")
        return o, has_tb

    # IMEX: Diagonalized (R_TB defaults to 1)
    w("// Reaction::Diagonalized per cell: CMS (kg/m^3/s) and MD(s, s)")
    w("__device__ __forceinline__ void diagonalized_spec(const TPow &p, const double G[NS], const double Mc[NS],")
    w("                                                  const double Di[NS], const double PT[NS], double CMS[NS],")
    w("                                                  double MD[NS])")
    w("{")
    w("    double Wi[NS];")
    # The reference divides each term by Di (src/Reaction.cpp:798); here
    # the term is multiplied by 1/Di.  Below 2^-1022 (a subnormal partial
    # density, which trace species reach in cold air) 1/Di overflows, so such a
    # Di is scaled by 2^64 and its numerator with it: both scalings are exact,
    # and a normal Di keeps the scale 1.
    w("    // 1/Di, with a subnormal Di (and its numerator) scaled by 2^64 so that the")
    w("    // reciprocal stays finite; the scalings are exact")
    w("    double iDi[NS], sDi[NS];")
    w("#pragma unroll")
    w("    for (int s = 0; s < NS; s++) {")
    w("        sDi[s] = fabs(Di[s]) < 0x1p-1022 ? 0x1p+64 : 1.0;")
    w("        iDi[s] = Di[s] == 0.0 ? 0.0 : 1.0 / (Di[s] * sDi[s]);")
    w("    }")
    w("    const double tdep = 1.0 / (RU_CAL * (p.T * p.T));")
    w("#pragma unroll")
    w("    for (int s = 0; s < NS; s++) { Wi[s] = 0.0; MD[s] = 0.0; }")
    for r in range(NR):
        w("    {")
        blk, has_tb = reaction(r, "if (tb == 0.0) tb = 1.0;")
        L.extend(blk)
        wt = []
        if mech.bf[r] != 0.0:
            wt.append(f"{lit(mech.bf[r])} * p.tm1")
        if mech.eaf[r] != 0.0:
            wt.append(f"{lit(mech.eaf[r])} * tdep")
        w(f"        const double wjh2 = rr * ({' + '.join(wt) if wt else '0.0'});")
        for s in range(NS):
            nu = sb[s, r] - sf[s, r]
            if nu == 0:
                continue
            w(f"        Wi[{s}] += {lit(nu)} * tb * rr;")
            parts = []
            if sf[s, r] != 0:
                parts.append(f"kf * {lit(sf[s, r])} * rf")
            if sb[s, r] != 0:
                parts.append(f"- kb * {lit(sb[s, r])} * rb")
            wj = " ".join(parts) if parts else "0.0"
            if wj.startswith("- "):
                wj = "-" + wj[2:]
            tbterm = f" + rr * {lit(tb[s, r] / mech.mw[s])}" if tb[s, r] != 0 else ""
            w(f"        MD[{s}] += {lit(nu)} * (((({wj}) * sDi[{s}]) * iDi[{s}] + wjh2 * PT[{s}]) * tb{tbterm});")
        w("    }")
    w("#pragma unroll")
    w("    for (int s = 0; s < NS; s++) {")
    w("        CMS[s] = (cM.mw[s] * Wi[s]) * 1e3;")
    w("        MD[s] = cM.mw[s] * MD[s];")
    w("    }")
    w("}")
    w("")

    # trapezoid: P, Q, Wi with run-time R_TB mode
    w("// Point-implicit trapezoid production/loss (src/Reaction.cpp:455-482);")
    w("// rtb_mode 0: R_TB -> 1 when 0, 1: left as summed, 2: forced to 0")
    w("__device__ __forceinline__ void trap_rates_spec(const TPow &p, const double Mc[NS], int rtb_mode, double Wi[NS],")
    w("                                                double Pv[NS], double Qv[NS])")
    w("{")
    w("    double G[NS];")
    w("    gibbs_spec(p, G);")
    w("#pragma unroll")
    w("    for (int s = 0; s < NS; s++) { Wi[s] = 0.0; Pv[s] = 0.0; Qv[s] = 0.0; }")
    for r in range(NR):
        w("    {")
        blk, has_tb = reaction(r, "if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }")
        L.extend(blk)
        for s in range(NS):
            nu = sb[s, r] - sf[s, r]
            if nu != 0:
                w(f"        Wi[{s}] += {lit(nu)} * tb * rr;")
            qp = []
            pp = []
            if sb[s, r] != 0:
                qp.append(f"{lit(sb[s, r])} * kf * rf")
                pp.append(f"{lit(sb[s, r])} * kb * rb")
            if sf[s, r] != 0:
                qp.append(f"{lit(sf[s, r])} * kb * rb * tb")
                pp.append(f"{lit(sf[s, r])} * kf * rf * tb")
            if qp:
                w(f"        Qv[{s}] += {' + '.join(qp)};")
                w(f"        Pv[{s}] += {' + '.join(pp)};")
        w("    }")
    w("#pragma unroll")
    w("    for (int s = 0; s < NS; s++) Wi[s] = cM.mw[s] * Wi[s];")
    w("}")
    w("")
    w("}  // namespace h2ja919")
    w("}  // namespace eu3d")
    return "\n".join(L) + "\n"


def main():
    src = gen(load_h2_ja919())
    with open(OUT, "w") as fh:
        fh.write(src)
    print(OUT)


if __name__ == "__main__":
    main()
