"""Operation count of the per-cell FP64 chemistry (test and measurement
infrastructure only: the product never imports this file).

A scalar restatement of the reference's per-cell arithmetic in its own
operation order, run on values of a counting type:

  * Flowfield::Get_temp's Newton inversion and Update_after_CS's decode
    (src/Flowfield.cpp:1542-1566, :1246-1284), with Reaction::GetCpi/GetHi/GetSi
    (src/Reaction.cpp:893-948);
  * Flowfield::GetPartial_T (src/Flowfield.cpp:1578-1595);
  * Reaction::Diagonalized (src/Reaction.cpp:736-811) and Flowfield::Update_IMEX
    (src/Flowfield.cpp:1215-1234): one IMEX step of a cell;
  * one substep of the adaptive chemistry (the composition part of
    Diagonalized, the substep controller, the species update and a decode),
    the integrator the surrogate falls back to.

Counting rules: add, sub, mul, div = 1 FLOP each (an FMA is a mul and an
add, 2); comparisons, sign flips, fabs and selections are not counted, nor
are expressions of the mechanism's constants alone (sums and differences of
stoichiometric coefficients): they do not depend on the cell.  The
reference calls pow with integer exponents -- pow(T, 2), pow(Mc, nu) with
stoichiometric nu, pow(R T, -Xr) -- which are |n| - 1 multiplies (and one
division for n < 0) and are counted so; pow with a non-integer exponent
(the Arrhenius T^b), exp, log and sqrt are tallied separately.  EQUIV gives
the FLOP equivalents the roofline figures use for them (a stated
convention: a range reduction plus a polynomial of about ten terms for exp
and log, both for pow, one division for sqrt).

The restatement is pinned to the oracle: with plain floats it reproduces the
C oracle's CMS, MD, T and conserved state (tests/test_opcount.py)."""
from __future__ import annotations

import math
from collections import Counter

import numpy as np

R = 8.31434
RU = 1.987
P0 = 101325.0

EQUIV = {"exp": 20, "log": 20, "pow": 40, "sqrt": 1}


class Tally(Counter):
    @property
    def flops(self) -> int:
        return self["add"] + self["mul"] + self["div"]

    def flops_with_transcendentals(self) -> float:
        return self.flops + sum(EQUIV[k] * self[k] for k in EQUIV)


class Num:
    """A float that counts the arithmetic done with it into `tally`."""

    __slots__ = ("v", "t")
    __array_ufunc__ = None  # numpy scalars defer to the reflected operators

    def __init__(self, v, t):
        self.v = float(v)
        self.t = t

    def _o(self, x):
        return x.v if isinstance(x, Num) else float(x)

    def _r(self, v, kind):
        self.t[kind] += 1
        return Num(v, self.t)

    def __add__(self, x):
        return self._r(self.v + self._o(x), "add")

    __radd__ = __add__

    def __sub__(self, x):
        return self._r(self.v - self._o(x), "add")

    def __rsub__(self, x):
        return self._r(self._o(x) - self.v, "add")

    def __mul__(self, x):
        return self._r(self.v * self._o(x), "mul")

    __rmul__ = __mul__

    def __truediv__(self, x):
        return self._r(self.v / self._o(x), "div")

    def __rtruediv__(self, x):
        return self._r(self._o(x) / self.v, "div")

    def __neg__(self):
        return Num(-self.v, self.t)

    def __abs__(self):
        return Num(abs(self.v), self.t)

    def __lt__(self, x):
        return self.v < self._o(x)

    def __le__(self, x):
        return self.v <= self._o(x)

    def __gt__(self, x):
        return self.v > self._o(x)

    def __ge__(self, x):
        return self.v >= self._o(x)

    def __eq__(self, x):
        return self.v == self._o(x)

    def __float__(self):
        return self.v


def _val(x):
    return x.v if isinstance(x, Num) else float(x)


def _tally_of(*xs):
    for x in xs:
        if isinstance(x, Num):
            return x.t
    return None


def exp(x):
    t = _tally_of(x)
    if t is None:
        return math.exp(x)
    t["exp"] += 1
    return Num(math.exp(x.v), t)


def log(x):
    t = _tally_of(x)
    if t is None:
        return math.log(x)
    t["log"] += 1
    return Num(math.log(x.v), t)


def sqrt(x):
    t = _tally_of(x)
    if t is None:
        return math.sqrt(x)
    t["sqrt"] += 1
    return Num(math.sqrt(x.v), t)


def pow_(x, y):
    """pow as the reference calls it: integer exponents are repeated
    multiplies (one division for a negative one), others a transcendental.
    The value is glibc's pow, as the reference computes it."""
    t = _tally_of(x, y)
    v = math.pow(_val(x), _val(y))
    if t is None:
        return v
    n = _val(y)
    if n == int(n) and abs(n) <= 16:
        n = int(n)
        t["mul"] += max(abs(n) - 1, 0)
        if n < 0:
            t["div"] += 1
    else:
        t["pow"] += 1
    return Num(v, t)


class Mech:
    """The mechanism arrays the per-cell functions read (plain floats)."""

    def __init__(self, mech):
        L = lambda a: np.asarray(a, dtype=np.float64).tolist()
        self.NS, self.NR = mech.NS, mech.NR
        self.c0, self.c1 = L(mech.c0), L(mech.c1)
        self.mw, self.ri = L(mech.mw), L(mech.ri)
        self.sf, self.sb, self.tb = L(mech.stoi_f), L(mech.stoi_b), L(mech.react_tb)
        self.af, self.bf, self.eaf = L(mech.af), L(mech.bf), L(mech.eaf)


# ------------------------------------------------ thermo (fixed policy)
def getcpi(m, T, Rs, s):
    c = m.c0 if T < 1000 else m.c1
    return Rs * (c[0][s] * pow_(T, -2) + c[1][s] * pow_(T, -1) + c[2][s] + c[3][s] * T + c[4][s] * pow_(T, 2) +
                 c[5][s] * pow_(T, 3) + c[6][s] * pow_(T, 4))


def gethi(m, T, Rs, s):
    c = m.c0 if T < 1000 else m.c1
    return Rs * (-c[0][s] * pow_(T, -1) + c[1][s] * log(T) + c[2][s] * T + c[3][s] * pow_(T, 2) / 2 +
                 c[4][s] * pow_(T, 3) / 3 + c[5][s] * pow_(T, 4) / 4 + c[6][s] * pow_(T, 5) / 5 + c[7][s])


def getsi(m, T, Rs, s):
    c = m.c0 if T < 1000 else m.c1
    return Rs * (-c[0][s] * pow_(T, -2) / 2 - c[1][s] * pow_(T, -1) + c[2][s] * log(T) + c[3][s] * T +
                 c[4][s] * pow_(T, 2) / 2 + c[5][s] * pow_(T, 3) / 3 + c[6][s] * pow_(T, 4) / 4 + c[8][s])


def _sum_mul(a, b):
    s = 0.0
    for x, y in zip(a, b):
        s = s + (x * y)
    return s


def _sum_div(a, b):
    s = 0.0
    for x, y in zip(a, b):
        s = s + (x / y)
    return s


# ------------------------------------------------------------- decode
def get_temp(m, T, Eval, Y):
    """Get_temp's Newton iteration; returns (T, iterations)."""
    T0 = T_temp = T
    count = 0
    while count < 10:
        T0 = T_temp
        Cpi0 = [getcpi(m, T0, m.ri[s], s) for s in range(m.NS)]
        Hi0 = [gethi(m, T0, m.ri[s], s) for s in range(m.NS)]
        temp1 = (_sum_mul(Y, Hi0) - Eval * 1e-3) - _sum_mul(Y, m.ri) * T0
        temp2 = _sum_mul(Y, Cpi0) - _sum_mul(Y, m.ri)
        T_temp = T0 - temp1 / temp2
        if abs(T_temp - T0) < 1e-6:
            break
        count = count + 1
    return T_temp, min(count + 1, 10)


def decode(m, cs, T):
    """Update_after_CS for one cell: (state dict, Newton iterations)."""
    NS = m.NS
    D = 0.0
    Di, Mc = [], []
    for s in range(NS):
        D = D + cs[s]
        Di.append(cs[s])
        Mc.append(cs[s] / m.mw[s] * 1000)
    Y = [cs[s] / D for s in range(NS)]
    U, V, W = cs[NS] / D, cs[NS + 1] / D, cs[NS + 2] / D
    E = (cs[NS + 3] - 0.5 * D * (pow_(U, 2) + pow_(V, 2) + pow_(W, 2))) / D
    T, it = get_temp(m, T, E, Y)
    Wav = 1.0 / _sum_div(Y, m.mw)
    Rgas = R * 1000 / Wav
    P = T * D * Rgas
    H = P / D + E
    Cpi = [getcpi(m, T, m.ri[s], s) for s in range(NS)]
    Cp = _sum_mul(Cpi, Y) * 1000
    G = Cp / (Cp - R * _sum_div(Y, m.mw) * 1000)
    C = sqrt(G * P / D)
    Ma = sqrt(pow_(U, 2) + pow_(V, 2) + pow_(W, 2)) / C
    return dict(D=D, Di=Di, Mc=Mc, Y=Y, U=U, V=V, W=W, E=E, T=T, Rgas=Rgas, P=P, H=H, Cp=Cp, Gamma=G, C=C,
                Ma=Ma), it


def partial_t(m, st):
    """GetPartial_T for one decoded cell (the first NS entries)."""
    CV = st["Cp"] - st["Rgas"]
    out = []
    for s in range(m.NS):
        Hi = gethi(m, st["T"], m.ri[s], s) * 1e3
        out.append((0.5 * (pow_(st["U"], 2) + pow_(st["V"], 2) + pow_(st["W"], 2)) - Hi + m.ri[s] * 1e3 * st["T"]) /
                   (CV * st["D"]))
    return out


# ---------------------------------------------------------- chemistry
def diagonalized(m, Di_in, Mc_in, T, PT):
    """Reaction::Diagonalized for one cell: CMS (NS), MD diagonal (NS)."""
    NS, NR = m.NS, m.NR
    Di = [Di_in[s] * 1e-3 for s in range(NS)]
    Mc = [Mc_in[s] * 1e-6 for s in range(NS)]
    Hi = [gethi(m, T, R, s) for s in range(NS)]
    Si = [getsi(m, T, R, s) for s in range(NS)]
    Gi = [Hi[s] - Si[s] * T for s in range(NS)]
    RR_F, RR_B, R_TB, KF, KB, RR = [], [], [], [], [], []
    for r in range(NR):
        rf, rb, rtb = 1.0, 1.0, 0.0
        Xr, dg = 0.0, 0.0
        kf = m.af[r] * pow_(T, m.bf[r]) * exp(-m.eaf[r] / (RU * T))
        for s in range(NS):
            Xr = Xr + (m.sb[s][r] - m.sf[s][r])
            dg = dg + (m.sb[s][r] - m.sf[s][r]) * Gi[s]
            rf = rf * pow_(Mc[s], m.sf[s][r])
            rb = rb * pow_(Mc[s], m.sb[s][r])
            rtb = rtb + Mc[s] * m.tb[s][r]
        kp = exp(-dg / (R * T)) * pow_(P0 * 1e-6, _val(Xr))
        kc = kp * pow_(R * T, -_val(Xr))
        kb = kf / kc
        if rtb == 0.0:
            rtb = 1.0
        RR_F.append(rf)
        RR_B.append(rb)
        R_TB.append(rtb)
        KF.append(kf)
        KB.append(kb)
        RR.append(kf * rf - kb * rb)
    CMS = []
    for s in range(NS):
        temp = 0.0
        for r in range(NR):
            temp = temp + (m.sb[s][r] - m.sf[s][r]) * R_TB[r] * RR[r]
        CMS.append(m.mw[s] * temp * 1e3)
    MD = []
    for s in range(NS):
        temp = 0.0
        for r in range(NR):
            if _val(Di[s]) == 0:
                w1 = 0.0
            else:
                w1 = KF[r] * m.sf[s][r] * RR_F[r] / Di[s] - KB[r] * m.sb[s][r] * RR_B[r] / Di[s]
            w2 = RR[r] * (m.bf[r] / T + m.eaf[r] / (RU * pow_(T, 2)))
            temp = temp + (m.sb[s][r] - m.sf[s][r]) * ((w1 + w2 * PT[s]) * R_TB[r] + RR[r] * m.tb[s][r] / m.mw[s])
        MD.append(m.mw[s] * temp)
    return CMS, MD


def imex_cell(m, cs, rhs, T, PT, dt):
    """Diagonalized + Update_IMEX + decode + GetPartial_T of one cell (the
    reference's IMEX step for a cell whose previous decode left T, PT)."""
    NS = m.NS
    Di = [cs[s] for s in range(NS)]
    Mc = [cs[s] / m.mw[s] * 1000 for s in range(NS)]
    CMS, MD = diagonalized(m, Di, Mc, T, PT)
    r = list(rhs)
    for s in range(NS):
        r[s] = r[s] + CMS[s] * dt
    out = list(cs)
    for v in range(NS + 4):
        md = MD[v] if v < NS else 0.0
        out[v] = cs[v] + r[v] / (1.0 - dt * md)
    st, it = decode(m, out, T)
    return out, st, partial_t(m, st), it


def adaptive_substep(m, cs, T, trem, dt, rel=0.02, amp=0.5, nmax=1024, k=0):
    """One substep of the adaptive chemistry at constant density and energy:
    (new cs, T, time left, Newton iterations)."""
    NS = m.NS
    Di = [cs[s] for s in range(NS)]
    Mc = [cs[s] / m.mw[s] * 1000 for s in range(NS)]
    CMS, MD = diagonalized(m, Di, Mc, T, [0.0] * NS)
    D = 0.0
    for s in range(NS):
        D = D + cs[s]
    h = trem
    for s in range(NS):
        w = abs(CMS[s])
        if w > 0.0:
            c = rel * (cs[s] + 1e-9 * D) / w
            h = c if c < h else h
        if MD[s] > 0.0:
            c = amp / MD[s]
            h = c if c < h else h
    hmin = dt / nmax
    h = hmin if h < hmin else h
    h = trem if h > trem else h
    if k == nmax - 1:
        h = trem
    out = list(cs)
    for s in range(NS):
        v = cs[s] + h * CMS[s] / (1.0 - h * MD[s])
        out[s] = v if v > 0.0 else 0.0
    st, it = decode(m, out, T)
    return out, st["T"], trem - h, it


def counted(t, x):
    if isinstance(x, (list, tuple)):
        return [counted(t, v) for v in x]
    return Num(x, t)


def count_imex(mech, cs, rhs, T, PT, dt):
    """Tally of one cell's IMEX step."""
    m = Mech(mech)
    t = Tally()
    imex_cell(m, counted(t, cs), counted(t, rhs), Num(T, t), counted(t, PT), dt)
    return t


def count_adaptive_substep(mech, cs, T, dt):
    m = Mech(mech)
    t = Tally()
    adaptive_substep(m, counted(t, cs), Num(T, t), Num(dt, t), dt)
    return t


def state_set(mech, n: int = 64, seed: int = 0):
    """Thermochemical states of the surrogate's standalone set: T uniform in
    300-3500 K, p log-uniform in 0.05-50 atm, compositions at the element
    ratios of stoichiometric H2-air (reactants burnt to a random extent, with
    a random radical pool), at rest.  Returns (cs (n, NS+4), T (n,))."""
    from eu3d_b200.cases import complete_state
    from eu3d_b200.readers import stoichiometric_h2_air
    rng = np.random.default_rng(seed)
    sp = mech.species
    Yr = stoichiometric_h2_air(mech)
    Yp = np.zeros(mech.NS)
    Yp[sp.index("H2O")] = Yr[sp.index("H2")] + Yr[sp.index("O2")]
    Yp[sp.index("N2")] = Yr[sp.index("N2")]
    out_cs, out_T = [], []
    for _ in range(n):
        b = rng.uniform()
        Y = (1 - b) * Yr + b * Yp
        for r in ("H", "O", "OH", "HO2", "H2O2"):
            Y[sp.index(r)] += 10 ** rng.uniform(-8, -3)
        Y /= Y.sum()
        T = rng.uniform(300.0, 3500.0)
        P = 101325.0 * np.exp(rng.uniform(np.log(0.05), np.log(50.0)))
        st = complete_state(mech, P, T, 0.0, 0.0, 0.0, Y)
        out_cs.append(np.asarray(st["CS"]).tolist())
        out_T.append(T)
    return out_cs, out_T


def reference_counts(mech, n: int = 64, seed: int = 0, newton: int = 2):
    """Average tallies over state_set: one IMEX cell-step (Diagonalized,
    Update_IMEX, the decode and GetPartial_T) whose decode starts `newton`
    iterations away from convergence, and one adaptive substep (likewise).
    The decode's start is a temperature off by 2^(newton-1) K, which the
    quadratically converging Newton iteration needs about `newton` + 1
    iterations to settle; the counts are returned with the average
    iterations taken."""
    m = Mech(mech)
    cs_set, T_set = state_set(mech, n, seed)
    tot_i, tot_a = Tally(), Tally()
    its_i = its_a = 0
    for cs, T in zip(cs_set, T_set):
        t = Tally()
        st, _ = decode(m, counted(Tally(), cs), Num(T, Tally()))
        PT = [p.v for p in partial_t(m, st)]
        Tstart = T + 2.0 ** (newton - 1)
        _, _, _, it = imex_cell(m, counted(t, cs), counted(t, [0.0] * (m.NS + 4)), Num(Tstart, t), counted(t, PT),
                                1e-8)
        tot_i.update(t)
        its_i += it
        t = Tally()
        _, _, _, it = adaptive_substep(m, counted(t, cs), Num(Tstart, t), Num(1e-8, t), 1e-8)
        tot_a.update(t)
        its_a += it
    avg = lambda tt: {k: v / n for k, v in tt.items()}
    fl = lambda tt: (tt["add"] + tt["mul"] + tt["div"]) / n
    fe = lambda tt: fl(tt) + sum(EQUIV[k] * tt[k] for k in EQUIV) / n
    return {"imex_cell": {"flops": fl(tot_i), "flops_equiv": fe(tot_i), "tally": avg(tot_i), "newton": its_i / n},
            "adaptive_substep": {"flops": fl(tot_a), "flops_equiv": fe(tot_a), "tally": avg(tot_a),
                                 "newton": its_a / n},
            "equivalents": dict(EQUIV), "states": n, "seed": seed}
