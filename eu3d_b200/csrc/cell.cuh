// Per-cell FP64 kernels: conservative -> primitive decode with the Newton
// temperature inversion, IMEX diagonal chemistry, point-implicit trapezoid
// chemistry (field form and adaptive substeps), each fused with the state
// update that precedes it and the decode that follows it.
#pragma once

#include "common.cuh"
#include "mech_h2_ja919.cuh"

namespace eu3d {

constexpr int NCHEM_CAP = 1 << 20;  // adaptive substeps per cell per step

struct Decoded {
    double D, U, V, W, E, T, P, H, G, Cp, Rgas;
    double Y[NS];
};

// Mixture-averaged NASA-9 coefficients sum_s (Y_s Ri_s) a_k,s of the range
// `hi`, b1 taken from range `rb` (the reference's high-range defect selects 0).
__device__ __forceinline__ void mix_coeffs(const double yr[NS], int hi, int rb, double A[8])
{
#pragma unroll
    for (int k = 0; k < 7; k++) {
        double a = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) a += yr[s] * cM.c[hi][k][s];
        A[k] = a;
    }
    double b = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) b += yr[s] * cM.c[rb][7][s];
    A[7] = b;
}

// Flowfield::Update_after_CS per cell (src/Flowfield.cpp:1246-1284) with
// Flowfield::Get_temp (:1542-1566).  Eold is the E of the previous decode
// (the Newton target under EU3D_Q_STALE_E); T0 the Newton start.  The
// reference sums Y_s Ri_s h_s(T) species by species at every iteration; the
// same sums are formed here once per cell as mixture polynomial
// coefficients, so an iteration evaluates one polynomial instead of nine
// (equal up to rounding).
__device__ __forceinline__ void decode(const double cs[NV], double T0, double Eold, unsigned q, Decoded &o,
                                       int &capped)
{
    double D = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) D += cs[s];
    // one reciprocal of the density serves every quotient (within an ulp of dividing)
    const double iD = 1.0 / D;
    double yr[NS], sYR = 0.0, sdiv = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        o.Y[s] = cs[s] * iD;
        yr[s] = o.Y[s] * cM.ri[s];
        sYR += yr[s];
        sdiv += o.Y[s] * cM.imw[s];
    }
    const double U = cs[NS] * iD, V = cs[NS + 1] * iD, W = cs[NS + 2] * iD;
    const double Enew = (cs[NS + 3] - 0.5 * D * (U * U + V * V + W * W)) * iD;
    const double Et = (q & EU3D_Q_STALE_E) ? Eold : Enew;
    double A[8];
    int cur = -1;
    double Tn = T0, Tp;
    int count = 0;
    while (count < 10) {
        Tp = Tn;
        const TPow p = tpow(Tp, q);
        if (p.hi != cur) {
            cur = p.hi;
            mix_coeffs(yr, p.hi, p.rb, A);
        }
        const double sh = -A[0] * p.tm1 + A[1] * p.lnT + A[2] * p.T + A[3] * p.t2 * 0.5 +
                          A[4] * p.t3 * (1.0 / 3.0) + A[5] * p.t4 * 0.25 + A[6] * p.t5 * 0.2 + A[7];
        const double scp = A[0] * p.tm2 + A[1] * p.tm1 + A[2] + A[3] * p.T + A[4] * p.t2 + A[5] * p.t3 + A[6] * p.t4;
        const double t1 = (sh - Et * 1e-3) - sYR * Tp;
        const double t2 = scp - sYR;
        Tn = Tp - t1 / t2;
        if (fabs(Tn - Tp) < 1e-6) break;
        count++;
    }
    capped = count >= 10;
    const TPow p = tpow(Tn, q);
    if (p.hi != cur) mix_coeffs(yr, p.hi, p.rb, A);
    const double scp = A[0] * p.tm2 + A[1] * p.tm1 + A[2] + A[3] * p.T + A[4] * p.t2 + A[5] * p.t3 + A[6] * p.t4;
    const double Wav = 1.0 / sdiv;
    o.Rgas = R_GAS * 1000 / Wav;
    o.P = Tn * D * o.Rgas;
    o.H = o.P / D + Enew;
    o.Cp = scp * 1000;
    o.G = o.Cp / (o.Cp - R_GAS * sdiv * 1000);
    o.D = D;
    o.U = U;
    o.V = V;
    o.W = W;
    o.E = Enew;
    o.T = Tn;
}

template <class P>
__device__ __forceinline__ void store_prims(const Decoded &o, P *__restrict__ q, long long fs, long long c)
{
    q[PD * fs + c] = (P)o.D;
    q[PU * fs + c] = (P)o.U;
    q[PV * fs + c] = (P)o.V;
    q[PW * fs + c] = (P)o.W;
    q[PP * fs + c] = (P)o.P;
    q[PH * fs + c] = (P)o.H;
    q[PG * fs + c] = (P)o.G;
#pragma unroll
    for (int s = 0; s < NS; s++) q[(PY + s) * fs + c] = (P)o.Y[s];
}

// pow(Mc, nu) for the stoichiometric exponents 0, 1, 2 (validated on the
// host); pow(x, 2) in the reference is the correctly rounded x * x.
__device__ __forceinline__ double mcpow(double x, double nu)
{
    return nu == 0.0 ? 1.0 : (nu == 1.0 ? x : (nu == 2.0 ? x * x : pow(x, nu)));
}

__device__ __forceinline__ double powT(const TPow &p, double b)
{
    return b == 0.0 ? 1.0 : (b == 1.0 ? p.T : pow(p.T, b));
}

// Reaction-rate quantities of one reaction (src/Reaction.cpp:755-775).
struct Rxn {
    double KF, KB, RRF, RRB, RTB, RR;
};

// rtb_mode: 0 = R_TB defaults to 1 when its sum is 0 (Diagonalized),
// 1 = left at 0 (field Trapezoid), 2 = every R_TB set to 0 (adaptive).
__device__ __forceinline__ Rxn rxn(int r, const TPow &p, const double Mc[NS], const double G[NS], int rtb_mode)
{
    Rxn x;
    const double T = p.T;
    x.KF = cM.af[r] * powT(p, cM.bf[r]) * exp(-cM.eaf[r] / (RU_CAL * T));
    double dg = 0.0, rf = 1.0, rb = 1.0, tb = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        dg += cM.nu[s][r] * G[s];
        rf *= mcpow(Mc[s], cM.sf[s][r]);
        rb *= mcpow(Mc[s], cM.sb[s][r]);
        tb += Mc[s] * cM.tb[s][r];
    }
    const double Kp = exp(-dg / (R_GAS * T)) * cM.p0xr[r];
    const double xr = cM.xr[r];
    const double RT = R_GAS * T;
    const double Kc = Kp * (xr == 0.0 ? 1.0 : (xr == 1.0 ? 1.0 / RT : (xr == -1.0 ? RT : pow(RT, -xr))));
    x.KB = x.KF / Kc;
    if (rtb_mode == 0) {
        if (tb == 0.0) tb = 1.0;
    } else if (rtb_mode == 2) {
        tb = 0.0;
    }
    x.RRF = rf;
    x.RRB = rb;
    x.RTB = tb;
    x.RR = x.KF * rf - x.KB * rb;
    return x;
}

// Gibbs energies G_s = H_s - S_s T in J/mol at one temperature
__device__ __forceinline__ void gibbs(const TPow &p, double G[NS])
{
#pragma unroll
    for (int s = 0; s < NS; s++) G[s] = R_GAS * h_r(s, p) - (R_GAS * s_r(s, p)) * p.T;
}

// Reaction::Diagonalized per cell (src/Reaction.cpp:736-811): source CMS and
// diagonal Jacobian MD of the partial densities.  Mc in mol/cm^3, Di in g/cm^3.
__device__ __forceinline__ void diagonalized(const TPow &p, const double G[NS], const double Mc[NS], const double Di[NS],
                                             const double PT[NS], double CMS[NS], double MD[NS])
{
    double Wi[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        Wi[s] = 0.0;
        MD[s] = 0.0;
    }
    const double T = p.T;
#pragma unroll 1
    for (int r = 0; r < NR; r++) {
        const Rxn x = rxn(r, p, Mc, G, 0);
        const double wjh2 = x.RR * (cM.bf[r] / T + cM.eaf[r] / (RU_CAL * (T * T)));
#pragma unroll
        for (int s = 0; s < NS; s++) {
            const double nu = cM.nu[s][r];
            Wi[s] += nu * x.RTB * x.RR;
            const double wjh1 =
                (Di[s] == 0) ? 0.0 : x.KF * cM.sf[s][r] * x.RRF / Di[s] - x.KB * cM.sb[s][r] * x.RRB / Di[s];
            MD[s] += nu * ((wjh1 + wjh2 * PT[s]) * x.RTB + x.RR * cM.tb[s][r] / cM.mw[s]);
        }
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        CMS[s] = (cM.mw[s] * Wi[s]) * 1e3;
        MD[s] = cM.mw[s] * MD[s];
    }
}

// Point-implicit trapezoid update of one cell (src/Reaction.cpp:412-485,
// :489-591): Di in kg/m^3 in and out.  Wi (net production, g/cm^3/s) is
// returned for the substep prediction.
template <bool SPEC>
__device__ __forceinline__ void trapezoid(const TPow &p, const double cs_di[NS], double dt, int rtb_mode, double out[NS],
                                          double Wi[NS])
{
    double Mc[NS], Di[NS], Pv[NS], Qv[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        Di[s] = cs_di[s] * 1e-3;
        Mc[s] = (cs_di[s] / cM.mw[s] * 1000) * 1e-6;
        Pv[s] = 0.0;
        Qv[s] = 0.0;
        Wi[s] = 0.0;
    }
    if (SPEC) {
        h2ja919::trap_rates_spec(p, Mc, rtb_mode, Wi, Pv, Qv);
    } else {
        double G[NS];
        gibbs(p, G);
#pragma unroll 1
        for (int r = 0; r < NR; r++) {
            const Rxn x = rxn(r, p, Mc, G, rtb_mode);
#pragma unroll
            for (int s = 0; s < NS; s++) {
                Wi[s] += cM.nu[s][r] * x.RTB * x.RR;
                Qv[s] += (cM.sb[s][r] * x.KF * x.RRF + cM.sf[s][r] * x.KB * x.RRB * x.RTB);
                Pv[s] += (cM.sb[s][r] * x.KB * x.RRB + cM.sf[s][r] * x.KF * x.RRF * x.RTB);
            }
        }
#pragma unroll
        for (int s = 0; s < NS; s++) Wi[s] = cM.mw[s] * Wi[s];
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double q = cM.mw[s] * Qv[s];
        const double pp = (Mc[s] == 0) ? 0.0 : Pv[s] / Mc[s];
        out[s] = ((1.0 - dt / 2.0 * pp) * Di[s] + dt * q) / (1.0 + dt / 2.0 * pp) * 1e3;
    }
}

// Reaction::TrapezoidPrediction per cell (src/Reaction.cpp:593-670)
template <bool SPEC>
__device__ __forceinline__ int predict_nchem(const TPow &p, const double cs_di[NS], const double Y[NS], double dtm,
                                             int rtb_mode)
{
    double Mc[NS], Wi[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        Mc[s] = (cs_di[s] / cM.mw[s] * 1000) * 1e-6;
        Wi[s] = 0.0;
    }
    if (SPEC) {
        double Pv[NS], Qv[NS];
        h2ja919::trap_rates_spec(p, Mc, rtb_mode, Wi, Pv, Qv);
    } else {
        double G[NS];
        gibbs(p, G);
#pragma unroll 1
        for (int r = 0; r < NR; r++) {
            const Rxn x = rxn(r, p, Mc, G, rtb_mode);
#pragma unroll
            for (int s = 0; s < NS; s++) Wi[s] += cM.nu[s][r] * x.RTB * x.RR;
        }
#pragma unroll
        for (int s = 0; s < NS; s++) Wi[s] = cM.mw[s] * Wi[s];
    }
    double dt = dtm;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double w = Wi[s];
        if (Y[s] >= 1e-6 && w != 0) {
            const double t = fabs(-(cs_di[s] * 1e-3) / w);
            if (t < dt) dt = t;
        }
    }
    const double n = ceil(dtm / dt);
    if (!(n >= 1.0)) return 1;
    return n > (double)NCHEM_CAP ? NCHEM_CAP + 1 : (int)n;
}

__device__ __forceinline__ void load_cs(const double *__restrict__ cs, long long fs, long long c, double v[NV])
{
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = cs[q * fs + c];
}

__device__ __forceinline__ void store_cs(double *__restrict__ cs, long long fs, long long c, const double v[NV])
{
#pragma unroll
    for (int q = 0; q < NV; q++) cs[q * fs + c] = v[q];
}

__device__ __forceinline__ void warp_count(unsigned long long *ctr, bool flag)
{
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, flag);
    if (m && (threadIdx.x & 31) == (__ffs(act) - 1)) atomicAdd(ctr, (unsigned long long)__popc(m));
}

__device__ __forceinline__ void warp_sum(unsigned long long *ctr, unsigned long long v)
{
    const unsigned act = __activemask();
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_down_sync(act, v, o);
        if (((threadIdx.x & 31) + o) < 32 && ((act >> ((threadIdx.x & 31) + o)) & 1u)) v += w;
    }
    if ((threadIdx.x & 31) == (__ffs(act) - 1) && v) atomicAdd(ctr, v);
}

// Reaction::Diagonalized for the state of the previous decode (the stored CS
// and T), with GetPartial_T (src/Flowfield.cpp:1578-1595) for its Jacobian:
// source CMS (kg/m^3/s) and diagonal MD of the partial densities.
// tcouple = false drops the temperature coupling of the Jacobian (PT = 0),
// leaving its composition part (the adaptive integrator below).
template <bool SPEC>
__device__ __forceinline__ void imex_source(const double cs[NV], double T, unsigned qk, double CMS[NS], double MD[NS],
                                            bool tcouple = true)
{
    // state of the previous decode, recomputed from the stored CS and T
    double D = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) D += cs[s];
    const double U = cs[NS] / D, V = cs[NS + 1] / D, W = cs[NS + 2] / D;
    const TPow p = tpow(T, qk);
    double hr[NS], sr[NS], cpr[NS];
    if (SPEC) {
        h2ja919::thermo_spec(p, hr, sr, cpr);
    } else {
#pragma unroll
        for (int s = 0; s < NS; s++) {
            hr[s] = h_r(s, p);
            sr[s] = s_r(s, p);
            cpr[s] = cp_r(s, p);
        }
    }
    double sdiv = 0.0, scp = 0.0, Mc[NS], Di[NS], PT[NS], G[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double Y = cs[s] / D;
        sdiv += Y / cM.mw[s];
        scp += (cM.ri[s] * cpr[s]) * Y;
    }
    const double Rgas = R_GAS * 1000 / (1.0 / sdiv);
    const double CV = scp * 1000 - Rgas;
    const double ke = 0.5 * (U * U + V * V + W * W);
    // GetPartial_T, src/Flowfield.cpp:1578-1595; Gibbs energies for the rates
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double hs = (qk & EU3D_Q_PARTIAL_T_UNITS) ? cM.ri[s] * hr[s] : (cM.ri[s] * hr[s]) * 1e3;
        PT[s] = tcouple ? (ke - hs + cM.ri[s] * 1e3 * T) / (CV * D) : 0.0;
        G[s] = R_GAS * hr[s] - (R_GAS * sr[s]) * T;
        Di[s] = cs[s] * 1e-3;
        Mc[s] = (cs[s] / cM.mw[s] * 1000) * 1e-6;
    }
    if (SPEC)
        h2ja919::diagonalized_spec(p, G, Mc, Di, PT, CMS, MD);
    else
        diagonalized(p, G, Mc, Di, PT, CMS, MD);
}

// FP64 adaptive closed-reactor chemistry (new; the reference's one-step IMEX
// and adaptive trapezoid both diverge through H2-air ignition at the step
// sizes of its detonation cases).  Substeps of the species-diagonal implicit
// update rho_s += h CMS_s / (1 - h MD_s), with CMS and the composition part of
// the diagonal Jacobian MD from Reaction::Diagonalized at the current state,
// and a decode at constant density and energy after each.  The substep is the
// largest h <= the time left with h |CMS_s| <= rel (rho_s + 1e-9 rho) for
// every species and h MD_s <= amp where MD_s > 0 (growth stays bounded and
// consumed species stay positive), but at least dt / nmax; the last allowed
// substep takes the time left.
struct AdaptCfg {
    double rel, amp;
    int nmax;
};

// One substep of chem_adaptive: cs, T advance by h, the time left trem
// shrinks by h, the count k grows by one.  forced is set when the substep
// cap made h longer than the controller's choice (h = dt / nmax at least,
// the last allowed substep takes the time left).
template <bool SPEC>
__device__ __forceinline__ void adapt_substep(double cs[NV], double &T, double Eold, unsigned qk, double &trem, int &k,
                                              double hmin, const AdaptCfg &cfg, Decoded &o, int &capped_any,
                                              int &forced)
{
    double CMS[NS], MD[NS];
    imex_source<SPEC>(cs, T, qk, CMS, MD, false);
    double D = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) D += cs[s];
    double h = trem;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double w = fabs(CMS[s]);
        if (w > 0.0) h = fmin(h, cfg.rel * (cs[s] + 1e-9 * D) / w);
        if (MD[s] > 0.0) h = fmin(h, cfg.amp / MD[s]);
    }
    const double hc = h;
    h = fmin(fmax(h, hmin), trem);
    if (k == cfg.nmax - 1) h = trem;
    if (h > hc) forced = 1;
#pragma unroll
    for (int s = 0; s < NS; s++) cs[s] = fmax(cs[s] + h * CMS[s] / (1.0 - h * MD[s]), 0.0);
    int cp = 0;
    decode(cs, T, Eold, qk, o, cp);
    capped_any |= cp;
    T = o.T;
    trem -= h;
    k++;
}

template <bool SPEC>
__device__ __forceinline__ int chem_adaptive(double cs[NV], double &T, double Eold, unsigned qk, double dt,
                                             const AdaptCfg &cfg, int &capped_any, int &forced)
{
    double trem = dt;
    int k = 0;
    const double hmin = dt / cfg.nmax;
    Decoded o;
    while (trem > 0.0 && k < cfg.nmax) adapt_substep<SPEC>(cs, T, Eold, qk, trem, k, hmin, cfg, o, capped_any, forced);
    return k;
}

// Element projection of a composition change: the least change in the
// metric sum_k dY_k^2 / (Y_k + eps) that conserves the atoms of each element.
constexpr int SUR_NELEM = 3;  // H, O, N
// atoms of element e per unit mass of species k (atoms / W_k)
__constant__ double c_sur_elem[SUR_NELEM][NS];

__device__ __forceinline__ void elem_project(const double Y[NS], double dY[NS], double eps)
{
    double r[SUR_NELEM], M[SUR_NELEM][SUR_NELEM];
#pragma unroll
    for (int e = 0; e < SUR_NELEM; e++) {
        double a = 0.0;
#pragma unroll
        for (int k = 0; k < NS; k++) a += c_sur_elem[e][k] * dY[k];
        r[e] = a;
#pragma unroll
        for (int f = 0; f < SUR_NELEM; f++) {
            double m = 0.0;
#pragma unroll
            for (int k = 0; k < NS; k++) m += c_sur_elem[e][k] * (Y[k] + eps) * c_sur_elem[f][k];
            M[e][f] = m;
        }
    }
    // 3x3 solve by cofactors
    const double c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
    const double c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
    const double c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
    const double det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
    if (!(fabs(det) > 0.0)) return;
    const double id = 1.0 / det;
    const double inv[3][3] = {{c00 * id, (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * id,
                               (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * id},
                              {c01 * id, (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * id,
                               (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * id},
                              {c02 * id, (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * id,
                               (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * id}};
    double lam[SUR_NELEM];
#pragma unroll
    for (int e = 0; e < SUR_NELEM; e++) lam[e] = inv[e][0] * r[0] + inv[e][1] * r[1] + inv[e][2] * r[2];
#pragma unroll
    for (int k = 0; k < NS; k++) {
        double a = 0.0;
#pragma unroll
        for (int e = 0; e < SUR_NELEM; e++) a += c_sur_elem[e][k] * lam[e];
        dY[k] -= (Y[k] + eps) * a;
    }
}

// Chemistry increment of one cell over dt with the adaptive integrator: the
// closed reactor at the cell's density, momentum and energy, then the
// mass-fraction change projected to element conservation.  Tchem: the
// temperature the integrator reached (a Newton start for the next decode).
template <bool SPEC>
__device__ __forceinline__ int chem_increment(const double cs0[NV], double T0, double Eold, unsigned qk, double dt,
                                              const AdaptCfg &cfg, double proj_eps, double dY[NS], double &Tchem,
                                              int &capped_any, int &forced)
{
    double cs[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) cs[v] = cs0[v];
    double T = T0;
    const int n = chem_adaptive<SPEC>(cs, T, Eold, qk, dt, cfg, capped_any, forced);
    double D0 = 0.0, Dn = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        D0 += cs0[s];
        Dn += cs[s];
    }
    double Y0[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        Y0[s] = cs0[s] / D0;
        dY[s] = cs[s] / Dn - Y0[s];
    }
    elem_project(Y0, dY, proj_eps);
    Tchem = T;
    return n;
}

enum CellMode {
    M_DECODE = 0,
    M_ADV = 1,
    M_IMEX = 2,
    M_TRAP0 = 3,
    M_TRAP1 = 4,
    M_RK_STAGE1 = 5,
    M_RK_STAGE2 = 6,
    M_NOCHEM = 7,
    M_TRAP1_PREDICT = 8,
    M_ADAPT = 9,
    M_RK3_STAGE2 = 10,
    M_RK3_STAGE3 = 11
};

// Work queue of the adaptive trapezoid: cells binned by floor(log2 Nchem),
// listed heaviest bin first so that the warps that pull them together get
// similar substep counts, and pulled 32 at a time by persistent warps.
constexpr int QBINS = 32;
struct ChemQueue {
    int *list;   // interior cells in bin order
    int *bins;   // [0, 32) counts, [32, 64) start offsets, [64, 96) fill cursors, [96] work cursor, [97] total
    long long away_lo = 0, away_hi = 0;  // interior rows (k nj + j) integrated on another rank
};

__device__ __forceinline__ int nchem_bin(int n) { return 31 - __clz(max(n, 1)); }

struct CellArgs {
    Layout L;
    unsigned quirks;
    double *cs, *T, *E, *cs0;
    const void *rhs;  // flux residual, in the primitives' precision (P)
    int *nchem;
    const double *scal;  // [0] = dt
    Status *st;
    const double *xn, *yn;
    double wedge[3];
    int wedge_on;
    int *qbins;       // work-queue bin counts (M_TRAP1_PREDICT)
    AdaptCfg acfg;    // adaptive chemistry (M_ADAPT)
    double proj_eps;  // weight floor of its element projection
    int rhs_applied;  // M_ADAPT: the flux update is in the state and decoded already
};

__device__ __forceinline__ bool solid_cell(const CellArgs &a, int i, int j)
{
    if (!a.wedge_on) return false;
    const double x = a.xn[i], y = a.yn[j];
    return x > a.wedge[0] && (y - a.wedge[1]) < (x - a.wedge[0]) * a.wedge[2];
}

// the flux residual of cell index i as FP64 (its storage has the primitives' precision)
template <class P>
__device__ __forceinline__ double rhs_at(const CellArgs &a, long long i)
{
    return (double)static_cast<const P *>(a.rhs)[i];
}

// Split adaptive step of one cell: the flux residual (CS += RHS, then a
// decode; skipped with with_rhs = false when it was applied already), the
// closed-reactor chemistry over dt at that state with the adaptive
// integrator, applied as CS_s = rho (Y_s + dY_s) with negatives clipped, and
// a decode (o).  Returns the substeps taken.
template <class P, bool SPEC>
__device__ __forceinline__ int adapt_split_step(const CellArgs &a, long long c, double cs[NV], double T, double Eold,
                                                bool with_rhs, Decoded &o, int &capped_any, int &forced)
{
    const long long fs = a.L.fs;
    const unsigned qk = a.quirks;
    const double dt = a.scal[0];
    int cp = 0;
    if (with_rhs) {
#pragma unroll
        for (int v = 0; v < NV; v++) cs[v] = cs[v] + rhs_at<P>(a, v * fs + c);
        decode(cs, T, Eold, qk, o, cp);
        capped_any |= cp;
    } else {
        // the state is decoded already: re-derive it from CS and T
        double D = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) D += cs[s];
        const double iD = 1.0 / D;
#pragma unroll
        for (int s = 0; s < NS; s++) o.Y[s] = cs[s] * iD;
        o.U = cs[NS] * iD;
        o.V = cs[NS + 1] * iD;
        o.W = cs[NS + 2] * iD;
        o.E = (cs[NS + 3] - 0.5 * D * (o.U * o.U + o.V * o.V + o.W * o.W)) * iD;
        o.T = T;
        o.D = D;
    }
    double dY[NS], Tc;
    const int n = chem_increment<SPEC>(cs, o.T, o.E, qk, dt, a.acfg, a.proj_eps, dY, Tc, capped_any, forced);
    const double D = o.D;
#pragma unroll
    for (int s = 0; s < NS; s++) cs[s] = fmax(D * (o.Y[s] + dY[s]), 0.0);
    const double E1 = o.E;
    decode(cs, Tc, E1, qk, o, cp);
    capped_any |= cp;
    return n;
}

// One thread per interior cell.  MODE selects the reference sequence:
//  M_DECODE  Update_after_CS
//  M_ADV     Update_after_Adv (+ decode)
//  M_IMEX    Diagonalized + Update_IMEX (+ decode, + GetPartial_T for the next step)
//  M_TRAP0   Update_after_Adv, field Trapezoid, Explicit()
//  M_TRAP1   Update_after_Adv, TrapezoidPrediction and the per-cell substeps
//  M_RK_STAGE1/2  SSP-RK2 stage updates (new); M_RK_STAGE1 is also SSP-RK3's first
//  M_RK3_STAGE2/3 SSP-RK3 stage updates (new)
//  M_NOCHEM  Update_after_Adv, Explicit() (Euler::DNN, src/Euler.cpp:773-780)
// What the SSP-RK2 stage 2 with the fused frozen-chemistry gate needs of a
// cell (cell_body with GOUT): its index, decoded T and the FP32 sum of the
// mass fractions of the species in `mask`, each rounded to the primitives'
// precision first (the values the separate gate kernel loads).
struct CellGate {
    unsigned mask;
    bool valid;
    long long c;
    double T;
    float y;
};

template <class P, int MODE, bool SPEC, bool GOUT = false>
__device__ __forceinline__ void cell_body(const CellArgs &a, P *__restrict__ q, CellGate *gout = nullptr)
{
    const Layout &L = a.L;
    const int i = L.bc + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = L.bc + blockIdx.y;
    const int k = L.bc + blockIdx.z;
    if (i >= L.ni + L.bc) return;
    if (solid_cell(a, i, j)) return;
    const long long c = L.at(i, j, k);
    const long long fs = L.fs;
    const unsigned qk = a.quirks;
    const double dt = a.scal[0];
    double cs[NV];
    load_cs(a.cs, fs, c, cs);
    // the previous decode's energy is the Newton target only under the
    // stale-energy quirk; otherwise it is not read
    double T = a.T[c];
    const double Eold = (qk & EU3D_Q_STALE_E) ? a.E[c] : 0.0;
    Decoded o;
    int capped = 0, capped_any = 0;

    if (MODE == M_IMEX) {
        double CMS[NS], MD[NS];
        imex_source<SPEC>(cs, T, qk, CMS, MD);
        // Flowfield::Update_IMEX, src/Flowfield.cpp:1219-1228
#pragma unroll
        for (int v = 0; v < NV; v++) {
            double r = rhs_at<P>(a, v * fs + c);
            if (v < NS) {
                r = r + CMS[v] * dt;
                cs[v] = cs[v] + r / (1.0 - dt * MD[v]);
            } else {
                cs[v] = cs[v] + r;
            }
        }
        decode(cs, T, Eold, qk, o, capped);
        capped_any |= capped;
    } else if (MODE == M_ADAPT) {
        // split step: the flux residual first (Update_after_Adv + decode),
        // then the chemistry of the closed reactor at that state over dt
        // (adaptive integrator, element-projected), then a decode
        int forced = 0;
        const int nsub = adapt_split_step<P, SPEC>(a, c, cs, T, Eold, !a.rhs_applied, o, capped_any, forced);
        warp_sum(&a.st->substeps, (unsigned long long)nsub);
        if (forced) atomicAdd(&a.st->substep_capped, 1);
    } else if (MODE == M_DECODE) {
        decode(cs, T, Eold, qk, o, capped);
        capped_any |= capped;
    } else if (MODE == M_RK_STAGE1 || MODE == M_RK_STAGE2 || MODE == M_RK3_STAGE2 || MODE == M_RK3_STAGE3) {
        // Stage 1 leaves CS^n where it is and puts the stage state
        // CS^n + R(q^n) into cs0; SSP-RK2's stage 2 forms
        // 0.5 CS^n + 0.5 (CS1 + R(q1)) back into cs.  SSP-RK3 (Shu and Osher,
        // J. Comput. Phys. 77, 1988) forms CS2 = 3/4 CS^n + 1/4 (CS1 + R(q1))
        // into cs0 and CS^{n+1} = 1/3 CS^n + 2/3 (CS2 + R(q2)) into cs.  No
        // copy of CS^n is made.
        constexpr double wn = MODE == M_RK_STAGE2 ? 0.5 : MODE == M_RK3_STAGE2 ? 0.75 : 1.0 / 3.0;
        constexpr double ws = MODE == M_RK_STAGE2 ? 0.5 : MODE == M_RK3_STAGE2 ? 0.25 : 2.0 / 3.0;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const double r = rhs_at<P>(a, v * fs + c);
            if (MODE == M_RK_STAGE1)
                cs[v] = cs[v] + r;
            else
                cs[v] = __dadd_rn(__dmul_rn(wn, cs[v]), __dmul_rn(ws, __dadd_rn(a.cs0[v * fs + c], r)));
        }
        decode(cs, T, Eold, qk, o, capped);
        capped_any |= capped;
    } else {
        // Update_after_Adv, src/Flowfield.cpp:1140-1157
        const int nv = (qk & EU3D_Q_ADV_SPECIES_ONLY) ? NS : NV;
#pragma unroll
        for (int v = 0; v < NV; v++)
            if (v < nv) cs[v] = cs[v] + rhs_at<P>(a, v * fs + c);
        decode(cs, T, Eold, qk, o, capped);
        capped_any |= capped;
        if (MODE == M_TRAP0 || MODE == M_NOCHEM) {
            double dn[NS], Wi[NS];
            if (MODE == M_TRAP0) {
                const int rtb = (qk & EU3D_Q_TRAP_RTB_ZERO) ? 1 : 0;
                trapezoid<SPEC>(tpow(o.T, qk), cs, dt, rtb, dn, Wi);
            } else {
#pragma unroll
                for (int s = 0; s < NS; s++) dn[s] = cs[s];
            }
            // Flowfield::Explicit(), src/Flowfield.cpp:1169-1186
            double D = 0.0;
#pragma unroll
            for (int s = 0; s < NS; s++) {
                cs[s] = dn[s];
                D += cs[s];
            }
            cs[NS] = o.U * D;
            cs[NS + 1] = o.V * D;
            const double e = D * o.E + 0.5 * (o.U * o.U + o.V * o.V + o.W * o.W) * D;
            if (qk & EU3D_Q_EXPLICIT_ENERGY) {
                cs[NS + 2] = e;
            } else {
                cs[NS + 2] = o.W * D;
                cs[NS + 3] = e;
            }
            const double E1 = o.E;
            decode(cs, o.T, E1, qk, o, capped);
            capped_any |= capped;
        } else if (MODE == M_TRAP1 || MODE == M_TRAP1_PREDICT) {
            const int rtb = (qk & EU3D_Q_ADAPT_RTB_ZERO) ? 2 : 0;
            int n = predict_nchem<SPEC>(tpow(o.T, qk), cs, o.Y, dt, rtb);
            const bool over = n > NCHEM_CAP;
            if (over) n = NCHEM_CAP;
            if (over) atomicAdd(&a.st->substep_capped, 1);
            atomicMax(&a.st->nchem_max, n);
            if (a.nchem) a.nchem[c] = n;
            if (MODE == M_TRAP1_PREDICT) {
                // the substeps run later on the work queue (k_trap1_work)
                store_cs(a.cs, fs, c, cs);
                a.T[c] = o.T;
                a.E[c] = o.E;
                const unsigned act = __activemask();
                const int b = nchem_bin(n);
                const unsigned peers = __match_any_sync(act, b);
                if ((threadIdx.x & 31) == (__ffs(peers) - 1)) atomicAdd(a.qbins + b, __popc(peers));
                warp_count(&a.st->newton_capped, capped_any != 0);
                return;
            }
            const double dts = dt / n;
            for (int step = 0; step < n; step++) {
                double dn[NS], Wi[NS];
                trapezoid<SPEC>(tpow(o.T, qk), cs, dts, rtb, dn, Wi);
                // Flowfield::Explicit(step, i, j, k), src/Flowfield.cpp:1189-1203
                double D = 0.0;
#pragma unroll
                for (int s = 0; s < NS; s++) {
                    cs[s] = dn[s];
                    D += cs[s];
                }
                cs[NS] = o.U * D;
                cs[NS + 1] = o.V * D;
                cs[NS + 2] = o.W * D;
                cs[NS + 3] = D * o.E + 0.5 * (o.U * o.U + o.V * o.V + o.W * o.W) * D;
                decode(cs, o.T, o.E, qk, o, capped);
                capped_any |= capped;
            }
            atomicAdd(&a.st->substeps, (unsigned long long)n);
        }
    }
    store_cs(MODE == M_RK_STAGE1 || MODE == M_RK3_STAGE2 ? a.cs0 : a.cs, fs, c, cs);
    a.T[c] = o.T;
    a.E[c] = o.E;
    store_prims<P>(o, q, fs, c);
    if constexpr (GOUT) {
        float y = 0.f;
        if (gout->mask) {
#pragma unroll
            for (int s = 0; s < NS; s++)
                if ((gout->mask >> s) & 1u) y += fmaxf((float)(P)o.Y[s], 0.f);
        }
        gout->valid = true;
        gout->c = c;
        gout->T = o.T;
        gout->y = y;
    }
    warp_count(&a.st->newton_capped, capped_any != 0);
    warp_count(&a.st->nonfinite, !(isfinite(o.D) && isfinite(o.T)));
}

template <class P, int MODE, bool SPEC>
__global__ void __launch_bounds__(128, 3) k_cell(CellArgs a, P *__restrict__ q)
{
    cell_body<P, MODE, SPEC>(a, q);
}

// The same cell update compiled for NB resident blocks of 128 threads per SM
// (fewer registers a thread): the memory-bound SSP-RK2 stage updates, whose
// decode otherwise holds 167 registers and leaves 12 warps per SM to cover
// the HBM latency (tuning cell_blocks; NB = 4 gives the results of NB = 3
// bit for bit).
template <class P, int MODE, bool SPEC, int NB>
__global__ void __launch_bounds__(128, NB) k_cell_nb(CellArgs a, P *__restrict__ q)
{
    cell_body<P, MODE, SPEC>(a, q);
}

// Bin offsets of the adaptive-trapezoid queue, heaviest bin first (one warp).
__global__ void k_queue_scan(ChemQueue qu)
{
    const int b = 31 - (int)threadIdx.x;  // lane 0 takes the heaviest bin
    const int cnt = qu.bins[b];
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)threadIdx.x >= o) incl += v;
    }
    qu.bins[QBINS + b] = incl - cnt;
    qu.bins[2 * QBINS + b] = 0;
    if (threadIdx.x == 31) {
        qu.bins[3 * QBINS] = 0;
        qu.bins[3 * QBINS + 1] = incl;
    }
}

// Lists each interior cell in its bin.
__global__ void k_queue_scatter(CellArgs a, ChemQueue qu)
{
    const Layout &L = a.L;
    const int i = L.bc + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = L.bc + blockIdx.y;
    const int k = L.bc + blockIdx.z;
    if (i >= L.ni + L.bc) return;
    if (solid_cell(a, i, j)) return;
    const long long row = (long long)blockIdx.z * L.nj + blockIdx.y;
    if (row >= qu.away_lo && row < qu.away_hi) return;
    const long long c = L.at(i, j, k);
    const int b = nchem_bin(a.nchem[c]);
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, b);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(qu.bins + 2 * QBINS + b, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    qu.list[qu.bins[QBINS + b] + base + __popc(peers & ((1u << lane) - 1u))] = (int)c;
}

// One listed cell of the adaptive-trapezoid queue.
template <class P, bool SPEC>
__device__ __forceinline__ void trap1_cell(const CellArgs &a, P *__restrict__ q, long long c, double dt, int rtb)
{
    const long long fs = a.L.fs;
    const unsigned qk = a.quirks;
    {
        double cs[NV];
        load_cs(a.cs, fs, c, cs);
        // the decoded state of M_TRAP1_PREDICT, re-derived from CS and T
        Decoded o;
        double D = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) D += cs[s];
        const double iD = 1.0 / D;
#pragma unroll
        for (int s = 0; s < NS; s++) o.Y[s] = cs[s] * iD;
        o.U = cs[NS] * iD;
        o.V = cs[NS + 1] * iD;
        o.W = cs[NS + 2] * iD;
        o.E = (cs[NS + 3] - 0.5 * D * (o.U * o.U + o.V * o.V + o.W * o.W)) * iD;
        o.T = a.T[c];
        o.D = D;
        const int n = a.nchem[c];
        const double dts = dt / n;
        int capped = 0, capped_any = 0;
        for (int step = 0; step < n; step++) {
            double dn[NS], Wi[NS];
            trapezoid<SPEC>(tpow(o.T, qk), cs, dts, rtb, dn, Wi);
            double Dn = 0.0;
#pragma unroll
            for (int s = 0; s < NS; s++) {
                cs[s] = dn[s];
                Dn += cs[s];
            }
            cs[NS] = o.U * Dn;
            cs[NS + 1] = o.V * Dn;
            cs[NS + 2] = o.W * Dn;
            cs[NS + 3] = Dn * o.E + 0.5 * (o.U * o.U + o.V * o.V + o.W * o.W) * Dn;
            decode(cs, o.T, o.E, qk, o, capped);
            capped_any |= capped;
        }
        if (n == 0) {
            int cp = 0;
            decode(cs, o.T, o.E, qk, o, cp);
        }
        store_cs(a.cs, fs, c, cs);
        a.T[c] = o.T;
        a.E[c] = o.E;
        store_prims<P>(o, q, fs, c);
        atomicAdd(&a.st->substeps, (unsigned long long)n);
        if (capped_any) atomicAdd(&a.st->newton_capped, 1ull);
        if (!(isfinite(o.D) && isfinite(o.T))) atomicAdd(&a.st->nonfinite, 1ull);
    }
}

// Persistent workers of the adaptive trapezoid: each warp pulls 32 listed
// cells and runs their TrapezoidPrediction substeps (src/Reaction.cpp:489-591)
// with the re-encode and decode of Flowfield::Explicit(step, i, j, k)
// (src/Flowfield.cpp:1189-1203) after each, from the decoded state that
// M_TRAP1_PREDICT stored.
template <class P, bool SPEC>
__global__ void __launch_bounds__(128, 3) k_trap1_work(CellArgs a, P *__restrict__ q, ChemQueue qu)
{
    const int lane = threadIdx.x & 31;
    const int total = qu.bins[3 * QBINS + 1];
    const unsigned qk = a.quirks;
    const double dt = a.scal[0];
    const int rtb = (qk & EU3D_Q_ADAPT_RTB_ZERO) ? 2 : 0;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(qu.bins + 3 * QBINS, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const int slot = base + lane;
        if (slot < total) trap1_cell<P, SPEC>(a, q, qu.list[slot], dt, rtb);
    }
}

}  // namespace eu3d
