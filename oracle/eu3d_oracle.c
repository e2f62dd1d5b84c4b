/*
 * EU3D hot-path oracle (TEST INFRASTRUCTURE ONLY, see eu3d_oracle.h).
 *
 * A CPU restatement of the reference solver's arithmetic, written to follow
 * the reference's operation order term by term so that, compiled with the
 * same flags as the reference (-O2 -ffp-contract=off, no fast-math), it
 * agrees with the compiled reference bit for bit.  Quirk flags
 * (include/eu3d_quirks.h) select between the reference's defects and their
 * corrections.  The wedge immersed boundary, the transmissive ends and the
 * SSP-RK2 driver have no counterpart in the reference; they restate this
 * project's own definitions of those features.
 */
#include "eu3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double ORC_R = 8.31434;  /* Flowfield/Reaction `R`, include/Reaction.hpp:269 */
static const double ORC_RU = 1.987;   /* include/Reaction.hpp:270 */
static const double ORC_P0 = 101325;  /* include/Reaction.hpp:271 */

#define ORC_NCHEM_CAP 1048576.0

#define ID3(f, i, j, k) (((size_t)(i) * (f)->NJ + (size_t)(j)) * (f)->NK + (size_t)(k))
#define ID4(f, i, j, k, s, n) (ID3(f, i, j, k) * (size_t)(n) + (size_t)(s))

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

int orc_field_alloc(orc_field *f, int ni, int nj, int nk, int bc, int NS)
{
    memset(f, 0, sizeof(*f));
    f->ni = ni; f->nj = nj; f->nk = nk; f->bc = bc; f->NS = NS;
    f->NI = ni + 2 * bc; f->NJ = nj + 2 * bc; f->NK = nk + 2 * bc;
    size_t n3 = (size_t)f->NI * f->NJ * f->NK;
    f->xnode = zalloc(f->NI); f->ynode = zalloc(f->NJ); f->znode = zalloc(f->NK);
    f->U = zalloc(n3); f->V = zalloc(n3); f->W = zalloc(n3); f->P = zalloc(n3); f->D = zalloc(n3);
    f->T = zalloc(n3); f->C = zalloc(n3); f->Ma = zalloc(n3); f->Wav = zalloc(n3); f->Rgas = zalloc(n3);
    f->Cp = zalloc(n3); f->H = zalloc(n3); f->E = zalloc(n3); f->Gamma = zalloc(n3);
    f->Mc = zalloc(n3 * NS); f->Yi = zalloc(n3 * NS); f->Di = zalloc(n3 * NS);
    f->CS = zalloc(n3 * (NS + 4)); f->RHS = zalloc(n3 * (NS + 4)); f->Partion_T = zalloc(n3 * (NS + 4));
    f->F = zalloc(n3 * (NS + 4)); f->G = zalloc(n3 * (NS + 4)); f->Q = zalloc(n3 * (NS + 4));
    f->CMS = zalloc(n3 * NS); f->MDd = zalloc(n3 * (NS + 4));
    f->Nchem = (int *)calloc(n3, sizeof(int));
    for (size_t c = 0; c < n3; c++) f->Nchem[c] = 1;
    size_t n2 = (size_t)nj * nk;
    f->Uint = zalloc(n2); f->Vint = zalloc(n2); f->Wint = zalloc(n2); f->Pint = zalloc(n2); f->Dint = zalloc(n2);
    f->Tint = zalloc(n2); f->Hint = zalloc(n2); f->Eint = zalloc(n2); f->Gint = zalloc(n2);
    f->Yint = zalloc(n2 * NS);
    return f->Nchem ? 0 : -1;
}

void orc_field_free(orc_field *f)
{
    double **p[] = {&f->xnode, &f->ynode, &f->znode, &f->U, &f->V, &f->W, &f->P, &f->D, &f->T, &f->C, &f->Ma,
                    &f->Wav, &f->Rgas, &f->Cp, &f->H, &f->E, &f->Gamma, &f->Mc, &f->Yi, &f->Di, &f->CS, &f->RHS,
                    &f->Partion_T, &f->F, &f->G, &f->Q, &f->CMS, &f->MDd, &f->Uint, &f->Vint, &f->Wint,
                    &f->Pint, &f->Dint, &f->Tint, &f->Hint, &f->Eint, &f->Gint, &f->Yint};
    for (size_t a = 0; a < sizeof(p) / sizeof(p[0]); a++) { free(*p[a]); *p[a] = NULL; }
    free(f->Nchem);
    f->Nchem = NULL;
}

/* ---------------------------------------------------------------- thermo */
#define C0(k) m->c0[(k) * m->NS + sp]
#define C1(k) m->c1[(k) * m->NS + sp]

/* Reaction::GetCpi, src/Reaction.cpp:893-904 */
double orc_getcpi(const orc_mech *m, double T, double R, int sp)
{
    if (T < 1000)
        return R * (C0(0) * pow(T, -2) + C0(1) * pow(T, -1) + C0(2) + C0(3) * T + C0(4) * pow(T, 2) +
                    C0(5) * pow(T, 3) + C0(6) * pow(T, 4));
    return R * (C1(0) * pow(T, -2) + C1(1) * pow(T, -1) + C1(2) + C1(3) * T + C1(4) * pow(T, 2) +
                C1(5) * pow(T, 3) + C1(6) * pow(T, 4));
}

/* Reaction::GetHi, src/Reaction.cpp:916-926 (b1 quirk at :923) */
double orc_gethi(const orc_mech *m, double T, double R, int sp, unsigned q)
{
    if (T < 1000)
        return R * (-C0(0) * pow(T, -1) + C0(1) * log(T) + C0(2) * T + C0(3) * pow(T, 2) / 2 +
                    C0(4) * pow(T, 3) / 3 + C0(5) * pow(T, 4) / 4 + C0(6) * pow(T, 5) / 5 + C0(7));
    double b1 = (q & EU3D_Q_THERMO_B12_LOW) ? C0(7) : C1(7);
    return R * (-C1(0) * pow(T, -1) + C1(1) * log(T) + C1(2) * T + C1(3) * pow(T, 2) / 2 + C1(4) * pow(T, 3) / 3 +
                C1(5) * pow(T, 4) / 4 + C1(6) * pow(T, 5) / 5 + b1);
}

/* Reaction::GetSi, src/Reaction.cpp:938-948 (b2 quirk at :945) */
double orc_getsi(const orc_mech *m, double T, double R, int sp, unsigned q)
{
    if (T < 1000)
        return R * (-C0(0) * pow(T, -2) / 2 - C0(1) * pow(T, -1) + C0(2) * log(T) + C0(3) * T +
                    C0(4) * pow(T, 2) / 2 + C0(5) * pow(T, 3) / 3 + C0(6) * pow(T, 4) / 4 + C0(8));
    double b2 = (q & EU3D_Q_THERMO_B12_LOW) ? C0(8) : C1(8);
    return R * (-C1(0) * pow(T, -2) / 2 - C1(1) * pow(T, -1) + C1(2) * log(T) + C1(3) * T + C1(4) * pow(T, 2) / 2 +
                C1(5) * pow(T, 3) / 3 + C1(6) * pow(T, 4) / 4 + b2);
}
#undef C0
#undef C1

/* Function::sum flags 2 and 3, src/Function.cpp:17-42 */
static double sum_mul(int n, const double *a, const double *b)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += (a[i] * b[i]);
    return s;
}
static double sum_div(int n, const double *a, const double *b)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += (a[i] / b[i]);
    return s;
}

/* ------------------------------------------------------- reconstruction */
/* Minmod limiter, include/Differ.hpp:33-43 */
static double minmod(double R)
{
    double mm = 0.0;
    if (R > 0)
        mm = (1.0 < R) ? 1.0 : R; /* std::min(R, 1.0) */
    else
        mm = 0.0;
    return mm;
}

/* Third-order WENO (Jiang and Shu, J. Comput. Phys. 126, 1996; new -- the
   reference's WENO enum value has no scheme behind it): the state at the face
   of cell `ctr` towards `oth`, from the two-point candidates
   ctr + (ctr - far)/2 and ctr + (oth - ctr)/2 with linear weights 1/3, 2/3 and
   smoothness indicators (ctr - far)^2, (oth - ctr)^2, epsilon 1e-6:
   w0 = (1/3)/q0 / ((1/3)/q0 + (2/3)/q1) = q1 / (q1 + 2 q0), q = (eps + beta)^2. */
static double weno3(double far, double ctr, double oth)
{
    const double A0 = ctr - far, A1 = oth - ctr;
    double q0 = 1e-6 + A0 * A0, q1 = 1e-6 + A1 * A1;
    q0 = q0 * q0;
    q1 = q1 * q1;
    const double w0 = q1 / (q1 + 2.0 * q0);
    return ctr + 0.5 * (A1 + w0 * (A0 - A1));
}

/* MUSCL_2 with limiter 0 (include/Differ.hpp:149-238) or MUSCL_1
   (include/Differ.hpp:110-136), or WENO (above), into FLR (NI x NJ x NK x 2) */
static void muscl(const orc_field *f, int dir, int diff, const double *fi, size_t stride, double *FLR)
{
    const int bc = f->bc;
    const double kk = 1.0 / 3.0;
    for (int i = bc - 1; i < f->ni + bc; i++)
        for (int j = bc - 1; j < f->nj + bc; j++)
            for (int k = bc - 1; k < f->nk + bc; k++) {
                int di = dir == 1, dj = dir == 2, dk = dir == 3;
                double fm1 = fi[ID3(f, i - di, j - dj, k - dk) * stride];
                double f0 = fi[ID3(f, i, j, k) * stride];
                double f1 = fi[ID3(f, i + di, j + dj, k + dk) * stride];
                size_t o = ID3(f, i, j, k) * 2;
                if (diff == 0) {
                    FLR[o] = f0;
                    FLR[o + 1] = f1;
                    continue;
                }
                double f2 = fi[ID3(f, i + 2 * di, j + 2 * dj, k + 2 * dk) * stride];
                if (diff == EU3D_DIFF_WENO) {
                    FLR[o] = weno3(fm1, f0, f1);
                    FLR[o + 1] = weno3(f2, f1, f0);
                    continue;
                }
                double A0 = f0 - fm1;
                double A1 = f1 - f0;
                double A2 = f2 - f1;
                double L = A1 / (A0 + 1e-12);
                double R = A1 / (A2 + 1e-12);
                double L1 = minmod(L), L2 = minmod(1.0 / L), R1 = minmod(R), R2 = minmod(1.0 / R);
                FLR[o] = f0 + 0.25 * ((1.0 - kk) * L1 + (1 + kk) * L2 * L) * A0;
                FLR[o + 1] = f1 - 0.25 * ((1.0 - kk) * R1 + (1 + kk) * R2 * R) * A2;
            }
}

/* Flowfield::AUSM, src/Flowfield.cpp:1330-1502 */
static void ausm(orc_field *f, int dir, double *Fi, int diff)
{
    const int NS = f->NS, bc = f->bc;
    const size_t n3 = (size_t)f->NI * f->NJ * f->NK;
    double *LR[7];
    const double *src[7] = {f->P, f->D, f->U, f->V, f->W, f->H, f->Gamma};
    for (int a = 0; a < 7; a++) {
        LR[a] = zalloc(n3 * 2);
        muscl(f, dir, diff, src[a], 1, LR[a]);
    }
    double *YL = zalloc(n3 * NS), *YR = zalloc(n3 * NS), *YLR = zalloc(n3 * 2);
    const int ilim = (f->quirks & EU3D_Q_SPECIES_FACES) ? f->ni : f->ni + bc;
    for (int s = 0; s < NS; s++) {
        muscl(f, dir, diff, f->Yi + s, NS, YLR);
        for (int i = 1; i < ilim; i++)
            for (int j = 1; j < f->nj + bc; j++)
                for (int k = 1; k < f->nk + bc; k++) {
                    YL[ID4(f, i, j, k, s, NS)] = YLR[ID3(f, i, j, k) * 2];
                    YR[ID4(f, i, j, k, s, NS)] = YLR[ID3(f, i, j, k) * 2 + 1];
                }
    }
    for (int i = 1; i < f->ni + bc; i++)
        for (int j = 1; j < f->nj + bc; j++)
            for (int k = 1; k < f->nk + bc; k++) {
                size_t o = ID3(f, i, j, k) * 2;
                double PL = LR[0][o], PR = LR[0][o + 1], DL = LR[1][o], DR = LR[1][o + 1];
                double UL = LR[2][o], UR = LR[2][o + 1], VL = LR[3][o], VR = LR[3][o + 1];
                double WL = LR[4][o], WR = LR[4][o + 1], HL = LR[5][o], HR = LR[5][o + 1];
                double GL = LR[6][o], GR = LR[6][o + 1];
                double CL = sqrt(GL * PL / DL);
                double CR = sqrt(GR * PR / DR);
                double CI = 0.5 * (CL + CR);
                double MaL, MaR, B1, B2, G1, G2;
                if (dir == 1) { MaL = UL / CI; MaR = UR / CI; }
                else if (dir == 2) { MaL = VL / CI; MaR = VR / CI; }
                else { MaL = WL / CI; MaR = WR / CI; }
                if (fabs(MaL) < 1.0) {
                    B1 = 0.25 * pow((MaL + 1.0), 2) + 0.125 * pow((pow(MaL, 2) - 1.0), 2);
                    G1 = 0.25 * pow((MaL + 1.0), 2) * (2.0 - MaL) + 3.0 / 16.0 * MaL * pow((pow(MaL, 2) - 1.0), 2);
                } else {
                    B1 = 0.5 * (MaL + fabs(MaL));
                    G1 = B1 / MaL;
                }
                if (fabs(MaR) < 1.0) {
                    B2 = -0.25 * pow((MaR - 1.0), 2) - 0.125 * pow((pow(MaR, 2) - 1.0), 2);
                    G2 = 0.25 * pow((MaR - 1.0), 2) * (2.0 + MaR) - 3.0 / 16.0 * MaR * pow((pow(MaR, 2) - 1.0), 2);
                } else {
                    B2 = 0.5 * (MaR - fabs(MaR));
                    G2 = B2 / MaR;
                }
                double MaI = B1 + B2;
                double VI = MaI * CI;
                double *out = Fi + ID3(f, i, j, k) * (NS + 4);
                const double *Y = (VI >= 0.0) ? YL + ID4(f, i, j, k, 0, NS) : YR + ID4(f, i, j, k, 0, NS);
                double Ds = (VI >= 0.0) ? DL : DR, Us = (VI >= 0.0) ? UL : UR, Vs = (VI >= 0.0) ? VL : VR;
                double Ws = (VI >= 0.0) ? WL : WR, Hs = (VI >= 0.0) ? HL : HR;
                for (int s = 0; s < NS; s++) out[s] = VI * Ds * Y[s];
                out[NS] = VI * Ds * Us;
                out[NS + 1] = VI * Ds * Vs;
                out[NS + 2] = VI * Ds * Ws;
                if (dir == 1) out[NS] = VI * Ds * Us + G1 * PL + G2 * PR;
                if (dir == 2) out[NS + 1] = VI * Ds * Vs + G1 * PL + G2 * PR;
                if (dir == 3) out[NS + 2] = VI * Ds * Ws + G1 * PL + G2 * PR;
                out[NS + 3] = VI * (Ds * Hs + 0.5 * Ds * (pow(Us, 2) + pow(Vs, 2) + pow(Ws, 2)));
            }
    for (int a = 0; a < 7; a++) free(LR[a]);
    free(YL); free(YR); free(YLR);
}

/* TimeAdv::EE, src/TimeAdv.cpp:29-43 */
static void time_ee(orc_field *f)
{
    const int NS = f->NS, bc = f->bc;
    const double dt = f->dt;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++)
                for (int s = 0; s < NS + 4; s++)
                    f->RHS[ID4(f, i, j, k, s, NS + 4)] =
                        -dt / (f->xnode[i] - f->xnode[i - 1]) *
                            (f->F[ID4(f, i, j, k, s, NS + 4)] - f->F[ID4(f, i - 1, j, k, s, NS + 4)]) -
                        dt / (f->ynode[j] - f->ynode[j - 1]) *
                            (f->G[ID4(f, i, j, k, s, NS + 4)] - f->G[ID4(f, i, j - 1, k, s, NS + 4)]) -
                        dt / (f->znode[k] - f->znode[k - 1]) *
                            (f->Q[ID4(f, i, j, k, s, NS + 4)] - f->Q[ID4(f, i, j, k - 1, s, NS + 4)]);
}

/* Flowfield::Advection, src/Flowfield.cpp:1096-1128 */
void orc_advection(orc_field *f, int timeadv, int diff)
{
    const size_t n = (size_t)f->NI * f->NJ * f->NK * (f->NS + 4);
    memset(f->F, 0, n * sizeof(double));
    memset(f->G, 0, n * sizeof(double));
    memset(f->Q, 0, n * sizeof(double));
    ausm(f, 1, f->F, diff);
    ausm(f, 2, f->G, diff);
    ausm(f, 3, f->Q, diff);
    if (timeadv == EU3D_ADV_EE || timeadv == EU3D_ADV_SSPRK2) time_ee(f);
    /* EU3D_ADV_TVD_RK3: TimeAdv::TVD_RK3 leaves RHS as it is (src/TimeAdv.cpp:57-67) */
}

/* ------------------------------------------------------------ decoding */
/* Flowfield::Get_temp (the variant in use), src/Flowfield.cpp:1542-1566;
   Eval is the internal energy the Newton iteration targets */
static double get_temp_e(const orc_field *f, const orc_mech *m, double T, double Eval, const double *Y)
{
    const int NS = f->NS;
    double T0 = T, T_temp = T, temp1, temp2;
    double Cpi0[ORC_MAXS], Hi0[ORC_MAXS];
    int count = 0;
    while (count < 10) {
        T0 = T_temp;
        for (int s = 0; s < NS; s++) {
            Cpi0[s] = orc_getcpi(m, T0, m->ri[s], s);
            Hi0[s] = orc_gethi(m, T0, m->ri[s], s, f->quirks);
        }
        temp1 = (sum_mul(NS, Y, Hi0) - Eval * 1e-3) - sum_mul(NS, Y, m->ri) * T0;
        temp2 = sum_mul(NS, Y, Cpi0) - sum_mul(NS, Y, m->ri);
        T_temp = T0 - temp1 / temp2;
        if (fabs(T_temp - T0) < 1e-6)
            break;
        else
            count = count + 1;
    }
    return T_temp;
}

double orc_get_temp(const orc_field *f, const orc_mech *m, double T, int i, int j, int k, const double *Y)
{
    return get_temp_e(f, m, T, f->E[ID3(f, i, j, k)], Y);
}

/* Flowfield::Update_after_CS, field form src/Flowfield.cpp:1246-1284 and
   point form :1287-1319 (identical arithmetic) */
static void decode_cell(orc_field *f, const orc_mech *m, int i, int j, int k)
{
    const int NS = f->NS;
    const size_t c = ID3(f, i, j, k);
    const double *cs = f->CS + c * (NS + 4);
    double Y[ORC_MAXS], Cpi1[ORC_MAXS];
    double D = 0;
    for (int s = 0; s < NS; s++) {
        D += cs[s];
        f->Di[c * NS + s] = cs[s];
        f->Mc[c * NS + s] = f->Di[c * NS + s] / m->mw[s] * 1000;
    }
    f->D[c] = D;
    for (int s = 0; s < NS; s++) {
        f->Yi[c * NS + s] = cs[s] / D;
        Y[s] = f->Yi[c * NS + s];
    }
    double U = cs[NS] / D, V = cs[NS + 1] / D, W = cs[NS + 2] / D;
    double Enew = (cs[NS + 3] - 0.5 * D * (pow(U, 2) + pow(V, 2) + pow(W, 2))) / D;
    double Etarget = (f->quirks & EU3D_Q_STALE_E) ? f->E[c] : Enew;
    double T = get_temp_e(f, m, f->T[c], Etarget, Y);
    f->T[c] = T;
    f->U[c] = U;
    f->V[c] = V;
    f->W[c] = W;
    f->E[c] = Enew;
    f->Wav[c] = 1.0 / sum_div(NS, Y, m->mw);
    f->Rgas[c] = ORC_R * 1000 / f->Wav[c];
    f->P[c] = T * D * f->Rgas[c];
    f->H[c] = f->P[c] / D + f->E[c];
    for (int s = 0; s < NS; s++) Cpi1[s] = orc_getcpi(m, T, m->ri[s], s);
    f->Cp[c] = sum_mul(NS, Cpi1, Y) * 1000;
    f->Gamma[c] = f->Cp[c] / (f->Cp[c] - ORC_R * sum_div(NS, Y, m->mw) * 1000);
    f->C[c] = sqrt(f->Gamma[c] * f->P[c] / D);
    f->Ma[c] = sqrt(pow(U, 2) + pow(V, 2) + pow(W, 2)) / f->C[c];
}

void orc_update_after_cs(orc_field *f, const orc_mech *m)
{
    const int bc = f->bc;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) decode_cell(f, m, i, j, k);
}

/* Flowfield::Update_after_Adv, src/Flowfield.cpp:1140-1157 */
void orc_update_after_adv(orc_field *f, const orc_mech *m)
{
    const int NS = f->NS, bc = f->bc;
    const int nv = (f->quirks & EU3D_Q_ADV_SPECIES_ONLY) ? NS : NS + 4;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++)
                for (int s = 0; s < nv; s++)
                    f->CS[ID4(f, i, j, k, s, NS + 4)] = f->CS[ID4(f, i, j, k, s, NS + 4)] + f->RHS[ID4(f, i, j, k, s, NS + 4)];
    orc_update_after_cs(f, m);
}

/* Flowfield::GetPartial_T, src/Flowfield.cpp:1578-1595 */
void orc_get_partial_t(orc_field *f, const orc_mech *m)
{
    const int NS = f->NS, bc = f->bc;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                double CV = f->Cp[c] - f->Rgas[c];
                for (int s = 0; s < NS; s++) {
                    double Hi = orc_gethi(m, f->T[c], m->ri[s], s, f->quirks);
                    if (!(f->quirks & EU3D_Q_PARTIAL_T_UNITS)) Hi = Hi * 1e3;
                    f->Partion_T[c * (NS + 4) + s] =
                        (0.5 * (pow(f->U[c], 2) + pow(f->V[c], 2) + pow(f->W[c], 2)) - Hi + m->ri[s] * 1e3 * f->T[c]) /
                        (CV * f->D[c]);
                }
                f->Partion_T[c * (NS + 4) + NS + 1] = -f->U[c] / (CV * f->D[c]);
                f->Partion_T[c * (NS + 4) + NS + 2] = 1.0 / (CV * f->D[c]);
            }
}

/* ------------------------------------------------------------ chemistry */
typedef struct {
    double Hi[ORC_MAXS], Si[ORC_MAXS], Gi[ORC_MAXS], Wi[ORC_MAXS];
    double RR_F[ORC_MAXR], RR_B[ORC_MAXR], R_TB[ORC_MAXR], KF[ORC_MAXR], Kp[ORC_MAXR], Kc[ORC_MAXR],
        KB[ORC_MAXR], RR[ORC_MAXR];
} rates_t;

#define SF(s, r) m->stoi_f[(s) * m->NR + (r)]
#define SB(s, r) m->stoi_b[(s) * m->NR + (r)]
#define TBE(s, r) m->react_tb[(s) * m->NR + (r)]

/* rate evaluation shared by Trapezoid (src/Reaction.cpp:416-450, :493-530),
   TrapezoidPrediction (:600-640) and Diagonalized (:744-775).
   rtb_mode: 0 = `if (R_TB == 0) R_TB = 1` (Diagonalized), 1 = R_TB left as
   summed (field Trapezoid, `==` no-op), 2 = all R_TB set to 0 (adaptive,
   assignment in the condition). */
static void rates(const orc_mech *m, const double *Mc, double T_local, int rtb_mode, unsigned q, rates_t *ip)
{
    const int NS = m->NS, NR = m->NR;
    for (int s = 0; s < NS; s++) {
        ip->Hi[s] = orc_gethi(m, T_local, ORC_R, s, q);
        ip->Si[s] = orc_getsi(m, T_local, ORC_R, s, q);
        ip->Gi[s] = ip->Hi[s] - ip->Si[s] * T_local;
    }
    for (int r = 0; r < NR; r++) { ip->RR_F[r] = 1.0; ip->RR_B[r] = 1.0; ip->R_TB[r] = 0.0; }
    for (int r = 0; r < NR; r++) {
        double Xr = 0.0, delta_g = 0.0;
        ip->KF[r] = m->af[r] * pow(T_local, m->bf[r]) * exp(-m->eaf[r] / (ORC_RU * T_local));
        for (int s = 0; s < NS; s++) {
            Xr += (SB(s, r) - SF(s, r));
            delta_g += (SB(s, r) - SF(s, r)) * ip->Gi[s];
            ip->RR_F[r] *= pow(Mc[s], SF(s, r));
            ip->RR_B[r] *= pow(Mc[s], SB(s, r));
            ip->R_TB[r] += Mc[s] * TBE(s, r);
        }
        ip->Kp[r] = exp(-delta_g / (ORC_R * T_local)) * pow((ORC_P0 * 1e-6), Xr);
        ip->Kc[r] = ip->Kp[r] * pow(ORC_R * T_local, -Xr);
        ip->KB[r] = ip->KF[r] / ip->Kc[r];
        if (rtb_mode == 0) {
            if (ip->R_TB[r] == 0.0) ip->R_TB[r] = 1.0;
        } else if (rtb_mode == 2) {
            ip->R_TB[r] = 0.0;
        }
        ip->RR[r] = ip->KF[r] * ip->RR_F[r] - ip->KB[r] * ip->RR_B[r];
    }
    for (int s = 0; s < NS; s++) {
        double temp = 0.0;
        for (int r = 0; r < NR; r++) temp += (SB(s, r) - SF(s, r)) * ip->R_TB[r] * ip->RR[r];
        ip->Wi[s] = m->mw[s] * temp;
    }
}

/* Reaction::Diagonalized, src/Reaction.cpp:736-811 */
void orc_diagonalized(orc_field *f, const orc_mech *m)
{
    const int NS = f->NS, NR = m->NR, bc = f->bc;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                const double T_local = f->T[c];
                double Di[ORC_MAXS], Mc[ORC_MAXS];
                double WJH1[ORC_MAXS][ORC_MAXR], WJH2[ORC_MAXS][ORC_MAXR];
                rates_t ip;
                for (int s = 0; s < NS; s++) {
                    Di[s] = f->Di[c * NS + s] * 1e-3;
                    Mc[s] = f->Mc[c * NS + s] * 1e-6;
                }
                rates(m, Mc, T_local, 0, f->quirks, &ip);
                for (int s = 0; s < NS; s++) f->CMS[c * NS + s] = ip.Wi[s] * 1e3;
                for (int r = 0; r < NR; r++)
                    for (int s = 0; s < NS; s++) {
                        if (Di[s] == 0)
                            WJH1[s][r] = 0.0;
                        else
                            WJH1[s][r] = ip.KF[r] * SF(s, r) * ip.RR_F[r] / Di[s] - ip.KB[r] * SB(s, r) * ip.RR_B[r] / Di[s];
                        WJH2[s][r] = ip.RR[r] * (m->bf[r] / T_local + m->eaf[r] / (ORC_RU * pow(T_local, 2)));
                    }
                for (int s = 0; s < NS; s++) {
                    double temp = 0.0;
                    for (int r = 0; r < NR; r++)
                        temp += (SB(s, r) - SF(s, r)) *
                                ((WJH1[s][r] + WJH2[s][r] * f->Partion_T[c * (NS + 4) + s]) * ip.R_TB[r] +
                                 ip.RR[r] * TBE(s, r) / m->mw[s]);
                    f->MDd[c * (NS + 4) + s] = m->mw[s] * temp;
                }
            }
}

/* Flowfield::Update_IMEX, src/Flowfield.cpp:1215-1234.  MD(v, v) for v >= NS
   is never written by Diagonalized and reads as zero (MDd stays 0 there). */
void orc_update_imex(orc_field *f, const orc_mech *m)
{
    const int NS = f->NS, bc = f->bc;
    const double dt = f->dt;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                double *rhs = f->RHS + c * (NS + 4), *cs = f->CS + c * (NS + 4);
                for (int s = 0; s < NS; s++) rhs[s] = rhs[s] + f->CMS[c * NS + s] * dt;
                for (int s = 0; s < NS + 4; s++) cs[s] = cs[s] + rhs[s] / (1.0 - dt * f->MDd[c * (NS + 4) + s]);
            }
    orc_update_after_cs(f, m);
    orc_get_partial_t(f, m);
}

/* Euler::IMEX, src/Euler.cpp:748-760 */
void orc_imex(orc_field *f, const orc_mech *m)
{
    orc_diagonalized(f, m);
    orc_update_imex(f, m);
}

/* point-implicit trapezoid update of one cell's partial densities
   (src/Reaction.cpp:464-482 / :566-589).  Di_kg are kg/m^3 values;
   writes kg/m^3 results into out. */
static void trapezoid_cell(const orc_mech *m, const double *Di_kg, const double *Mc_mol, double T_local, double dt,
                           int rtb_mode, unsigned q, double *out, double *cms)
{
    const int NS = m->NS, NR = m->NR;
    double Di[ORC_MAXS], Mc[ORC_MAXS], Pv[ORC_MAXS], Qv[ORC_MAXS];
    rates_t ip;
    for (int s = 0; s < NS; s++) {
        Di[s] = Di_kg[s] * 1e-3;
        Mc[s] = Mc_mol[s] * 1e-6;
    }
    rates(m, Mc, T_local, rtb_mode, q, &ip);
    for (int s = 0; s < NS; s++) {
        if (cms) cms[s] = ip.Wi[s] * 1e3;
        Pv[s] = 0;
        Qv[s] = 0;
    }
    for (int s = 0; s < NS; s++) {
        for (int r = 0; r < NR; r++) {
            Qv[s] += (SB(s, r) * ip.KF[r] * ip.RR_F[r] + SF(s, r) * ip.KB[r] * ip.RR_B[r] * ip.R_TB[r]);
            Pv[s] += (SB(s, r) * ip.KB[r] * ip.RR_B[r] + SF(s, r) * ip.KF[r] * ip.RR_F[r] * ip.R_TB[r]);
        }
        Qv[s] = m->mw[s] * Qv[s];
        if (Mc[s] == 0)
            Pv[s] = 0.0;
        else
            Pv[s] = Pv[s] / Mc[s];
        out[s] = ((1.0 - dt / 2.0 * Pv[s]) * Di[s] + dt * Qv[s]) / (1.0 + dt / 2.0 * Pv[s]) * 1e3;
    }
}

/* Flowfield::Explicit() field form, src/Flowfield.cpp:1169-1186, without the
   trailing decode */
static void explicit_encode_field(orc_field *f)
{
    const int NS = f->NS, bc = f->bc;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                double *cs = f->CS + c * (NS + 4);
                double D = 0.0;
                for (int s = 0; s < NS; s++) {
                    cs[s] = f->Di[c * NS + s];
                    D += cs[s];
                }
                f->D[c] = D;
                double U = f->U[c], V = f->V[c], W = f->W[c], E = f->E[c];
                cs[NS] = U * D;
                cs[NS + 1] = V * D;
                if (f->quirks & EU3D_Q_EXPLICIT_ENERGY) {
                    cs[NS + 2] = D * E + 0.5 * (pow(U, 2) + pow(V, 2) + pow(W, 2)) * D;
                } else {
                    cs[NS + 2] = W * D;
                    cs[NS + 3] = D * E + 0.5 * (pow(U, 2) + pow(V, 2) + pow(W, 2)) * D;
                }
            }
}

void orc_explicit(orc_field *f, const orc_mech *m)
{
    explicit_encode_field(f);
    orc_update_after_cs(f, m);
}

/* Reaction::TrapezoidPrediction, src/Reaction.cpp:593-670 */
void orc_prediction(orc_field *f, const orc_mech *m)
{
    const int NS = f->NS, bc = f->bc;
    const double dtm = f->dt;
    const int rtb = (f->quirks & EU3D_Q_ADAPT_RTB_ZERO) ? 2 : 0;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                double dt = dtm, dt_temp;
                double Mc[ORC_MAXS], Di[ORC_MAXS];
                rates_t ip;
                for (int s = 0; s < NS; s++) {
                    Di[s] = f->Di[c * NS + s] * 1e-3;
                    Mc[s] = f->Mc[c * NS + s] * 1e-6;
                }
                rates(m, Mc, f->T[c], rtb, f->quirks, &ip);
                for (int s = 0; s < NS; s++)
                    if (f->Yi[c * NS + s] >= 1e-6)
                        if (ip.Wi[s] != 0) {
                            dt_temp = fabs(-Di[s] / ip.Wi[s]);
                            if (dt_temp < dt) dt = dt_temp;
                        }
                /* the reference aborts when the count overflows int
                   (src/Reaction.cpp:662-668); here, as on the device, the
                   count is clamped to ORC_NCHEM_CAP */
                double n = ceil(dtm / dt);
                if (!(n >= 1.0)) n = 1.0;
                if (n > ORC_NCHEM_CAP) n = ORC_NCHEM_CAP;
                f->Nchem[c] = (int)n;
            }
}

/* Euler::Trapezoid(type) on one rank, src/Euler.cpp:357-737 */
void orc_trapezoid(orc_field *f, const orc_mech *m, int type)
{
    const int NS = f->NS, bc = f->bc;
    orc_update_after_adv(f, m);
    if (type == 0) {
        /* Reaction::Trapezoid field form, src/Reaction.cpp:412-485 */
        const int rtb = (f->quirks & EU3D_Q_TRAP_RTB_ZERO) ? 1 : 0;
        for (int i = bc; i < f->ni + bc; i++)
            for (int j = bc; j < f->nj + bc; j++)
                for (int k = bc; k < f->nk + bc; k++) {
                    size_t c = ID3(f, i, j, k);
                    double out[ORC_MAXS];
                    trapezoid_cell(m, f->Di + c * NS, f->Mc + c * NS, f->T[c], f->dt, rtb, f->quirks, out,
                                   f->CMS + c * NS);
                    for (int s = 0; s < NS; s++) f->Di[c * NS + s] = out[s];
                }
        orc_explicit(f, m);
        return;
    }
    orc_prediction(f, m);
    const int rtb = (f->quirks & EU3D_Q_ADAPT_RTB_ZERO) ? 2 : 0;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                for (int step = 0; step < f->Nchem[c]; step++) {
                    /* per-cell Reaction::Trapezoid, src/Reaction.cpp:489-591 */
                    double dt = f->dt / f->Nchem[c];
                    double out[ORC_MAXS];
                    trapezoid_cell(m, f->Di + c * NS, f->Mc + c * NS, f->T[c], dt, rtb, f->quirks, out,
                                   f->CMS + c * NS);
                    for (int s = 0; s < NS; s++) f->Di[c * NS + s] = out[s];
                    /* Flowfield::Explicit(step,i,j,k), src/Flowfield.cpp:1189-1203 */
                    double *cs = f->CS + c * (NS + 4);
                    double D = 0.0;
                    for (int s = 0; s < NS; s++) {
                        cs[s] = f->Di[c * NS + s];
                        D += cs[s];
                    }
                    f->D[c] = D;
                    double U = f->U[c], V = f->V[c], W = f->W[c], E = f->E[c];
                    cs[NS] = U * D;
                    cs[NS + 1] = V * D;
                    cs[NS + 2] = W * D;
                    cs[NS + 3] = D * E + 0.5 * (pow(U, 2) + pow(V, 2) + pow(W, 2)) * D;
                    decode_cell(f, m, i, j, k);
                }
            }
}
#undef SF
#undef SB
#undef TBE

/* ------------------------------------------------------------- ghosts */
/* ghost thermo recompute used by the reflective faces of
   FieldBoundary_3dRSBI (y-lower, src/Flowfield.cpp:619-647) and
   FieldBoundary_3dODM (src/Flowfield.cpp:409-436 and the other walls) */
static void ghost_thermo(orc_field *f, const orc_mech *m, size_t c)
{
    const int NS = f->NS;
    double Y[ORC_MAXS], Cpi[ORC_MAXS], Hi[ORC_MAXS], Ei[ORC_MAXS];
    const double T = f->T[c];
    for (int s = 0; s < NS; s++) {
        Y[s] = f->Yi[c * NS + s];
        Cpi[s] = orc_getcpi(m, T, m->ri[s], s);
        Hi[s] = orc_gethi(m, T, m->ri[s], s, f->quirks);
        Ei[s] = Hi[s] - m->ri[s] * T;
    }
    f->Rgas[c] = sum_mul(NS, Y, m->ri) * 1000;
    f->D[c] = f->P[c] / (T * f->Rgas[c]);
    f->Cp[c] = sum_mul(NS, Cpi, Y) * 1000;
    f->H[c] = sum_mul(NS, Y, Hi) * 1000;
    f->E[c] = sum_mul(NS, Y, Ei) * 1000;
    f->Gamma[c] = f->Cp[c] / (f->Cp[c] - f->Rgas[c]);
}

/* copy every field the flux sweeps read from cell s to cell d */
static void ghost_copy(orc_field *f, size_t d, size_t s)
{
    const int NS = f->NS;
    f->U[d] = f->U[s]; f->V[d] = f->V[s]; f->W[d] = f->W[s]; f->P[d] = f->P[s]; f->D[d] = f->D[s];
    f->T[d] = f->T[s]; f->H[d] = f->H[s]; f->Gamma[d] = f->Gamma[s]; f->E[d] = f->E[s];
    for (int q = 0; q < NS; q++) f->Yi[d * NS + q] = f->Yi[s * NS + q];
}

/* wall mirror with thermo recompute; sign flips the wall-normal velocity */
static void ghost_wall(orc_field *f, const orc_mech *m, size_t d, size_t s, int flipv, int flipw)
{
    const int NS = f->NS;
    f->U[d] = f->U[s];
    f->V[d] = flipv ? -f->V[s] : f->V[s];
    f->W[d] = flipw ? -f->W[s] : f->W[s];
    f->P[d] = f->P[s];
    f->T[d] = f->T[s];
    for (int q = 0; q < NS; q++) {
        f->Yi[d * NS + q] = f->Yi[s * NS + q];
        f->Mc[d * NS + q] = f->Mc[s * NS + q];
    }
    ghost_thermo(f, m, d);
}

/* wedge immersed boundary (new): cells whose centre lies below the line
   y = y0 + (x - x0) * tan(theta), x > x0, are solid.  Solid cells within
   three cells of the surface take the state of the fluid cell nearest to
   their mirror image across the surface, with the velocity reflected
   (v' = v - 2 (v.n) n); deeper solid cells take the state of the nearest
   band cell's source with zero velocity. */
int orc_wedge_solid(const double *w, double x, double y)
{
    return x > w[0] && (y - w[1]) < (x - w[0]) * w[2];
}

static void wedge_fill(orc_field *f, const orc_mech *m, const double *w)
{
    (void)m;
    const double x0 = w[0], y0 = w[1], tn = w[2];
    const double cs = 1.0 / sqrt(1.0 + tn * tn), sn = tn * cs; /* cos, sin of the wedge angle */
    const double nx = -sn, ny = cs;                            /* unit normal into the fluid */
    const double dx = f->xnode[f->bc + 1] - f->xnode[f->bc];
    const double dy = f->ynode[f->bc + 1] - f->ynode[f->bc];
    for (int i = 0; i < f->NI; i++)
        for (int j = 0; j < f->NJ; j++) {
            double x = f->xnode[i], y = f->ynode[j];
            if (!orc_wedge_solid(w, x, y)) continue;
            /* only the band the flux stencils reach: a fluid cell within two
               cells along x or y */
            int band = 0;
            for (int o = -2; o <= 2 && !band; o++) {
                if (o == 0) continue;
                if (i + o >= 0 && i + o < f->NI && !orc_wedge_solid(w, f->xnode[i + o], y)) band = 1;
                if (j + o >= 0 && j + o < f->NJ && !orc_wedge_solid(w, x, f->ynode[j + o])) band = 1;
            }
            if (!band) continue;
            double dist = ((x - x0) * sn - (y - y0) * cs); /* depth below the surface, >= 0 */
            double xi = x + 2.0 * dist * nx, yi = y + 2.0 * dist * ny;
            int si = (int)floor((xi - f->xnode[0]) / dx + 0.5);
            int sj = (int)floor((yi - f->ynode[0]) / dy + 0.5);
            if (si < 0) si = 0;
            if (si > f->NI - 1) si = f->NI - 1;
            if (sj < 0) sj = 0;
            if (sj > f->NJ - 1) sj = f->NJ - 1;
            /* walk up until the source is a fluid cell */
            while (sj < f->NJ - 1 && orc_wedge_solid(w, f->xnode[si], f->ynode[sj])) sj++;
            for (int k = 0; k < f->NK; k++) {
                size_t d = ID3(f, i, j, k), s = ID3(f, si, sj, k);
                ghost_copy(f, d, s);
                double u = f->U[s], v = f->V[s];
                double un = u * nx + v * ny;
                f->U[d] = u - 2.0 * un * nx;
                f->V[d] = v - 2.0 * un * ny;
            }
        }
}

void orc_boundary(orc_field *f, const orc_mech *m, int kind, const double *wedge)
{
    const int ni = f->ni, nj = f->nj, nk = f->nk, bc = f->bc, NI = f->NI, NJ = f->NJ;
    if (kind == EU3D_BC_RSBI || kind == EU3D_BC_TRANSMISSIVE) {
        /* FieldBoundary_3dRSBI, src/Flowfield.cpp:559-773; the transmissive
           variant copies the outermost interior cell into the x ghosts */
        const int transm = kind == EU3D_BC_TRANSMISSIVE;
        for (int i = 0; i < bc; i++)
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) ghost_copy(f, ID3(f, i, j, k), ID3(f, transm ? bc : 2 * bc - 1 - i, j, k));
        for (int i = ni + bc; i < ni + 2 * bc; i++)
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++)
                    ghost_copy(f, ID3(f, i, j, k), ID3(f, transm ? ni + bc - 1 : 2 * (ni + bc) - 1 - i, j, k));
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < bc; j++)
                for (int k = bc; k < nk + bc; k++) {
                    if (transm)
                        ghost_copy(f, ID3(f, i, j, k), ID3(f, i, 2 * bc - 1 - j, k));
                    else
                        ghost_wall(f, m, ID3(f, i, j, k), ID3(f, i, 2 * bc - 1 - j, k), 0, 0);
                }
        for (int i = 0; i < NI; i++)
            for (int j = nj + bc; j < nj + 2 * bc; j++)
                for (int k = bc; k < nk + bc; k++) ghost_copy(f, ID3(f, i, j, k), ID3(f, i, 2 * (nj + bc) - 1 - j, k));
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < NJ; j++)
                for (int k = 0; k < bc; k++) ghost_copy(f, ID3(f, i, j, k), ID3(f, i, j, 2 * bc - 1 - k));
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < NJ; j++)
                for (int k = nk + bc; k < nk + 2 * bc; k++) ghost_copy(f, ID3(f, i, j, k), ID3(f, i, j, 2 * (nk + bc) - 1 - k));
    } else if (kind == EU3D_BC_ODM) {
        /* FieldBoundary_3dODM, src/Flowfield.cpp:378-558 */
        const int NS = f->NS;
        for (int i = 0; i < bc; i++)
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) {
                    size_t c = ID3(f, i, j, k), p = (size_t)(j - bc) * nk + (k - bc);
                    f->U[c] = f->Uint[p]; f->V[c] = f->Vint[p]; f->W[c] = f->Wint[p]; f->P[c] = f->Pint[p];
                    f->D[c] = f->Dint[p]; f->T[c] = f->Tint[p]; f->H[c] = f->Hint[p]; f->Gamma[c] = f->Gint[p];
                    f->E[c] = f->Eint[p];
                    for (int s = 0; s < NS; s++) f->Yi[c * NS + s] = f->Yint[p * NS + s];
                }
        for (int i = ni + bc; i < ni + 2 * bc; i++)
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++)
                    ghost_wall(f, m, ID3(f, i, j, k), ID3(f, 2 * (ni + bc) - 1 - i, j, k), 0, 0);
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < bc; j++)
                for (int k = bc; k < nk + bc; k++) ghost_wall(f, m, ID3(f, i, j, k), ID3(f, i, 2 * bc - 1 - j, k), 1, 0);
        for (int i = 0; i < NI; i++)
            for (int j = nj + bc; j < nj + 2 * bc; j++)
                for (int k = bc; k < nk + bc; k++) ghost_copy(f, ID3(f, i, j, k), ID3(f, i, 2 * (nj + bc) - 1 - j, k));
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < NJ; j++)
                for (int k = 0; k < bc; k++) ghost_wall(f, m, ID3(f, i, j, k), ID3(f, i, j, 2 * bc - 1 - k), 0, 1);
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < NJ; j++)
                for (int k = nk + bc; k < nk + 2 * bc; k++)
                    ghost_wall(f, m, ID3(f, i, j, k), ID3(f, i, j, 2 * (nk + bc) - 1 - k), 0, 1);
    }
    if (wedge) wedge_fill(f, m, wedge);
}

/* Flowfield::CFLcondition, src/Flowfield.cpp:242-272 (single rank); with a
   wedge (new) its solid cells are left out, as the device reduction does. */
static void cfl_scan(orc_field *f, double cfl, double final_time, const double *wedge)
{
    const int bc = f->bc;
    double dx = f->xnode[1] - f->xnode[0];
    double dy = f->ynode[1] - f->ynode[0];
    double dz = f->znode[1] - f->znode[0];
    double dt_conv = 1e10, temp;
    for (int i = bc; i < f->ni + bc; i++)
        for (int j = bc; j < f->nj + bc; j++)
            for (int k = bc; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                if (wedge && orc_wedge_solid(wedge, f->xnode[i], f->ynode[j])) continue;
                double a = dx / (fabs(f->U[c]) + f->C[c]), b = dy / (fabs(f->V[c]) + f->C[c]);
                temp = (b < a) ? b : a;
                if (!(f->quirks & EU3D_Q_CFL_NO_Z)) {
                    double z = dz / (fabs(f->W[c]) + f->C[c]);
                    temp = (z < temp) ? z : temp;
                }
                if (temp < dt_conv) dt_conv = temp;
            }
    f->dt = cfl * dt_conv;
    if (f->time + f->dt > final_time) f->dt = final_time - f->time;
    f->time += f->dt;
}

void orc_cfl(orc_field *f, double cfl, double final_time) { cfl_scan(f, cfl, final_time, NULL); }

void orc_step(orc_field *f, const orc_mech *m, int react, int type, int timeadv, int diff, double cfl,
              double final_time, int bc_kind, const double *wedge)
{
    const int NS = f->NS, bc = f->bc;
    if (cfl != 0) cfl_scan(f, cfl, final_time, wedge);
    orc_boundary(f, m, bc_kind, wedge);
    if (timeadv == EU3D_ADV_SSPRK2 || timeadv == EU3D_ADV_SSPRK3) {
        /* SSP Runge-Kutta for the advection (new), followed by the chemistry
           as a split step with a zero flux residual.  Two stages:
           CS1 = CS^n + R(CS^n), CS^{n+1} = 1/2 CS^n + 1/2 (CS1 + R(CS1)).
           Three (Shu-Osher): CS1 as above, CS2 = 3/4 CS^n + 1/4 (CS1 + R(CS1)),
           CS^{n+1} = 1/3 CS^n + 2/3 (CS2 + R(CS2)). */
        const int stages = timeadv == EU3D_ADV_SSPRK2 ? 2 : 3;
        size_t n = (size_t)f->NI * f->NJ * f->NK * (NS + 4);
        double *cs0 = (double *)malloc(n * sizeof(double));
        memcpy(cs0, f->CS, n * sizeof(double));
        orc_advection(f, EU3D_ADV_EE, diff);
        for (int i = bc; i < f->ni + bc; i++)
            for (int j = bc; j < f->nj + bc; j++)
                for (int k = bc; k < f->nk + bc; k++)
                    for (int s = 0; s < NS + 4; s++) f->CS[ID4(f, i, j, k, s, NS + 4)] += f->RHS[ID4(f, i, j, k, s, NS + 4)];
        orc_update_after_cs(f, m);
        for (int stage = 2; stage <= stages; stage++) {
            const double wn = stages == 2 ? 0.5 : stage == 2 ? 0.75 : 1.0 / 3.0;
            const double ws = stages == 2 ? 0.5 : stage == 2 ? 0.25 : 2.0 / 3.0;
            orc_boundary(f, m, bc_kind, wedge);
            orc_advection(f, EU3D_ADV_EE, diff);
            for (int i = bc; i < f->ni + bc; i++)
                for (int j = bc; j < f->nj + bc; j++)
                    for (int k = bc; k < f->nk + bc; k++)
                        for (int s = 0; s < NS + 4; s++) {
                            size_t o = ID4(f, i, j, k, s, NS + 4);
                            f->CS[o] = wn * cs0[o] + ws * (f->CS[o] + f->RHS[o]);
                        }
            if (stage < stages) orc_update_after_cs(f, m);
        }
        free(cs0);
        orc_update_after_cs(f, m);
        memset(f->RHS, 0, n * sizeof(double));
        if (react == EU3D_REACT_IMEX) {
            orc_get_partial_t(f, m);
            orc_imex(f, m);
        } else if (react == EU3D_REACT_TRAPEZOID) {
            orc_trapezoid(f, m, type);
        }
        return;
    }
    orc_advection(f, timeadv, diff);
    if (react == EU3D_REACT_TRAPEZOID)
        orc_trapezoid(f, m, type);
    else if (react == EU3D_REACT_IMEX)
        orc_imex(f, m);
    else {
        /* Euler::DNN, src/Euler.cpp:773-780 */
        orc_update_after_adv(f, m);
        orc_explicit(f, m);
    }
}

/* ReactionInitial (src/Reaction.cpp:339-398) + FieldInitial
   (src/Flowfield.cpp:159-230) for the shipped RSBI case */
void orc_rsbi_initial(orc_field *f, const orc_mech *m, double P_pre, double T_pre, double M_wave)
{
    const int NS = f->NS, bc = f->bc;
    const double cx = 0.038, cy = 0.0, Ir = 0.022, Or = 1.2 * Ir, alpha = 5;
    double *Yr = zalloc((size_t)f->NI * f->NJ * f->NK * NS);
    for (int i = 0; i < f->NI; i++)
        for (int j = 0; j < f->NJ; j++)
            for (int k = 0; k < f->NK; k++) {
                double Mr[ORC_MAXS] = {0}, Mr_SUM = 0.0, Total_Mw = 0.0;
                double *Y = Yr + ID4(f, i, j, k, 0, NS);
                double d2 = pow(f->xnode[i] - cx, 2) + pow(f->ynode[j] - cy, 2);
                if (d2 > pow(Or, 2) || d2 < pow(Ir, 2)) {
                    if (d2 > pow(Or, 2)) { Mr[4] = 1.0; Mr[8] = 3.76; }
                    else Mr[5] = 1.0;
                    for (int s = 0; s < NS; s++) { Mr_SUM += Mr[s]; Total_Mw += Mr[s] * m->mw[s]; }
                    for (int s = 0; s < NS; s++) Y[s] = Mr[s] * m->mw[s] / Total_Mw;
                } else {
                    double r = sqrt(d2);
                    Y[5] = exp(-alpha * pow((r - Ir) / (Or - Ir), 2));
                    Y[4] = (1 - Y[5]) * m->mw[4] / (m->mw[4] + 3.76 * m->mw[8]);
                    Y[8] = (1 - Y[5]) * 3.76 * m->mw[8] / (m->mw[4] + 3.76 * m->mw[8]);
                }
            }
    f->dt = 0.0;
    f->time = 0.0;
    double U_post = M_wave * (1 - (2 + 0.40 * pow(M_wave, 2)) / (2.40 * pow(M_wave, 2))) * sqrt(1.40 * 287 * T_pre);
    double P_post = P_pre * (1 + 2 * 1.4 / 2.4 * (pow(M_wave, 2) - 1.0));
    double T_post = T_pre * (2 + 0.40 * pow(M_wave, 2)) / (2.40 * pow(M_wave, 2)) * P_post / P_pre;
    for (int i = 0; i < f->NI; i++)
        for (int j = 0; j < f->NJ; j++)
            for (int k = 0; k < f->NK; k++) {
                size_t c = ID3(f, i, j, k);
                f->W[c] = 0.0;
                f->V[c] = 0.0;
                if (f->xnode[i] >= 0.01) { f->P[c] = P_pre; f->T[c] = T_pre; f->U[c] = 0.0; }
                else { f->P[c] = P_post; f->T[c] = T_post; f->U[c] = U_post; }
            }
    for (int i = 0; i < f->ni + bc; i++)
        for (int j = 0; j < f->nj + bc; j++)
            for (int k = 0; k < f->nk + bc; k++) {
                size_t c = ID3(f, i, j, k);
                const double *Y = Yr + c * NS;
                double Cpi[ORC_MAXS], Hi[ORC_MAXS], Ei[ORC_MAXS];
                f->Wav[c] = 1.0 / sum_div(NS, Y, m->mw);
                f->Rgas[c] = ORC_R * 1000 / f->Wav[c];
                f->D[c] = f->P[c] / (f->Rgas[c] * f->T[c]);
                for (int s = 0; s < NS; s++) {
                    f->Yi[c * NS + s] = Y[s];
                    f->Di[c * NS + s] = f->Yi[c * NS + s] * f->D[c];
                    f->Mc[c * NS + s] = f->Di[c * NS + s] / m->mw[s] * 1000;
                    Cpi[s] = orc_getcpi(m, f->T[c], m->ri[s], s);
                    Hi[s] = orc_gethi(m, f->T[c], m->ri[s], s, f->quirks);
                    Ei[s] = Hi[s] - m->ri[s] * f->T[c];
                }
                f->Cp[c] = sum_mul(NS, Cpi, Y) * 1000;
                f->H[c] = sum_mul(NS, Y, Hi) * 1000;
                f->E[c] = sum_mul(NS, Y, Ei) * 1000;
                f->Gamma[c] = f->Cp[c] / (f->Cp[c] - ORC_R * sum_div(NS, Y, m->mw) * 1000);
                f->C[c] = sqrt(f->Gamma[c] * f->P[c] / f->D[c]);
                double *cs = f->CS + c * (NS + 4);
                for (int s = 0; s < NS; s++) cs[s] = f->D[c] * f->Yi[c * NS + s];
                cs[NS] = f->D[c] * f->U[c];
                cs[NS + 1] = f->D[c] * f->V[c];
                cs[NS + 2] = f->D[c] * f->W[c];
                cs[NS + 3] = f->D[c] * f->E[c] + 0.5 * (pow(f->U[c], 2) + pow(f->V[c], 2) + pow(f->W[c], 2)) * f->D[c];
            }
    free(Yr);
    orc_get_partial_t(f, m);
}

/* Derived primitives from (P, T, U, V, W, Yi) for every cell, with the
   arithmetic of FieldInitial (src/Flowfield.cpp:193-229): used to build
   consistent synthetic states for tests and benchmarks. */
void orc_prims_from_state(orc_field *f, const orc_mech *m)
{
    const int NS = f->NS;
    for (int i = 0; i < f->NI; i++)
        for (int j = 0; j < f->NJ; j++)
            for (int k = 0; k < f->NK; k++) {
                size_t c = ID3(f, i, j, k);
                const double *Y = f->Yi + c * NS;
                double Cpi[ORC_MAXS], Hi[ORC_MAXS], Ei[ORC_MAXS];
                f->Wav[c] = 1.0 / sum_div(NS, Y, m->mw);
                f->Rgas[c] = ORC_R * 1000 / f->Wav[c];
                f->D[c] = f->P[c] / (f->Rgas[c] * f->T[c]);
                for (int s = 0; s < NS; s++) {
                    f->Di[c * NS + s] = Y[s] * f->D[c];
                    f->Mc[c * NS + s] = f->Di[c * NS + s] / m->mw[s] * 1000;
                    Cpi[s] = orc_getcpi(m, f->T[c], m->ri[s], s);
                    Hi[s] = orc_gethi(m, f->T[c], m->ri[s], s, f->quirks);
                    Ei[s] = Hi[s] - m->ri[s] * f->T[c];
                }
                f->Cp[c] = sum_mul(NS, Cpi, Y) * 1000;
                f->H[c] = sum_mul(NS, Y, Hi) * 1000;
                f->E[c] = sum_mul(NS, Y, Ei) * 1000;
                f->Gamma[c] = f->Cp[c] / (f->Cp[c] - ORC_R * sum_div(NS, Y, m->mw) * 1000);
                f->C[c] = sqrt(f->Gamma[c] * f->P[c] / f->D[c]);
                double *cs = f->CS + c * (NS + 4);
                for (int s = 0; s < NS; s++) cs[s] = f->D[c] * Y[s];
                cs[NS] = f->D[c] * f->U[c];
                cs[NS + 1] = f->D[c] * f->V[c];
                cs[NS + 2] = f->D[c] * f->W[c];
                cs[NS + 3] = f->D[c] * f->E[c] + 0.5 * (pow(f->U[c], 2) + pow(f->V[c], 2) + pow(f->W[c], 2)) * f->D[c];
            }
    orc_get_partial_t(f, m);
}
