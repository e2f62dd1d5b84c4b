// Flux sweeps: MUSCL reconstruction with the minmod limiter, AUSM splitting
// and the TimeAdv EE residual, fused into one kernel over interior cells.
//
// Reference: Flowfield::Advection (src/Flowfield.cpp:1096-1128),
// Flowfield::AUSM (:1330-1502), MUSCL_1/MUSCL_2 + Minmod
// (include/Differ.hpp:33-43, :110-238), TimeAdv::EE (src/TimeAdv.cpp:29-43).
//
// The reference materialises left/right states of 16 primitives per
// direction into full-size arrays, then face fluxes F, G, Q, then RHS.  Here
// no intermediate array exists: k_advection gives each interior cell one
// thread, which reconstructs the two faces of the cell in each direction from
// the primitives (read through the read-only cache) and writes only the
// residual
//     RHS = -dt/dx (F_i - F_{i-1}) - dt/dy (G_j - G_{j-1}) - dt/dz (Q_k - Q_{k-1})
// accumulated in FP64 in the reference's operation order.  Reconstruction
// and AUSM run in P (double or float); differences and the residual in FP64.
#pragma once

#include "common.cuh"

namespace eu3d {

template <class P>
__device__ __forceinline__ P minmod_lim(P R)
{
    // Minmod, include/Differ.hpp:33-43: R > 0 ? min(R, 1) : 0
    return (R > P(0)) ? ((P(1) < R) ? P(1) : R) : P(0);
}

// MUSCL_2 (limiter 0) face states from f(i-1), f(i), f(i+1), f(i+2);
// MUSCL_1 when DIFF == 0.  include/Differ.hpp:149-238
template <class P, int DIFF>
__device__ __forceinline__ void recon(P a, P b, P c, P d, P &L, P &R)
{
    if (DIFF == EU3D_DIFF_MUSCL1) {
        L = b;
        R = c;
        return;
    }
    const P kk = P(1.0) / P(3.0);
    const P eps = P(1e-12);
    P A0 = b - a, A1 = c - b, A2 = d - c;
    P Lr = A1 / (A0 + eps);
    P Rr = A1 / (A2 + eps);
    P L1 = minmod_lim(Lr), L2 = minmod_lim(P(1.0) / Lr), R1 = minmod_lim(Rr), R2 = minmod_lim(P(1.0) / Rr);
    L = b + P(0.25) * ((P(1.0) - kk) * L1 + (P(1) + kk) * L2 * Lr) * A0;
    R = c - P(0.25) * ((P(1.0) - kk) * R1 + (P(1) + kk) * R2 * Rr) * A2;
}

// AUSM face flux (src/Flowfield.cpp:1395-1500) from reconstructed states.
// ql/qr hold D U V W P H G; species are passed through yl/yr.
template <class P, int DIR>
__device__ __forceinline__ void ausm(const P ql[7], const P qr[7], const P yl[NS], const P yr[NS], P out[NV])
{
    const P DL = ql[0], UL = ql[1], VL = ql[2], WL = ql[3], PL = ql[4], HL = ql[5], GL = ql[6];
    const P DR = qr[0], UR = qr[1], VR = qr[2], WR = qr[3], PR = qr[4], HR = qr[5], GR = qr[6];
    P CL = sqrt(GL * PL / DL);
    P CR = sqrt(GR * PR / DR);
    P CI = P(0.5) * (CL + CR);
    P MaL = (DIR == 1 ? UL : DIR == 2 ? VL : WL) / CI;
    P MaR = (DIR == 1 ? UR : DIR == 2 ? VR : WR) / CI;
    P B1, G1, B2, G2;
    if (fabs(MaL) < P(1.0)) {
        P mp = MaL + P(1.0), m2 = MaL * MaL - P(1.0);
        B1 = P(0.25) * (mp * mp) + P(0.125) * (m2 * m2);
        G1 = P(0.25) * (mp * mp) * (P(2.0) - MaL) + P(3.0) / P(16.0) * MaL * (m2 * m2);
    } else {
        B1 = P(0.5) * (MaL + fabs(MaL));
        G1 = B1 / MaL;
    }
    if (fabs(MaR) < P(1.0)) {
        P mm = MaR - P(1.0), m2 = MaR * MaR - P(1.0);
        B2 = P(-0.25) * (mm * mm) - P(0.125) * (m2 * m2);
        G2 = P(0.25) * (mm * mm) * (P(2.0) + MaR) - P(3.0) / P(16.0) * MaR * (m2 * m2);
    } else {
        B2 = P(0.5) * (MaR - fabs(MaR));
        G2 = B2 / MaR;
    }
    P VI = (B1 + B2) * CI;
    const bool left = VI >= P(0.0);
    const P Ds = left ? DL : DR, Us = left ? UL : UR, Vs = left ? VL : VR, Ws = left ? WL : WR, Hs = left ? HL : HR;
#pragma unroll
    for (int s = 0; s < NS; s++) out[s] = VI * Ds * (left ? yl[s] : yr[s]);
    out[NS] = VI * Ds * Us;
    out[NS + 1] = VI * Ds * Vs;
    out[NS + 2] = VI * Ds * Ws;
    if (DIR == 1) out[NS] = VI * Ds * Us + G1 * PL + G2 * PR;
    if (DIR == 2) out[NS + 1] = VI * Ds * Vs + G1 * PL + G2 * PR;
    if (DIR == 3) out[NS + 2] = VI * Ds * Ws + G1 * PL + G2 * PR;
    out[NS + 3] = VI * (Ds * Hs + P(0.5) * Ds * (Us * Us + Vs * Vs + Ws * Ws));
}

// Face flux between cells c1 = c0 + st and c2 = c0 + 2 st, reading the four
// cells c0 .. c0 + 3 st of every primitive.  zspec: species states are zero
// (reference defect at src/Flowfield.cpp:1353).
template <class P, int DIR, int DIFF>
__device__ __forceinline__ void face_flux_g(const P *__restrict__ q, long long fs, long long c0, long long st, bool zspec,
                                            P out[NV])
{
    P ql[7], qr[7], yl[NS], yr[NS];
#pragma unroll
    for (int f = 0; f < 7; f++) {
        const P *b = q + f * fs + c0;
        recon<P, DIFF>(__ldg(b), __ldg(b + st), __ldg(b + 2 * st), __ldg(b + 3 * st), ql[f], qr[f]);
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const P *b = q + (PY + s) * fs + c0;
        recon<P, DIFF>(__ldg(b), __ldg(b + st), __ldg(b + 2 * st), __ldg(b + 3 * st), yl[s], yr[s]);
        if (zspec) {
            yl[s] = P(0);
            yr[s] = P(0);
        }
    }
    ausm<P, DIR>(ql, qr, yl, yr, out);
}

// One thread per interior cell; both faces of each direction are evaluated
// (the reference order of the residual is kept exactly).
template <class P, int DIFF>
__global__ void __launch_bounds__(128) k_advection(Layout L, const P *__restrict__ q, const double *__restrict__ xn,
                                                   const double *__restrict__ yn, const double *__restrict__ zn,
                                                   const double *__restrict__ dtp, double *__restrict__ rhs,
                                                   int species_quirk)
{
    const int i = L.bc + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = L.bc + blockIdx.y;
    const int k = L.bc + blockIdx.z;
    if (i >= L.ni + L.bc) return;
    const long long c = L.at(i, j, k);
    const long long fs = L.fs;
    const double dt = *dtp;
    const double ax = -dt / (xn[i] - xn[i - 1]);
    const double by = dt / (yn[j] - yn[j - 1]);
    const double cz = dt / (zn[k] - zn[k - 1]);
    const bool zs_cell = species_quirk && i >= L.ni;
    double r[NV];
    P fr[NV], fl[NV];
    // x: face i uses cells i-1..i+2; face i-1 uses i-2..i+1
    face_flux_g<P, 1, DIFF>(q, fs, c - 1, 1, zs_cell, fr);
    face_flux_g<P, 1, DIFF>(q, fs, c - 2, 1, species_quirk && (i - 1) >= L.ni, fl);
#pragma unroll
    for (int v = 0; v < NV; v++) r[v] = ax * ((double)fr[v] - (double)fl[v]);
    const long long sy = L.px;
    face_flux_g<P, 2, DIFF>(q, fs, c - sy, sy, zs_cell, fr);
    face_flux_g<P, 2, DIFF>(q, fs, c - 2 * sy, sy, zs_cell, fl);
#pragma unroll
    for (int v = 0; v < NV; v++) r[v] = r[v] - by * ((double)fr[v] - (double)fl[v]);
    const long long sz = (long long)L.px * L.NJ;
    face_flux_g<P, 3, DIFF>(q, fs, c - sz, sz, zs_cell, fr);
    face_flux_g<P, 3, DIFF>(q, fs, c - 2 * sz, sz, zs_cell, fl);
#pragma unroll
    for (int v = 0; v < NV; v++) rhs[v * fs + c] = r[v] - cz * ((double)fr[v] - (double)fl[v]);
}

}  // namespace eu3d
