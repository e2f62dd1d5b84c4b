// Flux sweeps: MUSCL reconstruction with the minmod limiter, AUSM splitting
// and the TimeAdv EE residual, fused into one kernel over interior cells.
//
// Reference: Flowfield::Advection (src/Flowfield.cpp:1096-1128),
// Flowfield::AUSM (:1330-1502), MUSCL_1/MUSCL_2 + Minmod
// (include/Differ.hpp:33-43, :110-238), TimeAdv::EE (src/TimeAdv.cpp:29-43).
//
// The reference materialises left/right states of 16 primitives per
// direction into full-size arrays, then face fluxes F, G, Q, then RHS.  Here
// no intermediate array exists: k_flux_tile computes each face flux once per
// step (x and y faces of a block's tile through shared memory, z faces in
// registers while the block walks its z planes) and writes only the residual
//     RHS = -dt/dx (F_i - F_{i-1}) - dt/dy (G_j - G_{j-1}) - dt/dz (Q_k - Q_{k-1})
// accumulated in FP64 in the reference's operation order.  Reconstruction
// and AUSM run in P (double or float); differences and the residual in FP64.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "tc.cuh"

namespace eu3d {

template <class P>
__device__ __forceinline__ P minmod_lim(P R)
{
    // Minmod, include/Differ.hpp:33-43: R > 0 ? min(R, 1) : 0
    return (R > P(0)) ? ((P(1) < R) ? P(1) : R) : P(0);
}

// Third-order WENO (Jiang and Shu, J. Comput. Phys. 126, 1996; new -- the
// reference's WENO enum value has no scheme behind it): the state at the face
// of cell ctr towards oth from the candidates ctr + (ctr - far)/2 and
// ctr + (oth - ctr)/2, linear weights 1/3 and 2/3, smoothness indicators the
// squared differences, epsilon 1e-6; w0 = q1 / (q1 + 2 q0), q = (eps + beta)^2.
// Every operation is rounded explicitly so that no kernel contracts it
// differently (FP64: the oracle's IEEE sequence; FP32: one sequence for all
// FP32 kernels).
__device__ __forceinline__ double weno3(double far, double ctr, double oth)
{
    const double A0 = ctr - far, A1 = oth - ctr;
    double q0 = __dadd_rn(1e-6, __dmul_rn(A0, A0)), q1 = __dadd_rn(1e-6, __dmul_rn(A1, A1));
    q0 = __dmul_rn(q0, q0);
    q1 = __dmul_rn(q1, q1);
    const double w0 = __ddiv_rn(q1, __dadd_rn(q1, __dmul_rn(2.0, q0)));
    return __dadd_rn(ctr, __dmul_rn(0.5, __dadd_rn(A1, __dmul_rn(w0, __dsub_rn(A0, A1)))));
}

__device__ __forceinline__ float weno3(float far, float ctr, float oth)
{
    const float A0 = ctr - far, A1 = oth - ctr;
    const float s0 = __fmaf_rn(A0, A0, 1e-6f), s1 = __fmaf_rn(A1, A1, 1e-6f);
    const float q0 = __fmul_rn(s0, s0), q1 = __fmul_rn(s1, s1);
    const float w0 = __fdividef(q1, __fmaf_rn(2.0f, q0, q1));
    return __fmaf_rn(0.5f, __fmaf_rn(w0, A0 - A1, A1), ctr);
}

// MUSCL_2 (limiter 0) face states, include/Differ.hpp:149-238 (MUSCL_1 when
// DIFF == 0, :110-136; WENO above when DIFF == 2): the left state of the face
// (i, i+1) from f(i-1), f(i), f(i+1), the right state from f(i), f(i+1),
// f(i+2).
template <class P, int DIFF>
__device__ __forceinline__ P recon_left(P a, P b, P c)
{
    if (DIFF == EU3D_DIFF_MUSCL1) return b;
    if (DIFF == EU3D_DIFF_WENO) return weno3(a, b, c);
    const P kk = P(1.0) / P(3.0);
    P A0 = b - a, A1 = c - b;
    P Lr = A1 / (A0 + P(1e-12));
    P L1 = minmod_lim(Lr), L2 = minmod_lim(P(1.0) / Lr);
    return b + P(0.25) * ((P(1.0) - kk) * L1 + (P(1) + kk) * L2 * Lr) * A0;
}

template <class P, int DIFF>
__device__ __forceinline__ P recon_right(P b, P c, P d)
{
    if (DIFF == EU3D_DIFF_MUSCL1) return c;
    if (DIFF == EU3D_DIFF_WENO) return weno3(d, c, b);
    const P kk = P(1.0) / P(3.0);
    P A1 = c - b, A2 = d - c;
    P Rr = A1 / (A2 + P(1e-12));
    P R1 = minmod_lim(Rr), R2 = minmod_lim(P(1.0) / Rr);
    return c - P(0.25) * ((P(1.0) - kk) * R1 + (P(1) + kk) * R2 * Rr) * A2;
}

// FP32 path: the same limited states without divisions.  With the minmod
// limiter and kappa = 1/3, the reconstruction reduces to
//     left  = f_i   + 0.5 * (L >= 1 ? A0 : L A0),  L = A1 / (A0 + 1e-12) > 0, else f_i
//     right = f_i+1 - 0.5 * (R >= 1 ? A2 : R A2),  R = A1 / (A2 + 1e-12) > 0, else f_i+1
// and L A0 = A1 A0 / (A0 + 1e-12) is taken as A1 (relative difference
// 1e-12 / |A0|, far below FP32 resolution unless the slope itself is ~1e-12).
template <>
__device__ __forceinline__ float recon_left<float, EU3D_DIFF_MUSCL2>(float a, float b, float c)
{
    const float A0 = b - a, A1 = c - b, d = A0 + 1e-12f;
    const float r = __fmaf_rn(0.5f, fabsf(A1) >= fabsf(d) ? A0 : A1, b);
    return __fmul_rn(A1, d) > 0.f ? r : b;
}

template <>
__device__ __forceinline__ float recon_right<float, EU3D_DIFF_MUSCL2>(float b, float c, float d)
{
    const float A1 = c - b, A2 = d - c, e = A2 + 1e-12f;
    const float r = __fmaf_rn(-0.5f, fabsf(A1) >= fabsf(e) ? A2 : A1, c);
    return __fmul_rn(A1, e) > 0.f ? r : c;
}

// a / b: IEEE in FP64 (parity path), the fast approximate form in FP32
__device__ __forceinline__ double pdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float pdiv(float a, float b) { return __fdividef(a, b); }

// the hardware's approximate reciprocal square root and reciprocal (PTX
// rsqrt.approx / rcp.approx, subnormals flushed: the FP32 flux never meets
// them in a sound speed)
__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Upwind-side MUSCL_2 state in one formula for both sides, FP32.  For the
// left state pass (far, ctr, oth) = f(a-1), f(a), f(a+1) and seps = +1e-12;
// for the right state f(a+2), f(a+1), f(a) and seps = -1e-12.  Negating both
// differences and the epsilon turns recon_right's arithmetic into
// recon_left's with every rounding mirrored, so the result equals
// recon_left / recon_right bit for bit and no branch picks the side.
__device__ __forceinline__ float up_muscl2(float far, float ctr, float oth, float seps)
{
    const float A0 = ctr - far, A1 = oth - ctr, d = A0 + seps;
    const float h = fabsf(A1) >= fabsf(d) ? A0 : A1;
    return (__fmul_rn(A1, d) > 0.f) ? __fmaf_rn(0.5f, h, ctr) : ctr;
}

// AUSM face flux from the four cells a-1 .. a+2 around the face (a, a+1).
// Only the states AUSM reads are reconstructed: both sides of P, D, gamma
// and the normal velocity (they set the interface Mach number), then only
// the upwind side of the tangential velocities, H and the species.  The
// source gives field f of cell a-1+n as v(f, n) and the upwind triple of a
// field as up3(f, left, far, ctr, oth) (cells a-1, a, a+1 when left, else
// a+2, a+1, a); both are plain loads, from global or shared memory.
// src/Flowfield.cpp:1395-1500 (AUSM), include/Differ.hpp:149-238 (MUSCL_2).
template <int DIR, int DIFF, class Src>
__device__ __forceinline__ void face_flux_src(const Src &src, bool zspec, float out[NV])
{
    // Every sum of products is written out with explicit rounding
    // (__fmaf_rn / __fmul_rn), so that the compiler cannot contract it
    // differently in different kernels: all FP32 flux kernels give the same
    // bits for the same face.
    auto both = [&](int f, float &L, float &R) {
        const float v0 = src.v(f, 0), v1 = src.v(f, 1), v2 = src.v(f, 2), v3 = src.v(f, 3);
        L = recon_left<float, DIFF>(v0, v1, v2);
        R = recon_right<float, DIFF>(v1, v2, v3);
    };
    constexpr int FN = DIR == 1 ? PU : DIR == 2 ? PV : PW;
    float DL, DR, PL, PR, GL, GR, NL, NR;
    both(PD, DL, DR);
    both(PP, PL, PR);
    both(PG, GL, GR);
    both(FN, NL, NR);
    // sound speeds sqrt(g p / D) = x rsqrt(x D) with x = g p: one approximate
    // reciprocal square root (relative error below 2^-22) in place of a
    // division and a correctly rounded square root with its special-case
    // path; one reciprocal of CI serves both Mach numbers
    const float xL = __fmul_rn(GL, PL), xR = __fmul_rn(GR, PR);
    const float CL = __fmul_rn(xL, rsqrt_approx(__fmul_rn(xL, DL)));
    const float CR = __fmul_rn(xR, rsqrt_approx(__fmul_rn(xR, DR)));
    const float CI = __fmul_rn(0.5f, CL + CR);
    const float rCI = rcp_approx(CI);
    const float MaL = __fmul_rn(NL, rCI), MaR = __fmul_rn(NR, rCI);
    // both branches of the split Mach numbers are evaluated and one is
    // selected (the unused one may divide by ~0; its result is dropped)
    float B1, G1, B2, G2;
    {
        const float mp = MaL + 1.0f, m2 = __fmaf_rn(MaL, MaL, -1.0f);
        const float mp2 = __fmul_rn(mp, mp), m22 = __fmul_rn(m2, m2);
        const float b_sub = __fmaf_rn(0.125f, m22, __fmul_rn(0.25f, mp2));
        const float g_sub = __fmaf_rn(__fmul_rn(0.1875f, MaL), m22, __fmul_rn(__fmul_rn(0.25f, mp2), 2.0f - MaL));
        const float b_sup = __fmul_rn(0.5f, MaL + fabsf(MaL));
        const bool sub = fabsf(MaL) < 1.0f;
        B1 = sub ? b_sub : b_sup;
        G1 = sub ? g_sub : __fdividef(b_sup, MaL);
    }
    {
        const float mm = MaR - 1.0f, m2 = __fmaf_rn(MaR, MaR, -1.0f);
        const float mm2 = __fmul_rn(mm, mm), m22 = __fmul_rn(m2, m2);
        const float b_sub = __fmaf_rn(-0.125f, m22, __fmul_rn(-0.25f, mm2));
        const float g_sub = __fmaf_rn(__fmul_rn(-0.1875f, MaR), m22, __fmul_rn(__fmul_rn(0.25f, mm2), 2.0f + MaR));
        const float b_sup = __fmul_rn(0.5f, MaR - fabsf(MaR));
        const bool sub = fabsf(MaR) < 1.0f;
        B2 = sub ? b_sub : b_sup;
        G2 = sub ? g_sub : __fdividef(b_sup, MaR);
    }
    const float VI = __fmul_rn(B1 + B2, CI);
    const bool left = VI >= 0.0f;
    const float seps = left ? 1e-12f : -1e-12f;
    auto up = [&](int f) -> float {
        float far, ctr, oth;
        src.up3(f, left, far, ctr, oth);
        if (DIFF == EU3D_DIFF_MUSCL1) return ctr;
        if (DIFF == EU3D_DIFF_WENO) return weno3(far, ctr, oth);
        return up_muscl2(far, ctr, oth, seps);
    };
    const float Ds = left ? DL : DR;
    const float Us = DIR == 1 ? (left ? NL : NR) : up(PU);
    const float Vs = DIR == 2 ? (left ? NL : NR) : up(PV);
    const float Ws = DIR == 3 ? (left ? NL : NR) : up(PW);
    const float Hs = up(PH);
    const float VD = __fmul_rn(VI, Ds);
#pragma unroll
    for (int s = 0; s < NS; s++) out[s] = zspec ? __fmul_rn(0.0f, VD) : __fmul_rn(VD, up(PY + s));
    // normal momentum: VD u_n + G1 PL + G2 PR
    const float pn = __fmaf_rn(G2, PR, __fmul_rn(G1, PL));
    out[NS] = DIR == 1 ? __fmaf_rn(VD, Us, pn) : __fmul_rn(VD, Us);
    out[NS + 1] = DIR == 2 ? __fmaf_rn(VD, Vs, pn) : __fmul_rn(VD, Vs);
    out[NS + 2] = DIR == 3 ? __fmaf_rn(VD, Ws, pn) : __fmul_rn(VD, Ws);
    // energy: VI (D H + D/2 |u|^2)
    const float q2 = __fmaf_rn(Ws, Ws, __fmaf_rn(Vs, Vs, __fmul_rn(Us, Us)));
    out[NS + 3] = __fmul_rn(VI, __fmaf_rn(__fmul_rn(0.5f, Ds), q2, __fmul_rn(Ds, Hs)));
}

// TimeAdv::EE's residual of one conserved variable (src/TimeAdv.cpp:29-43:
// RHS = -dt (dF/dx + dG/dy + dQ/dz)) from the face fluxes of the cell, with
// ax = -dt/dx, by = dt/dy, cz = dt/dz.  FP64 fluxes: FP64 in the
// reference's order.  FP32 fluxes: the three differences and the sum in
// FP32, each operation rounded explicitly so that every FP32 kernel forms
// the same bits, stored in FP32 -- its rounding (2^-24 of the residual) is
// below the error the FP32 fluxes carry already.
__device__ __forceinline__ double residual(double ax, double by, double cz, double xr, double xl, double yt, double yb,
                                           double za, double zb)
{
    const double r = ax * (xr - xl);
    return (r - by * (yt - yb)) - cz * (za - zb);
}

__device__ __forceinline__ float residual(float ax, float by, float cz, float xr, float xl, float yt, float yb,
                                          float za, float zb)
{
    const float r = __fmaf_rn(-by, __fsub_rn(yt, yb), __fmul_rn(ax, __fsub_rn(xr, xl)));
    return __fmaf_rn(-cz, __fsub_rn(za, zb), r);
}

// Cells a-1 .. a+2 at element step st from qc (cell a-1 of field 0), fields
// fs elements apart; global memory through the read-only path (LDG) or
// shared memory.
template <bool LDG>
struct StridedSrc {
    const float *qc;
    int fs, st;
    __device__ __forceinline__ float ld(const float *p) const { return LDG ? __ldg(p) : *p; }
    __device__ __forceinline__ float v(int f, int n) const { return ld(qc + f * fs + n * st); }
    __device__ __forceinline__ void up3(int f, bool left, float &far, float &ctr, float &oth) const
    {
        const float *p = left ? qc : qc + 3 * st;
        const int s = left ? st : -st;
        far = ld(p + f * fs);
        ctr = ld(p + f * fs + s);
        oth = ld(p + f * fs + 2 * s);
    }
};

// Face flux between cells a and a+1 (cells a-1 .. a+2 along the direction,
// element stride st, qc the index of cell a-1 of field 0).  FP64: the
// reference's reconstruction with divisions; FP32: face_flux_src.
template <class P, int DIR, int DIFF, bool LDG = true>
__device__ __forceinline__ void face_flux_up(const P *__restrict__ qc, int fs, int st, bool zspec, P out[NV])
{
    if constexpr (sizeof(P) == 4) {
        face_flux_src<DIR, DIFF>(StridedSrc<LDG>{qc, fs, st}, zspec, out);
        return;
    } else {
    // qc points at cell a-1 of field 0; field f of cell a-1+n is qc[f * fs + n * st]
    auto ld = [&](int f, int n) -> P { return LDG ? __ldg(qc + f * fs + n * st) : qc[f * fs + n * st]; };
    auto both = [&](int f, P &L, P &R) {
        const P v0 = ld(f, 0), v1 = ld(f, 1), v2 = ld(f, 2), v3 = ld(f, 3);
        L = recon_left<P, DIFF>(v0, v1, v2);
        R = recon_right<P, DIFF>(v1, v2, v3);
    };
    constexpr int FN = DIR == 1 ? PU : DIR == 2 ? PV : PW;
    P DL, DR, PL, PR, GL, GR, NL, NR;
    both(PD, DL, DR);
    both(PP, PL, PR);
    both(PG, GL, GR);
    both(FN, NL, NR);
    const P CL = sqrt(pdiv(GL * PL, DL));
    const P CR = sqrt(pdiv(GR * PR, DR));
    const P CI = P(0.5) * (CL + CR);
    const P MaL = pdiv(NL, CI), MaR = pdiv(NR, CI);
    P B1, G1, B2, G2;
    if (fabs(MaL) < P(1.0)) {
        P mp = MaL + P(1.0), m2 = MaL * MaL - P(1.0);
        B1 = P(0.25) * (mp * mp) + P(0.125) * (m2 * m2);
        G1 = P(0.25) * (mp * mp) * (P(2.0) - MaL) + P(3.0) / P(16.0) * MaL * (m2 * m2);
    } else {
        B1 = P(0.5) * (MaL + fabs(MaL));
        G1 = pdiv(B1, MaL);
    }
    if (fabs(MaR) < P(1.0)) {
        P mm = MaR - P(1.0), m2 = MaR * MaR - P(1.0);
        B2 = P(-0.25) * (mm * mm) - P(0.125) * (m2 * m2);
        G2 = P(0.25) * (mm * mm) * (P(2.0) + MaR) - P(3.0) / P(16.0) * MaR * (m2 * m2);
    } else {
        B2 = P(0.5) * (MaR - fabs(MaR));
        G2 = pdiv(B2, MaR);
    }
    const P VI = (B1 + B2) * CI;
    const bool left = VI >= P(0.0);
    // upwind-side reconstruction of one field
    auto up = [&](int f) -> P {
        return left ? recon_left<P, DIFF>(ld(f, 0), ld(f, 1), ld(f, 2)) : recon_right<P, DIFF>(ld(f, 1), ld(f, 2), ld(f, 3));
    };
    const P Ds = left ? DL : DR;
    const P Us = DIR == 1 ? (left ? NL : NR) : up(PU);
    const P Vs = DIR == 2 ? (left ? NL : NR) : up(PV);
    const P Ws = DIR == 3 ? (left ? NL : NR) : up(PW);
    const P Hs = up(PH);
    const P VD = VI * Ds;
#pragma unroll
    for (int s = 0; s < NS; s++) out[s] = zspec ? P(0) * VD : VD * up(PY + s);
    out[NS] = VD * Us;
    out[NS + 1] = VD * Vs;
    out[NS + 2] = VD * Ws;
    if (DIR == 1) out[NS] = VD * Us + G1 * PL + G2 * PR;
    if (DIR == 2) out[NS + 1] = VD * Vs + G1 * PL + G2 * PR;
    if (DIR == 3) out[NS + 2] = VD * Ws + G1 * PL + G2 * PR;
    out[NS + 3] = VI * (Ds * Hs + P(0.5) * Ds * (Us * Us + Vs * Vs + Ws * Ws));
    }
}

// Wedge immersed boundary as the flux kernels see it: a tile none of whose
// cells is fluid forms no residual (nothing reads the residual of a solid
// cell: the stage updates, the chemistry and the surrogate skip them).
struct FluxSolid {
    double x0, y0, tn;
    int on;
    __device__ __forceinline__ bool solid(double x, double y) const
    {
        return on && x > x0 && (y - y0) < (x - x0) * tn;
    }
};

constexpr int FT_X = 32;
// tile height: 8 rows for FP32 primitives, 4 for FP64; face fluxes live in
// dynamic shared memory (two buffers of x and y faces)
template <class P>
struct FluxTile {
    static constexpr int TY = sizeof(P) == 8 ? 4 : 8;
    static constexpr int FX = TY * (FT_X + 1) * NV;  // elements of one x-face buffer
    static constexpr int FY = (TY + 1) * FT_X * NV;  // elements of one y-face buffer
    static constexpr size_t SMEM = sizeof(P) * 2 * (FX + FY);
};

// Tiled flux + residual kernel.  A block owns a 32 x TY tile of x-y columns
// and walks `kz` z planes.  At each plane every x face and y face of the tile
// is computed once (by one thread) into shared memory, every z face once in
// registers (the face below a cell is the face above the previous plane's
// cell), and each thread then forms its cell's residual in the reference's
// order ((-dt/dx dF - dt/dy dG) - dt/dz dQ) in FP64.
// A tile of 32 x TY cells has 33 x TY x faces and 32 x (TY + 1) y faces: the
// block carries two extra warps, one for the last y-face row (ty == TY) and
// one for the last x face of each row (ty == TY + 1), so that every warp
// evaluates at most one face of each direction per plane.
template <class P>
constexpr int flux_threads()
{
    return FT_X * (FluxTile<P>::TY + 2);
}

template <class P, int DIFF>
__global__ void __launch_bounds__(flux_threads<P>(), 2) k_flux_tile(
    Layout L, const P *__restrict__ q, const double *__restrict__ xn, const double *__restrict__ yn,
    const double *__restrict__ zn, const double *__restrict__ dtp, P *__restrict__ rhs, int species_quirk, int kz,
    FluxSolid wedge)
{
    constexpr int TY = FluxTile<P>::TY;
    // two buffers: plane k+1 may fill one while slow threads still read plane k
    extern __shared__ __align__(16) unsigned char flux_smem[];
    auto fx = reinterpret_cast<P(*)[TY][FT_X + 1][NV]>(flux_smem);
    auto fy = reinterpret_cast<P(*)[TY + 1][FT_X][NV]>(flux_smem + sizeof(P) * 2 * FluxTile<P>::FX);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = L.bc + blockIdx.x * FT_X, j0 = L.bc + blockIdx.y * TY;
    const int kb = L.bc + blockIdx.z * kz;
    const int ke = min(kb + kz, L.nk + L.bc);
    const int i = i0 + tx, j = j0 + ty;
    const int ilast = L.ni + L.bc - 1, jlast = L.nj + L.bc - 1;
    const bool cellw = ty < TY;  // warps that own cells (the other two only add faces)
    const bool act = cellw && i <= ilast && j <= jlast;
    if (!__syncthreads_or(act && !wedge.solid(xn[i], yn[j]))) return;  // an all-solid tile
    const int fs = (int)L.fs, sy = L.px, sz = L.px * L.NJ;
    const double dt = *dtp;
    const bool zs_cell = species_quirk && i >= L.ni;
    P qb[NV], qa[NV];
    const P ax = (P)(act ? -dt / (xn[i] - xn[i - 1]) : 0.0);
    const P by = (P)(act ? dt / (yn[j] - yn[j - 1]) : 0.0);
    if (act) face_flux_up<P, 3, DIFF>(q + L.at(i, j, kb) - 2 * (long long)sz, fs, sz, zs_cell, qb);
    for (int k = kb, it = 0; k < ke; k++, it ^= 1) {
        // x faces of row r: face f sits between a = i0+f-1 and a+1 and is
        // needed when a <= ilast; it reads cells a-1 .. a+2.  Faces 0..31 by
        // the cell warps, face 32 of row tx by lane tx of warp TY + 1.
        {
            const int r = cellw ? ty : tx;
            const int f = cellw ? tx : FT_X;
            const int jr = j0 + r;
            const int a = i0 + f - 1;
            if ((cellw || (ty == TY + 1 && tx < TY)) && jr <= jlast && a <= ilast)
                face_flux_up<P, 1, DIFF>(q + L.at(a - 1, jr, k), fs, 1, species_quirk && a >= L.ni, fx[it][r][f]);
        }
        // y faces of column i: face g sits between b = j0+g-1 and b+1;
        // faces 0..TY-1 by the cell warps, face TY by warp TY
        if (ty <= TY && i <= ilast) {
            const int b = j0 + ty - 1;
            if (b <= jlast) face_flux_up<P, 2, DIFF>(q + L.at(i, b - 1, k), fs, sy, species_quirk && i >= L.ni, fy[it][ty][tx]);
        }
        if (act) face_flux_up<P, 3, DIFF>(q + L.at(i, j, k) - sz, fs, sz, zs_cell, qa);
        __syncthreads();
        if (act) {
            const P cz = (P)(dt / (zn[k] - zn[k - 1]));
            const long long c = L.at(i, j, k);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                rhs[v * L.fs + c] = residual(ax, by, cz, fx[it][ty][tx + 1][v], fx[it][ty][tx][v], fy[it][ty + 1][tx][v],
                                             fy[it][ty][tx][v], qa[v], qb[v]);
                qb[v] = qa[v];
            }
        }
    }
}

// FP32 flux kernel with the primitives staged through shared memory.  Same
// tile, thread roles and residual order as k_flux_tile, but at each z plane
// the block first copies the plane's 36 x (TY + 4) cells (the tile and a
// two-cell halo) of all 16 primitives into shared memory with coalesced
// loads, then evaluates the x and y faces from there; z faces read their
// column from global memory as before.
constexpr int FS_TY = 8, FS_HX = FT_X + 4, FS_HY = FS_TY + 4;
struct FluxStage {
    static constexpr int PLANE = NPRIM * FS_HY * FS_HX;  // floats of one staged plane
    static constexpr int FX = FS_TY * (FT_X + 1) * NV;
    static constexpr int FY = (FS_TY + 1) * FT_X * NV;
    static constexpr size_t SMEM = sizeof(float) * (PLANE + FX + FY);
};

template <int DIFF>
__global__ void __launch_bounds__(FT_X *(FS_TY + 2), 2) k_flux_stage(
    Layout L, const float *__restrict__ q, const double *__restrict__ xn, const double *__restrict__ yn,
    const double *__restrict__ zn, const double *__restrict__ dtp, float *__restrict__ rhs, int species_quirk, int kz,
    FluxSolid wedge)
{
    constexpr int TY = FS_TY, HX = FS_HX, HY = FS_HY, PL = HX * HY;
    extern __shared__ __align__(16) unsigned char flux_smem[];
    float *S = reinterpret_cast<float *>(flux_smem);
    auto fx = reinterpret_cast<float(*)[FT_X + 1][NV]>(S + FluxStage::PLANE);
    auto fy = reinterpret_cast<float(*)[FT_X][NV]>(S + FluxStage::PLANE + FluxStage::FX);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * FT_X + tx, nthr = FT_X * (TY + 2);
    const int i0 = L.bc + blockIdx.x * FT_X, j0 = L.bc + blockIdx.y * TY;
    const int kb = L.bc + blockIdx.z * kz;
    const int ke = min(kb + kz, L.nk + L.bc);
    const int i = i0 + tx, j = j0 + ty;
    const int ilast = L.ni + L.bc - 1, jlast = L.nj + L.bc - 1;
    const bool cellw = ty < TY;
    const bool act = cellw && i <= ilast && j <= jlast;
    if (!__syncthreads_or(act && !wedge.solid(xn[i], yn[j]))) return;  // an all-solid tile
    const int fs = (int)L.fs, sz = L.px * L.NJ;
    const double dt = *dtp;
    const bool zs_cell = species_quirk && i >= L.ni;
    float qb[NV], qa[NV];
    const float ax = (float)(act ? -dt / (xn[i] - xn[i - 1]) : 0.0);
    const float by = (float)(act ? dt / (yn[j] - yn[j - 1]) : 0.0);
    if (act) face_flux_up<float, 3, DIFF>(q + L.at(i, j, kb) - 2 * (long long)sz, fs, sz, zs_cell, qb);
    for (int k = kb; k < ke; k++) {
        // stage cells x in [i0 - 2, i0 + 34), y in [j0 - 2, j0 + TY + 2) of plane k
        // (indices past the array, never needed by a face, are clamped)
        for (int e = tid; e < FluxStage::PLANE; e += nthr) {
            const int f = e / PL, r = e - f * PL;
            const int yy = r / HX, xx = r - yy * HX;
            const int gi = min(i0 - 2 + xx, L.NI - 1), gj = min(j0 - 2 + yy, L.NJ - 1);
            S[e] = __ldg(q + (long long)f * fs + L.at(gi, gj, k));
        }
        __syncthreads();
        // x face f of row r: between a = i0+f-1 and a+1, cells a-1 .. a+2 at
        // staged columns f .. f+3 of staged row r+2
        {
            const int r = cellw ? ty : tx;
            const int f = cellw ? tx : FT_X;
            const int jr = j0 + r;
            const int a = i0 + f - 1;
            if ((cellw || (ty == TY + 1 && tx < TY)) && jr <= jlast && a <= ilast)
                face_flux_up<float, 1, DIFF, false>(S + (r + 2) * HX + f, PL, 1, species_quirk && a >= L.ni, fx[r][f]);
        }
        // y face g of column i: between b = j0+g-1 and b+1, staged rows g .. g+3
        if (ty <= TY && i <= ilast) {
            const int b = j0 + ty - 1;
            if (b <= jlast)
                face_flux_up<float, 2, DIFF, false>(S + ty * HX + tx + 2, PL, HX, species_quirk && i >= L.ni, fy[ty][tx]);
        }
        if (act) face_flux_up<float, 3, DIFF>(q + L.at(i, j, k) - sz, fs, sz, zs_cell, qa);
        __syncthreads();
        if (act) {
            const float cz = (float)(dt / (zn[k] - zn[k - 1]));
            const long long c = L.at(i, j, k);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                rhs[v * L.fs + c] = residual(ax, by, cz, fx[ty][tx + 1][v], fx[ty][tx][v], fy[ty + 1][tx][v],
                                             fy[ty][tx][v], qa[v], qb[v]);
                qb[v] = qa[v];
            }
        }
    }
}

// FP32 flux kernel fed by TMA (k_flux_ring).  Same tile (32 x 8 cells plus
// two face warps), face ownership and residual order as k_flux_stage.
// Differences:
//  * each z plane of the tile with its two-cell halo (36 x 12 cells x 16
//    primitives, 27 KB) arrives by one TMA box load into a ring of three
//    shared-memory buffers: while plane c is processed, planes c and c+1 are
//    resident and c+2 is resident or in flight (it is waited for only after
//    the x and y faces, which need plane c alone), so no thread computes
//    load addresses;
//  * each cell thread keeps its own cell of plane c-1 in a private
//    shared-memory slot, so the z face above the cell reads its four cells
//    c-1 .. c+2 from shared memory;
//  * a cell's right x face is its right neighbour's left face, passed by a
//    warp shuffle (row ends through shared memory from the face warp);
//  * faces are evaluated by face_flux_pk: the left/right pairs of the AUSM
//    arithmetic, two upwind fields at a time, the species fluxes and the
//    residual in packed FP32 pairs, the upwind side picked by pointer
//    selection, not branches -- bit for bit face_flux_src's result;
//  * the cell warps evaluate their three faces with no per-lane condition
//    (lanes past a ragged tile edge compute on staged values and store
//    nothing), so the faces share one basic block;
//  * dt/dz of the next plane is formed by one thread of the y-face warp
//    while the others work (two-entry buffer); the species-face quirk is a
//    template switch (SQ), so the default build carries no test for it.
// Every wait on the ring is bounded: when one runs out the block counts a
// timeout in the status, waits (bounded) for its copies in flight and stops.
constexpr int FR_TY = 8, FR_HX = FT_X + 4, FR_HY = FR_TY + 4, FR_PL = FR_HX * FR_HY, FR_NBUF = 3;
constexpr int FR_CS = FT_X * FR_TY;  // field stride of the plane c-1 slots

// Packed FP32 pairs: Blackwell's two-lane add, multiply and fused
// multiply-add (CUDA's __fadd2_rn / __fmul2_rn / __ffma2_rn).  Each lane is
// rounded once, to nearest, exactly as the scalar __fadd_rn / __fmul_rn /
// __fmaf_rn of the same operands; a - b is fma(b, -1, a), the exact a - b
// rounded once, as the scalar subtraction.
__device__ __forceinline__ float2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// up_muscl2 of two fields on the same side at once: lane by lane the scalar
// up_muscl2 (differences, epsilon, product and the final fma in pairs; the
// comparisons and selections per lane)
__device__ __forceinline__ float2 up_muscl2_x2(float2 far, float2 ctr, float2 oth, float2 seps)
{
    const float2 A0 = sub2(ctr, far), A1 = sub2(oth, ctr);
    const float2 d = add2(A0, seps);
    const float2 pr = mul2(A1, d);
    const float2 h = pk(fabsf(A1.x) >= fabsf(d.x) ? A0.x : A1.x, fabsf(A1.y) >= fabsf(d.y) ? A0.y : A1.y);
    const float2 r = fma2(pk(0.5f, 0.5f), h, ctr);
    return pk(pr.x > 0.f ? r.x : ctr.x, pr.y > 0.f ? r.y : ctr.y);
}

// The upwind triple of a face (cells far, ctr, oth of field 0), chosen once
// per face; the fields follow at FR_PL floats (the staged planes' stride).
struct UpBase {
    const float *f, *c, *o;
};

// x or y face inside one staged plane: cells a-1 .. a+2, ST floats apart
// from qc (cell a-1, field 0)
template <int ST>
struct PlaneSrc {
    const float *qc;
    __device__ __forceinline__ float v(int f, int n) const { return qc[f * FR_PL + n * ST]; }
    __device__ __forceinline__ UpBase side(bool left) const
    {
        return left ? UpBase{qc, qc + ST, qc + 2 * ST} : UpBase{qc + 3 * ST, qc + 2 * ST, qc + ST};
    }
    __device__ __forceinline__ float far(const UpBase &b, bool, int f) const { return b.f[f * FR_PL]; }
};

// z face between planes c and c+1 of one column: cell c-1 from the thread's
// slot (fields FR_CS floats apart), c, c+1, c+2 from the ring.  The far cell
// of the upwind triple is the slot's (left) or plane c+2's (right): the two
// strides differ, so both are read and one is selected.
struct ZColSrc {
    const float *cm;            // the cell of plane c-1, field 0
    const float *sc, *sn, *sp;  // the cell in the staged planes c, c+1, c+2, field 0
    __device__ __forceinline__ float v(int f, int n) const
    {
        return n == 0 ? cm[f * FR_CS] : n == 1 ? sc[f * FR_PL] : n == 2 ? sn[f * FR_PL] : sp[f * FR_PL];
    }
    __device__ __forceinline__ UpBase side(bool left) const
    {
        return left ? UpBase{nullptr, sc, sn} : UpBase{nullptr, sn, sc};
    }
    __device__ __forceinline__ float far(const UpBase &, bool left, int f) const
    {
        const float a = cm[f * FR_CS], b = sp[f * FR_PL];
        return left ? a : b;
    }
};

// AUSM face flux of the ring kernel: face_flux_src's arithmetic with the
// left/right pairs of the sound speeds and split Mach numbers, the upwind
// reconstruction of two fields at a time and the species fluxes in packed
// pairs; the result equals face_flux_src's bit for bit.
template <int DIR, int DIFF, class Src>
__device__ __forceinline__ void face_flux_pk(const Src &src, bool zspec, float out[NV])
{
    auto both = [&](int f, float &L, float &R) {
        const float v0 = src.v(f, 0), v1 = src.v(f, 1), v2 = src.v(f, 2), v3 = src.v(f, 3);
        L = recon_left<float, DIFF>(v0, v1, v2);
        R = recon_right<float, DIFF>(v1, v2, v3);
    };
    constexpr int FN = DIR == 1 ? PU : DIR == 2 ? PV : PW;
    float DL, DR, PL, PR, GL, GR, NL, NR;
    both(PD, DL, DR);
    both(PP, PL, PR);
    both(PG, GL, GR);
    both(FN, NL, NR);
    // sound speeds x rsqrt(x D), x = g p: left and right in one pair
    const float2 X = mul2(pk(GL, GR), pk(PL, PR));
    const float2 Y = mul2(X, pk(DL, DR));
    const float2 C = mul2(X, pk(rsqrt_approx(Y.x), rsqrt_approx(Y.y)));
    const float CI = __fmul_rn(0.5f, C.x + C.y);
    const float rCI = rcp_approx(CI);
    const float2 M = mul2(pk(NL, NR), pk(rCI, rCI));  // (MaL, MaR)
    // split Mach numbers: lane x the "+" split of MaL, lane y the "-" split
    // of MaR, each in face_flux_src's operation order
    const float2 MP = add2(M, pk(1.0f, -1.0f));  // MaL + 1, MaR - 1
    const float2 M2 = fma2(M, M, pk(-1.0f, -1.0f));
    const float2 MP2 = mul2(MP, MP), M22 = mul2(M2, M2);
    const float2 BSUB = fma2(pk(0.125f, -0.125f), M22, mul2(pk(0.25f, -0.25f), MP2));
    const float2 TWO = fma2(M, pk(-1.0f, 1.0f), pk(2.0f, 2.0f));  // 2 - MaL, 2 + MaR
    const float2 GSUB = fma2(mul2(pk(0.1875f, -0.1875f), M), M22, mul2(mul2(pk(0.25f, 0.25f), MP2), TWO));
    const float2 BSUP = mul2(pk(0.5f, 0.5f), pk(M.x + fabsf(M.x), M.y - fabsf(M.y)));
    const bool subL = fabsf(M.x) < 1.0f, subR = fabsf(M.y) < 1.0f;
    const float B1 = subL ? BSUB.x : BSUP.x, G1 = subL ? GSUB.x : __fdividef(BSUP.x, M.x);
    const float B2 = subR ? BSUB.y : BSUP.y, G2 = subR ? GSUB.y : __fdividef(BSUP.y, M.y);
    const float VI = __fmul_rn(B1 + B2, CI);
    const bool left = VI >= 0.0f;
    const float seps = left ? 1e-12f : -1e-12f;
    const UpBase ub = src.side(left);
    auto up2 = [&](int f, int g) -> float2 {
        const float2 far = pk(src.far(ub, left, f), src.far(ub, left, g));
        const float2 ctr = pk(ub.c[f * FR_PL], ub.c[g * FR_PL]);
        const float2 oth = pk(ub.o[f * FR_PL], ub.o[g * FR_PL]);
        if (DIFF == EU3D_DIFF_MUSCL1) return ctr;
        if (DIFF == EU3D_DIFF_WENO) return pk(weno3(far.x, ctr.x, oth.x), weno3(far.y, ctr.y, oth.y));
        return up_muscl2_x2(far, ctr, oth, pk(seps, seps));
    };
    constexpr int T1 = DIR == 1 ? PV : PU, T2 = DIR == 3 ? PV : PW;  // the tangential velocities
    const float2 TT = up2(T1, T2);
    const float2 HY = up2(PH, PY);
    const float Ds = left ? DL : DR, Ns = left ? NL : NR;
    const float Us = DIR == 1 ? Ns : TT.x;
    const float Vs = DIR == 2 ? Ns : DIR == 1 ? TT.x : TT.y;
    const float Ws = DIR == 3 ? Ns : TT.y;
    const float VD = __fmul_rn(VI, Ds);
    const float zf = __fmul_rn(0.0f, VD);
    out[0] = zspec ? zf : __fmul_rn(VD, HY.y);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float2 o = mul2(pk(VD, VD), up2(PY + 1 + 2 * q, PY + 2 + 2 * q));
        out[1 + 2 * q] = zspec ? zf : o.x;
        out[2 + 2 * q] = zspec ? zf : o.y;
    }
    const float pn = __fmaf_rn(G2, PR, __fmul_rn(G1, PL));
    out[NS] = DIR == 1 ? __fmaf_rn(VD, Us, pn) : __fmul_rn(VD, Us);
    out[NS + 1] = DIR == 2 ? __fmaf_rn(VD, Vs, pn) : __fmul_rn(VD, Vs);
    out[NS + 2] = DIR == 3 ? __fmaf_rn(VD, Ws, pn) : __fmul_rn(VD, Ws);
    const float q2 = __fmaf_rn(Ws, Ws, __fmaf_rn(Vs, Vs, __fmul_rn(Us, Us)));
    out[NS + 3] = __fmul_rn(VI, __fmaf_rn(__fmul_rn(0.5f, Ds), q2, __fmul_rn(Ds, HY.x)));
}

// residual() of two conserved variables at once (the same roundings per lane)
__device__ __forceinline__ float2 residual2(float2 ax, float2 nby, float2 ncz, float2 xr, float2 xl, float2 yt,
                                            float2 yb, float2 za, float2 zb)
{
    const float2 r = fma2(nby, sub2(yt, yb), mul2(ax, sub2(xr, xl)));
    return fma2(ncz, sub2(za, zb), r);
}

struct FluxRing {
    static constexpr int PLANE = NPRIM * FR_PL;         // floats of one staged plane
    static constexpr uint32_t PLANE_BYTES = PLANE * 4;  // bytes of one TMA box (27648)
    static constexpr int FY = (FR_TY + 1) * FT_X * NV;  // y-face fluxes
    static constexpr int FXE = FR_TY * NV;              // the last x face of each row
    static constexpr int CORE = NPRIM * FR_CS;          // each cell thread's cell of plane c-1
    static constexpr int CZ = 2;                        // dt/dz of the current and the next plane
    static constexpr size_t BYTES = FR_NBUF * PLANE_BYTES + 4 * (FY + FXE + CORE + CZ) + 8 * FR_NBUF;
    // slack to align the ring to 128 B; two blocks (with the 1 KB the
    // hardware reserves for each) fit the SM's 228 KB
    static constexpr size_t SMEM = BYTES + 128;
    // TMA box {x, y, z, field}
    static constexpr unsigned BOX[4] = {FR_HX, FR_HY, 1, NPRIM};
};
static_assert(2 * (FluxRing::SMEM + 1024) <= 228 * 1024, "two ring blocks must fit one SM");

template <int DIFF, bool SQ>
__global__ void __launch_bounds__(FT_X *(FR_TY + 2), 2) k_flux_ring(
    const __grid_constant__ CUtensorMap tq, Layout L, const float *__restrict__ q, const double *__restrict__ xn,
    const double *__restrict__ yn, const double *__restrict__ zn, const double *__restrict__ dtp,
    float *__restrict__ rhs, int kz, Status *__restrict__ stat, FluxSolid wedge, unsigned wait_tries)
{
    constexpr int TY = FR_TY, HX = FR_HX, PL = FR_PL;
    extern __shared__ unsigned char fr_raw[];
    const uint32_t raw_s = tc::smem_u32(fr_raw);
    float *ring = reinterpret_cast<float *>(fr_raw + (((raw_s + 127u) & ~127u) - raw_s));
    auto fy = reinterpret_cast<float(*)[FT_X][NV]>(ring + FR_NBUF * FluxRing::PLANE);
    auto fxe = reinterpret_cast<float(*)[NV]>(ring + FR_NBUF * FluxRing::PLANE + FluxRing::FY);
    float *core = ring + FR_NBUF * FluxRing::PLANE + FluxRing::FY + FluxRing::FXE;
    float *czb = core + FluxRing::CORE;
    const uint32_t ring_s = tc::smem_u32(ring);
    const uint32_t mb_s =
        ring_s + 4u * (FR_NBUF * FluxRing::PLANE + FluxRing::FY + FluxRing::FXE + FluxRing::CORE + FluxRing::CZ);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * FT_X + tx;
    const int i0 = L.bc + blockIdx.x * FT_X, j0 = L.bc + blockIdx.y * TY;
    const int kb = L.bc + blockIdx.z * kz;
    const int np = min(kz, L.nk + L.bc - kb);  // planes whose residual this block forms
    const int i = i0 + tx, j = j0 + ty;
    const int ilast = L.ni + L.bc - 1, jlast = L.nj + L.bc - 1;
    const bool cellw = ty < TY;
    const bool act = cellw && i <= ilast && j <= jlast;
    // an all-solid tile leaves before its barriers and copies exist
    if (!__syncthreads_or(act && !wedge.solid(xn[i], yn[j]))) return;
    const int fs = (int)L.fs, sz = L.px * L.NJ;
    // plane kb + p into buffer p % 3; the block loads planes kb .. kb + np + 1
    // (the last two only feed the top z face; kb + np + 1 <= nk + bc + 1 is
    // the last ghost plane).  x = i0 - 2 = 32 blockIdx.x keeps the box start
    // on a 16-byte boundary.
    auto issue = [&](int p) {
        const uint32_t b = (uint32_t)(p % FR_NBUF);
        tc::mbar_expect_tx(mb_s + 8u * b, FluxRing::PLANE_BYTES);
        tc::tma_load_4d(ring_s + b * FluxRing::PLANE_BYTES, &tq, i0 - 2, j0 - 2, kb + p, 0, mb_s + 8u * b);
    };
    const double dt = *dtp;
    // dt/dz of plane kb + p, formed by one thread of the y-face warp
    const bool czw = tid == TY * FT_X;
    auto cz_of = [&](int p) { return (float)(dt / (zn[kb + p] - zn[kb + p - 1])); };
    if (tid == 0) {
        for (int b = 0; b < FR_NBUF; b++) tc::mbar_init(mb_s + 8u * b, 1);
        tc::fence_mbar_init();
    }
    if (czw) czb[0] = cz_of(0);
    __syncthreads();
    int issued = min(FR_NBUF, np + 2);
    if (tid == 0)
        for (int p = 0; p < issued; p++) issue(p);
    const bool zs_cell = SQ && i >= L.ni;
    const float ax = (float)(act ? -dt / (xn[i] - xn[i - 1]) : 0.0);
    const float by = (float)(act ? dt / (yn[j] - yn[j - 1]) : 0.0);
    const float2 ax2 = pk(ax, ax), nby2 = pk(-by, -by);
    float qb[NV], qa[NV], fo[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) qb[v] = qa[v] = fo[v] = 0.f;
    // the z face below the first plane from global memory, and the cell of
    // plane kb - 1 into the thread's slot
    float *slot = core + (cellw ? tid : 0);
    if (act) {
        face_flux_up<float, 3, DIFF>(q + L.at(i, j, kb) - 2 * (long long)sz, fs, sz, zs_cell, qb);
        const float *g = q + L.at(i, j, kb) - sz;
#pragma unroll
        for (int f = 0; f < NPRIM; f++) slot[f * FR_CS] = __ldg(g + (long long)f * fs);
    }
    const int so = (ty + 2) * HX + tx + 2;  // the cell inside a staged field plane
    // x faces: cell warps own face tx of row ty (cells i-2 .. i+1); the last
    // face warp lanes 0..7 own face 32 of row tx (lanes 8..31 repeat row
    // tx & 7 and store nothing)
    const int xr_row = cellw ? ty : (tx & (TY - 1));
    const int xr_col = cellw ? tx : FT_X;
    const bool xs_face = SQ && (i0 + xr_col - 1) >= L.ni;
    float *out = rhs + L.at(min(i, ilast), min(j, jlast), kb);
    bool ok = true;
    int p = 0;
    for (; p < np; p++) {
        const int b0 = p % FR_NBUF, b1 = (p + 1) % FR_NBUF, b2 = (p + 2) % FR_NBUF;
        if (p == 0) ok = tc::mbar_wait(mb_s + 8u * b0, 0, wait_tries) && ok;
        ok = tc::mbar_wait(mb_s + 8u * b1, ((p + 1) / FR_NBUF) & 1, wait_tries) && ok;
        const float *S0 = ring + b0 * FluxRing::PLANE, *S1 = ring + b1 * FluxRing::PLANE;
        const float *S2 = ring + b2 * FluxRing::PLANE;
        if (czw && p + 1 < np) czb[(p + 1) & 1] = cz_of(p + 1);
        // y face g of column i, between rows j0+g-1 and j0+g (staged rows
        // g .. g+3); x face f of row r, between columns i0+f-1 and i0+f
        // (staged columns f .. f+3).  A cell warp evaluates both in one
        // block of code (its y face g = ty, its x face f = tx); warp TY the
        // y faces g = 8, warp TY+1 the x faces f = 32.
        if (cellw) {
            face_flux_pk<2, DIFF>(PlaneSrc<HX>{S0 + ty * HX + tx + 2}, SQ && i >= L.ni, fy[ty][tx]);
            face_flux_pk<1, DIFF>(PlaneSrc<1>{S0 + (ty + 2) * HX + tx}, xs_face, fo);
        } else if (ty == TY) {
            face_flux_pk<2, DIFF>(PlaneSrc<HX>{S0 + ty * HX + tx + 2}, SQ && i >= L.ni, fy[ty][tx]);
        } else {
            face_flux_pk<1, DIFF>(PlaneSrc<1>{S0 + (xr_row + 2) * HX + FT_X}, xs_face, fo);
            if (tx < TY)
#pragma unroll
                for (int v = 0; v < NV; v++) fxe[tx][v] = fo[v];
        }
        // z face above the cell (between planes k and k+1): plane k+2 was
        // copied during the previous plane; then the cell of plane k
        // replaces that of plane k-1 in the slot
        ok = tc::mbar_wait(mb_s + 8u * b2, ((p + 2) / FR_NBUF) & 1, wait_tries) && ok;
        if (cellw) {
            face_flux_pk<3, DIFF>(ZColSrc{slot, S0 + so, S1 + so, S2 + so}, zs_cell, qa);
#pragma unroll
            for (int f = 0; f < NPRIM; f++) slot[f * FR_CS] = S0[so + f * PL];
        }
        if (__syncthreads_or(!ok)) break;
        // nothing reads plane p (buffer b0) after the barrier: plane p + 3
        // goes into it while the residuals are formed
        if (p + FR_NBUF <= np + 1) {
            if (tid == 0) issue(p + FR_NBUF);
            issued++;
        }
        if (cellw) {
            // every lane of a cell warp evaluates (inactive lanes on values
            // that are never stored): only the stores are predicated.  The
            // right x face comes from the next lane; lane 31's (face 32 of
            // the row) is sent by lane 0 from the face warp's slot.
            const float cz = czb[p & 1];
            const float2 ncz2 = pk(-cz, -cz);
            float fr[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                float send = fo[v];
                if (tx == 0) send = fxe[ty][v];
                fr[v] = __shfl_sync(0xffffffffu, send, (tx + 1) & (FT_X - 1));
            }
#pragma unroll
            for (int v = 0; v + 1 < NV; v += 2) {
                const float2 r = residual2(ax2, nby2, ncz2, pk(fr[v], fr[v + 1]), pk(fo[v], fo[v + 1]),
                                           pk(fy[ty + 1][tx][v], fy[ty + 1][tx][v + 1]),
                                           pk(fy[ty][tx][v], fy[ty][tx][v + 1]), pk(qa[v], qa[v + 1]),
                                           pk(qb[v], qb[v + 1]));
                if (act) {
                    out[v * (long long)fs] = r.x;
                    out[(v + 1) * (long long)fs] = r.y;
                }
            }
            const float rl = residual(ax, by, cz, fr[NV - 1], fo[NV - 1], fy[ty + 1][tx][NV - 1], fy[ty][tx][NV - 1],
                                      qa[NV - 1], qb[NV - 1]);
            if (act) out[(NV - 1) * (long long)fs] = rl;
#pragma unroll
            for (int v = 0; v < NV; v++) qb[v] = qa[v];
            out += sz;
        }
        __syncthreads();
    }
    if (p < np) {
        // a wait ran out: count it, let the copies in flight land (with the
        // full bound, whatever wait_tries was), stop.  If even that wait runs
        // out, copies may still be writing this block's shared memory when it
        // exits: drain_timeouts marks the device state as untrusted.
        if (tid == 0) {
            atomicAdd(&stat->wait_timeouts, 1ull);
            bool drained = true;
            for (int pl = p; pl < issued; pl++)
                drained = tc::mbar_wait(mb_s + 8u * (pl % FR_NBUF), (pl / FR_NBUF) & 1) && drained;
            if (!drained) atomicAdd(&stat->drain_timeouts, 1ull);
        }
        __syncthreads();
    }
}

}  // namespace eu3d
