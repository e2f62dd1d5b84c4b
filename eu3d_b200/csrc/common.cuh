// Device-side building blocks shared by all EU3D kernels: the HBM layout of
// the flowfield, the mechanism tables in constant memory and the NASA-9
// thermodynamic polynomials.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/eu3d_quirks.h"

namespace eu3d {

constexpr int NS = 9;        // species of the H2_JA919 mechanism
constexpr int NR = 19;       // reactions
constexpr int NV = NS + 4;   // conserved variables: NS partial densities, 3 momenta, total energy
constexpr int NPRIM = 7 + NS;  // primitive fields read by the flux sweeps
// primitive field order
constexpr int PD = 0, PU = 1, PV = 2, PW = 3, PP = 4, PH = 5, PG = 6, PY = 7;

constexpr double R_GAS = 8.31434;   // include/Reaction.hpp:269
constexpr double RU_CAL = 1.987;    // include/Reaction.hpp:270
constexpr double P0 = 101325.0;     // include/Reaction.hpp:271

// Ghost-padded structured grid in structure-of-arrays form: x fastest, each
// row padded to a multiple of 32 elements so that rows start 128-byte (FP32)
// or 256-byte (FP64) aligned, fields `fs` elements apart.
struct Layout {
    int ni, nj, nk, bc;
    int NI, NJ, NK;
    int px;        // row pitch in elements
    long long fs;  // field stride in elements
    __host__ __device__ long long at(int i, int j, int k) const { return ((long long)k * NJ + j) * px + i; }
    __host__ __device__ long long interior_cells() const { return (long long)ni * nj * nk; }
};

// Mechanism and thermo tables (constant memory, broadcast to all lanes).
struct MechConst {
    double c[2][9][NS];  // NASA-9 coefficients [range][a1..a7,b1,b2][species]
    double mw[NS], ri[NS];
    double imw[NS];      // 1 / mw
    double af[NR], bf[NR], eaf[NR];
    double sf[NS][NR], sb[NS][NR], tb[NS][NR];
    double nu[NS][NR];   // sb - sf
    double xr[NR];       // sum over species of (sb - sf)
    double p0xr[NR];     // pow(P0 * 1e-6, xr), evaluated on the host
    int has_tb[NR];      // reaction has third-body efficiencies
};

// defined once: every kernel lives in the single translation unit eu3d_gpu.cu
__constant__ MechConst cM;

struct Status {
    unsigned long long nonfinite;
    unsigned long long newton_capped;
    unsigned long long substeps;
    int nchem_max;
    int substep_capped;
    unsigned long long sur_cells;
    unsigned long long sur_fallback;
    unsigned long long audit_cells;        // surrogate cells also run through the integrator
    unsigned long long audit_max_dT_bits;  // largest |T_surrogate - T_integrator| (double bits)
    unsigned long long sur_reject[4];      // rejections: envelope, network output, energy residual, decode
    unsigned long long wait_timeouts;      // kernels that gave up a bounded wait (shared-memory ring, TMA)
    unsigned long long sur_frozen;         // cells the frozen-chemistry gate left out of the network
    unsigned long long frozen_audit_cells; // of those, cells also run through the integrator
    unsigned long long frozen_audit_max_dT_bits;  // largest |T_integrator - T| over them (double bits)
    unsigned long long drain_timeouts;     // a bounded wait for copies in flight after a timeout ran out too
};

// Powers of T shared by every species' polynomial at one temperature.
struct TPow {
    double T, lnT, tm1, tm2, t2, t3, t4, t5;
    int hi;  // 1 when T >= 1000 K (high-range table)
    int rb;  // table the integration constants b1, b2 come from
};

// q: the handle's EU3D_Q_* set (the b1/b2 defect selects rb)
__device__ __forceinline__ TPow tpow(double T, unsigned q)
{
    TPow p;
    p.T = T;
    p.lnT = log(T);
    p.tm1 = 1.0 / T;
    p.tm2 = p.tm1 * p.tm1;
    p.t2 = T * T;
    p.t3 = p.t2 * T;
    p.t4 = p.t2 * p.t2;
    p.t5 = p.t4 * T;
    p.hi = !(T < 1000.0);
    p.rb = (q & EU3D_Q_THERMO_B12_LOW) ? 0 : p.hi;
    return p;
}

// Cp/R, Reaction::GetCpi bracket (src/Reaction.cpp:893-904)
__device__ __forceinline__ double cp_r(int s, const TPow &p)
{
    const int r = p.hi;
    return cM.c[r][0][s] * p.tm2 + cM.c[r][1][s] * p.tm1 + cM.c[r][2][s] + cM.c[r][3][s] * p.T +
           cM.c[r][4][s] * p.t2 + cM.c[r][5][s] * p.t3 + cM.c[r][6][s] * p.t4;
}

// H/R, Reaction::GetHi bracket (src/Reaction.cpp:916-926); the b1 quirk
// takes the integration constant from the low range above 1000 K.
__device__ __forceinline__ double h_r(int s, const TPow &p)
{
    const int r = p.hi, rb = p.rb;
    return -cM.c[r][0][s] * p.tm1 + cM.c[r][1][s] * p.lnT + cM.c[r][2][s] * p.T + cM.c[r][3][s] * p.t2 * 0.5 +
           cM.c[r][4][s] * p.t3 * (1.0 / 3.0) + cM.c[r][5][s] * p.t4 * 0.25 + cM.c[r][6][s] * p.t5 * 0.2 +
           cM.c[rb][7][s];
}

// S/R, Reaction::GetSi bracket (src/Reaction.cpp:938-948)
__device__ __forceinline__ double s_r(int s, const TPow &p)
{
    const int r = p.hi, rb = p.rb;
    return -cM.c[r][0][s] * p.tm2 * 0.5 - cM.c[r][1][s] * p.tm1 + cM.c[r][2][s] * p.lnT + cM.c[r][3][s] * p.T +
           cM.c[r][4][s] * p.t2 * 0.5 + cM.c[r][5][s] * p.t3 * (1.0 / 3.0) + cM.c[r][6][s] * p.t4 * 0.25 +
           cM.c[rb][8][s];
}

template <class P>
struct PrimPtr {
    P *p;           // NPRIM fields
    long long fs;
    __device__ __forceinline__ P &operator()(int f, long long c) const { return p[f * fs + c]; }
};

}  // namespace eu3d
