// Learned chemistry surrogate: training-set generation, FP64 labels from the
// project's own integrators, the fused tensor-core MLP inference kernel and
// the per-cell apply step (conservation projection, envelope and residual
// checks, fallback list), plus the persistent fallback queue that runs the
// FP64 adaptive integrator (the network's teacher) on the cells the surrogate
// rejects.
//
// Sample record (states, FP64, 12 per sample): T [K], p [Pa], Y_0..Y_8, dt [s].
// Raw features (FP32, 12): T, ln(p / 1 atm), ln(Y_0 + 1e-12)..ln(Y_8 + 1e-12), ln dt.
// Raw labels (FP32, 12): dY_0..dY_8 (mass-fraction change over dt of a closed
// constant-density, constant-energy reactor, projected to element
// conservation), dT [K], weight (0 = unusable sample), label substeps.
//
// Targets: x_k = label_k / s_k with s_k = dt A(T) (Y_k + delta) for species
// and dt A(T) T for dT (relative rates; with delta = 0 the plain dt A(T)),
// A(T) = exp(Ta (1/Tr - 1/T)) an optional Arrhenius activity (Ta = 0: 1);
// y_k = asinh(x_k / lin_k), standardised with out_mean / out_std.  Inference
// inverts the chain.
#pragma once

#include "cell.cuh"
#include "mlp.cuh"

// offsets into the float normalisation vector (mirrored in include/eu3d_gpu.h)
#ifndef EU3D_SUR_NORM_LEN
#define EU3D_SUR_NORM_LEN 80
#endif

namespace eu3d {

constexpr int SN_IN_MEAN = 0, SN_IN_STD = 12, SN_OUT_MEAN = 24, SN_OUT_STD = 34, SN_LIN = 44, SN_TA = 54, SN_TR = 55,
              SN_ENV = 56, SN_RATIO = 62, SN_RATIO_TOL = 64, SN_RES_ABS = 65, SN_RES_REL = 66, SN_NEG_TOL = 67,
              SN_PROJ_EPS = 68, SN_DT_MAX = 69, SN_DELTA = 70;

struct SurNorm {
    float v[EU3D_SUR_NORM_LEN];
};

constexpr double ATM_PA = 101325.0;
constexpr float SUR_YFLOOR = 1e-12f;  // mass-fraction floor of the log inputs

// ------------------------------------------------------------------ RNG
__host__ __device__ __forceinline__ unsigned long long smix64(unsigned long long x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// uniform in [0, 1) from (seed, sample, draw)
__device__ __forceinline__ double urand(unsigned long long seed, unsigned long long idx, int k)
{
    return (double)(smix64(seed ^ smix64(idx * 64ull + (unsigned long long)k)) >> 11) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------ projection, energy
__device__ __forceinline__ void sur_project(const double Y[NS], double dY[NS], double eps) { elem_project(Y, dY, eps); }

// internal energy e(T) [J/kg] and cv [J/kg/K] of the mixture Y, with the
// arithmetic of the decode (mixture polynomial, kJ -> J)
__device__ __forceinline__ void mix_energy(const double Y[NS], double T, unsigned q, double &e, double &cv)
{
    double yr[NS], sYR = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        yr[s] = Y[s] * cM.ri[s];
        sYR += yr[s];
    }
    const TPow p = tpow(T, q);
    double A[8];
    mix_coeffs(yr, p.hi, p.rb, A);
    const double sh = -A[0] * p.tm1 + A[1] * p.lnT + A[2] * p.T + A[3] * p.t2 * 0.5 + A[4] * p.t3 * (1.0 / 3.0) +
                      A[5] * p.t4 * 0.25 + A[6] * p.t5 * 0.2 + A[7];
    const double scp = A[0] * p.tm2 + A[1] * p.tm1 + A[2] + A[3] * p.T + A[4] * p.t2 + A[5] * p.t3 + A[6] * p.t4;
    e = (sh - sYR * T) * 1e3;
    cv = (scp - sYR) * 1e3;
}

__device__ __forceinline__ double sur_activity(const SurNorm &n, double T)
{
    return exp((double)n.v[SN_TA] * (1.0 / (double)n.v[SN_TR] - 1.0 / T));
}

// ------------------------------------------------------- sample generation
struct SurSpecies {
    int H, O, H2O, OH, O2, H2, H2O2, HO2, N2;
};

// Random thermochemical states: T uniform, ln p uniform, ln dt uniform and a
// composition at the fixed element ratios of stoichiometric H2-air, built
// from the unburnt mixture 2 H2 + O2 + 3.76 N2 by element-preserving steps:
// progress to H2O, then dissociation into the radical pool.
__global__ void k_sur_random(double *__restrict__ states, long long base, long long n, unsigned long long seed,
                             SurSpecies sp, double Tlo, double Thi, double lnplo, double lnphi, double lndtlo,
                             double lndthi)
{
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (m >= n) return;
    const unsigned long long id = (unsigned long long)(base + m);
    double nm[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) nm[s] = 0.0;
    const double lam = urand(seed, id, 0);
    nm[sp.H2] = 2.0 - 2.0 * lam;
    nm[sp.O2] = 1.0 - lam;
    nm[sp.H2O] = 2.0 * lam;
    nm[sp.N2] = 3.76;
    double f[5];
#pragma unroll
    for (int r = 0; r < 5; r++) {
        const double u = urand(seed, id, 1 + r), v = urand(seed, id, 6 + r);
        f[r] = u < 0.15 ? 0.0 : pow(10.0, -7.0 + 6.5 * v);
    }
    double e;
    e = f[0] * nm[sp.H2];  // H2 -> 2 H
    nm[sp.H2] -= e;
    nm[sp.H] += 2 * e;
    e = f[1] * nm[sp.O2];  // O2 -> 2 O
    nm[sp.O2] -= e;
    nm[sp.O] += 2 * e;
    e = f[2] * nm[sp.H2O];  // H2O -> H + OH
    nm[sp.H2O] -= e;
    nm[sp.H] += e;
    nm[sp.OH] += e;
    e = f[3] * fmin(nm[sp.H], nm[sp.O2]);  // H + O2 -> HO2
    nm[sp.H] -= e;
    nm[sp.O2] -= e;
    nm[sp.HO2] += e;
    e = f[4] * 0.5 * nm[sp.OH];  // 2 OH -> H2O2
    nm[sp.OH] -= 2 * e;
    nm[sp.H2O2] += e;
    double tot = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        nm[s] = fmax(nm[s], 0.0) * cM.mw[s];
        tot += nm[s];
    }
    double *o = states + (base + m) * 12;
    o[0] = Tlo + (Thi - Tlo) * urand(seed, id, 11);
    o[1] = ATM_PA * exp(lnplo + (lnphi - lnplo) * urand(seed, id, 12));
#pragma unroll
    for (int s = 0; s < NS; s++) o[2 + s] = nm[s] / tot;
    o[11] = exp(lndtlo + (lndthi - lndtlo) * urand(seed, id, 13));
}

// Flowfield snapshot samples: every stride-th interior cell (from offset),
// its T, p and Y with multiplicative jitter on T and p and ln dt uniform.
template <class P>
__global__ void k_sur_snapshot(double *__restrict__ states, long long base, long long n, Layout L,
                               const double *__restrict__ T, const P *__restrict__ prim, long long stride,
                               long long offset, unsigned long long seed, double jT, double jP, double lndtlo,
                               double lndthi)
{
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (m >= n) return;
    const long long idx = offset + m * stride;
    const int i = (int)(idx % L.ni);
    const long long r = idx / L.ni;
    const int j = (int)(r % L.nj), k = (int)(r / L.nj);
    const long long c = L.at(i + L.bc, j + L.bc, k + L.bc);
    const unsigned long long id = (unsigned long long)(base + m);
    double Y[NS], tot = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        Y[s] = fmax((double)prim[(PY + s) * L.fs + c], 0.0);
        tot += Y[s];
    }
    double *o = states + (base + m) * 12;
    o[0] = T[c] * (1.0 + jT * (2.0 * urand(seed, id, 0) - 1.0));
    o[1] = (double)prim[PP * L.fs + c] * exp(jP * (2.0 * urand(seed, id, 1) - 1.0));
#pragma unroll
    for (int s = 0; s < NS; s++) o[2 + s] = Y[s] / tot;
    o[11] = exp(lndtlo + (lndthi - lndtlo) * urand(seed, id, 2));
}

// ------------------------------------------------------------------ labels
enum { SUR_LABEL_IMEX = 1, SUR_LABEL_TRAPEZOID = 0, SUR_LABEL_ADAPTIVE = 4 };

// Closed-reactor chemistry of one sample in FP64 with the project's
// integrators, then the element projection and the decode at constant
// density and internal energy.  kind SUR_LABEL_IMEX: one Diagonalized +
// Update_IMEX step with zero flux residual (the integrator the coupled run
// falls back to); SUR_LABEL_TRAPEZOID: TrapezoidPrediction substeps of the
// point-implicit trapezoid (capped at cap substeps); SUR_LABEL_ADAPTIVE: the
// adaptive species-implicit integrator (chem_adaptive, at most cap substeps).
template <bool SPEC>
__global__ void __launch_bounds__(128, 3)
    k_sur_label(const double *__restrict__ states, long long n, int kind, unsigned q, int cap, double proj_eps,
                AdaptCfg acfg, float *__restrict__ X, float *__restrict__ Lb)
{
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (m >= n) return;
    const double *sr = states + m * 12;
    const double T0 = sr[0], p0 = sr[1], dt = sr[11];
    double Y0[NS], sdiv = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        Y0[s] = sr[2 + s];
        sdiv += Y0[s] / cM.mw[s];
    }
    const double D0 = p0 / (R_GAS * 1000 * sdiv * T0);
    double E0, cv0;
    mix_energy(Y0, T0, q, E0, cv0);
    double cs[NV];
#pragma unroll
    for (int s = 0; s < NS; s++) cs[s] = D0 * Y0[s];
    cs[NS] = cs[NS + 1] = cs[NS + 2] = 0.0;
    cs[NS + 3] = D0 * E0;
    Decoded o;
    int capped = 0, bad = 0, nsub = 1;
    double Tg = T0;
    double dY[NS];
    bool projected = false;
    if (kind == SUR_LABEL_ADAPTIVE) {
        int cp = 0;
        acfg.nmax = cap;
        int forced = 0;
        nsub = chem_increment<SPEC>(cs, T0, E0, q, dt, acfg, proj_eps, dY, Tg, cp, forced);
        bad |= cp;
        projected = true;
    } else if (kind == SUR_LABEL_IMEX) {
        double CMS[NS], MD[NS];
        imex_source<SPEC>(cs, T0, q, CMS, MD);
#pragma unroll
        for (int s = 0; s < NS; s++) cs[s] = cs[s] + (CMS[s] * dt) / (1.0 - dt * MD[s]);
        decode(cs, T0, E0, q, o, capped);
        Tg = o.T;
    } else {
        const int rtb = (q & EU3D_Q_ADAPT_RTB_ZERO) ? 2 : 0;
        decode(cs, T0, E0, q, o, capped);
        int nn = predict_nchem<SPEC>(tpow(o.T, q), cs, o.Y, dt, rtb);
        if (nn > cap) {
            nn = cap;
            bad = 1;
        }
        nsub = nn;
        const double dts = dt / nn;
        for (int st = 0; st < nn; st++) {
            double dn[NS], Wi[NS];
            trapezoid<SPEC>(tpow(o.T, q), cs, dts, rtb, dn, Wi);
            double D = 0.0;
#pragma unroll
            for (int s = 0; s < NS; s++) {
                cs[s] = dn[s];
                D += cs[s];
            }
            cs[NS + 3] = D * o.E;
            decode(cs, o.T, o.E, q, o, capped);
            bad |= capped;
        }
        Tg = o.T;
    }
    if (!projected) {
        double Dn = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) Dn += cs[s];
#pragma unroll
        for (int s = 0; s < NS; s++) dY[s] = cs[s] / Dn - Y0[s];
        sur_project(Y0, dY, proj_eps);
    }
    // decode of the projected composition at (D0, E0)
    double cp[NV];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double y = Y0[s] + dY[s];
        if (y < -1e-7) bad = 1;
        cp[s] = D0 * fmax(y, 0.0);
    }
    cp[NS] = cp[NS + 1] = cp[NS + 2] = 0.0;
    cp[NS + 3] = D0 * E0;
    decode(cp, Tg, E0, q, o, capped);
    bad |= capped;
    const double dT = o.T - T0;
    bad |= !isfinite(dT);
#pragma unroll
    for (int s = 0; s < NS; s++) bad |= !isfinite(dY[s]);
    float *x = X + m * 12;
    x[0] = (float)T0;
    x[1] = (float)log(p0 / ATM_PA);
#pragma unroll
    for (int s = 0; s < NS; s++) x[2 + s] = logf((float)Y0[s] + SUR_YFLOOR);
    x[11] = (float)log(dt);
    float *l = Lb + m * 12;
#pragma unroll
    for (int s = 0; s < NS; s++) l[s] = bad ? 0.f : (float)dY[s];
    l[9] = bad ? 0.f : (float)dT;
    l[10] = bad ? 0.f : 1.f;
    l[11] = (float)nsub;
}

// ------------------------------------------------------- training batches
// Normalised network inputs.  BF16 keeps 8 significant bits, which would
// resolve T to several kelvin; the spare input columns 12..14 carry the BF16
// rounding residuals of T, ln p and ln dt scaled by 256, so that the first
// layer sees those three at about 16 bits.
__device__ __forceinline__ float bf16_residual(float x) { return (x - __bfloat162float(__float2bfloat16_rn(x))) * 256.f; }

__device__ __forceinline__ void sur_features(const SurNorm &n, const float raw[SUR_NIN], float f[SUR_IN])
{
#pragma unroll
    for (int i = 0; i < SUR_NIN; i++) f[i] = (raw[i] - n.v[SN_IN_MEAN + i]) / n.v[SN_IN_STD + i];
    f[12] = bf16_residual(f[0]);
    f[13] = bf16_residual(f[1]);
    f[14] = bf16_residual(f[11]);
    f[15] = 0.f;
}

// Random minibatch (with replacement): normalised features (B x 16) and
// standardised targets (B x 16, column 15 = sample weight).
__global__ void k_sur_batch(const float *__restrict__ X, const float *__restrict__ Lb, long long n, SurNorm nrm,
                            unsigned long long seed, long long step, int B, float *__restrict__ Xb,
                            float *__restrict__ Yb)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const long long idx = (long long)(smix64(seed ^ smix64((unsigned long long)step * 0x100000001ull + r)) % n);
    float raw[SUR_NIN], f[SUR_IN];
#pragma unroll
    for (int i = 0; i < SUR_NIN; i++) raw[i] = X[idx * 12 + i];
    sur_features(nrm, raw, f);
#pragma unroll
    for (int i = 0; i < SUR_IN; i++) Xb[(long long)r * SUR_IN + i] = f[i];
    const double T = raw[0], dt = exp((double)raw[11]);
    const double sc = dt * sur_activity(nrm, T);
    const double delta = nrm.v[SN_DELTA];
    const float *l = Lb + idx * 12;
    float *y = Yb + (long long)r * SUR_OUT;
#pragma unroll
    for (int k = 0; k < SUR_NOUT; k++) {
        const double rel = delta > 0 ? (k < NS ? exp((double)raw[2 + k]) - (double)SUR_YFLOOR + delta : T) : 1.0;
        const double x = (double)l[k] / (sc * rel);
        const double t = asinh(x / (double)nrm.v[SN_LIN + k]);
        y[k] = (float)((t - nrm.v[SN_OUT_MEAN + k]) / nrm.v[SN_OUT_STD + k]);
    }
    for (int k = SUR_NOUT; k < 15; k++) y[k] = 0.f;
    y[15] = l[10];
}

// normalised network output of one output -> raw label (dY_k or dT)
__device__ __forceinline__ float sur_unscale_f(const SurNorm &n, int k, float t, float sc)
{
    const float y = fmaf(t, n.v[SN_OUT_STD + k], n.v[SN_OUT_MEAN + k]);
    // sinh from one fast exponential (the network's output is BF16-accurate)
    const float e = __expf(fminf(fmaxf(y, -80.f), 80.f));
    return sc * n.v[SN_LIN + k] * (0.5f * (e - __frcp_rn(e)));
}

// ------------------------------------------------ fused inference kernel
// 12 -> 128 -> 128 -> 128 -> 10 MLP on the tensor cores.  One CTA holds the
// four weight matrices in shared memory for its whole life and runs NG tile
// groups of 128 threads; each group owns 128 TMEM columns and a 32 KB
// activation tile, and walks 128-cell tiles: features -> bf16 A tile ->
// tcgen05.mma (FP32 accumulators in TMEM) -> tcgen05.ld, GELU, bf16 -> the
// next layer's A tile.  While one group runs its epilogue on the CUDA cores,
// another group's MMAs occupy the tensor pipe.  The biases ride on the tensor
// cores too, in BF16: layer 1 through its spare input column 15 (held at 1,
// with the bias in W1's row 15), layers 2..4 through one more K = 16 MMA of
// a shared all-ones column against a bias column.
constexpr int SUR_NG = 4;
constexpr int SURK_W1 = 0;                             // 128 x 16
constexpr int SURK_W2 = SURK_W1 + SUR_H * SUR_IN * 2;  // 128 x 128
constexpr int SURK_W3 = SURK_W2 + SUR_H * SUR_H * 2;
constexpr int SURK_W4 = SURK_W3 + SUR_H * SUR_H * 2;   // 16 x 128
constexpr int SURK_ONES = SURK_W4 + SUR_OUT * SUR_H * 2;   // 128 x 16, column 0 = 1
constexpr int SURK_BB2 = SURK_ONES + 128 * 16 * 2;           // 128 x 16, column 0 = b2
constexpr int SURK_BB3 = SURK_BB2 + SUR_H * 16 * 2;          // 128 x 16, column 0 = b3
constexpr int SURK_BB4 = SURK_BB3 + SUR_H * 16 * 2;          // 16 x 16, column 0 = b4
constexpr int SURK_A = SURK_BB4 + SUR_OUT * 16 * 2;
constexpr int SURK_ATILE = 128 * SUR_H * 2;
constexpr int SURK_MBAR = SURK_A + SUR_NG * SURK_ATILE;
constexpr int SURK_SMEM = SURK_MBAR + SUR_NG * 8 + 16;

struct SurWeights {
    const __nv_bfloat16 *Wt[4];  // out x in, row-major
    const float *p;              // flat FP32 parameters (biases)
};

// feature sources / output sinks
struct SurSrcArray {  // normalised features, n x 16 FP32; outputs n x 16
    const float *X;
    float *out;
    long long n;
    long long ntiles() const { return (n + 127) / 128; }
    __device__ __forceinline__ long long tiles(long long host_tiles) const { return host_tiles; }
    __device__ __forceinline__ bool load(long long tile, int lane, const SurNorm &, float f[SUR_IN], long long &idx) const
    {
        idx = tile * 128 + lane;
        if (idx >= n) return false;
        const float4 *p = reinterpret_cast<const float4 *>(X + idx * SUR_IN);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const float4 a = p[v];
            f[4 * v] = a.x;
            f[4 * v + 1] = a.y;
            f[4 * v + 2] = a.z;
            f[4 * v + 3] = a.w;
        }
        return true;
    }
    __device__ __forceinline__ void store(long long, int, long long idx, const float o[SUR_OUT]) const
    {
        float4 *p = reinterpret_cast<float4 *>(out + idx * SUR_OUT);
#pragma unroll
        for (int v = 0; v < 4; v++) p[v] = make_float4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
    }
};

// Tiles follow x rows (tpr tiles of 128 cells per row) so that a tile's
// cells are contiguous in memory and no 64-bit division is needed.
// normalised network inputs of flowfield cell c: T, ln(p / 1 atm), ln(Y_k + floor), ln dt
template <class P>
__device__ __forceinline__ void sur_cell_features(const SurNorm &nrm, const double *__restrict__ T,
                                                  const P *__restrict__ prim, long long fs, const double *scal,
                                                  long long c, float f[SUR_IN])
{
    float raw[SUR_NIN];
    raw[0] = (float)T[c];
    raw[1] = __logf((float)prim[PP * fs + c] * (float)(1.0 / ATM_PA));
#pragma unroll
    for (int s = 0; s < NS; s++) raw[2 + s] = __logf(fmaxf((float)prim[(PY + s) * fs + c], 0.f) + SUR_YFLOOR);
    raw[11] = __logf((float)scal[0]);
    sur_features(nrm, raw, f);
}

template <class P>
struct SurSrcField {  // interior cells of a flowfield; outputs SoA (10 x n)
    Layout L;
    const double *T;
    const P *prim;
    const double *scal;
    float *out;
    long long n;
    int tpr;  // tiles per x row
    long long ntiles() const { return (long long)tpr * L.nj * L.nk; }
    __device__ __forceinline__ long long tiles(long long host_tiles) const { return host_tiles; }
    __device__ __forceinline__ bool load(long long tile, int lane, const SurNorm &nrm, float f[SUR_IN],
                                         long long &idx) const
    {
        const int t = (int)tile;
        const int r = t / tpr;
        const int i = (t - r * tpr) * 128 + lane;
        if (i >= L.ni) return false;
        const int j = r % L.nj, k = r / L.nj;
        idx = (long long)r * L.ni + i;
        sur_cell_features<P>(nrm, T, prim, L.fs, scal, L.at(i + L.bc, j + L.bc, k + L.bc), f);
        return true;
    }
    __device__ __forceinline__ void store(long long, int, long long idx, const float o[SUR_OUT]) const
    {
#pragma unroll
        for (int k = 0; k < SUR_NOUT; k++) out[k * n + idx] = o[k];
    }
};

// The cells of a list (the active cells the frozen-chemistry gate kept):
// tile t takes list positions 128 t .. 128 t + 127; the list's length is on
// the device, so the kernel reads its tile count there.  Outputs SoA
// (10 x cap) by list position.
template <class P>
struct SurSrcList {
    Layout L;
    const double *T;
    const P *prim;
    const double *scal;
    float *out;
    const int *list;
    const int *count;
    long long cap;
    long long ntiles() const { return (cap + 127) / 128; }  // a bound for the grid size
    __device__ __forceinline__ long long total() const { return min((long long)*count, cap); }
    __device__ __forceinline__ long long tiles(long long) const { return (total() + 127) / 128; }
    __device__ __forceinline__ bool load(long long tile, int lane, const SurNorm &nrm, float f[SUR_IN],
                                         long long &idx) const
    {
        idx = tile * 128 + lane;
        if (idx >= total()) return false;
        sur_cell_features<P>(nrm, T, prim, L.fs, scal, (long long)list[idx], f);
        return true;
    }
    __device__ __forceinline__ void store(long long, int, long long idx, const float o[SUR_OUT]) const
    {
#pragma unroll
        for (int k = 0; k < SUR_NOUT; k++) out[k * cap + idx] = o[k];
    }
};

// stage a row-major (R x K) bf16 matrix into the canonical K-major operand
// layout; half: every weight halved (exact in BF16) for layers fed by
// gelu2_bf16x2
__device__ __forceinline__ void sur_stage(unsigned char *dst, const __nv_bfloat16 *src, int R, int K, int tid,
                                          int nthr, bool half = false)
{
    const int vec = K >> 3;
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(0.5f, 0.5f);
    for (int v = tid; v < R * vec; v += nthr) {
        const int r = v / vec, kk = (v % vec) * 8;
        uint4 w = *reinterpret_cast<const uint4 *>(src + (size_t)r * K + kk);
        if (half) {
            __nv_bfloat162 *e = reinterpret_cast<__nv_bfloat162 *>(&w);
#pragma unroll
            for (int q = 0; q < 4; q++) e[q] = __hmul2(e[q], h2);
        }
        *reinterpret_cast<uint4 *>(dst + tc::op_off(R, r, kk)) = w;
    }
}

__device__ __forceinline__ void named_bar(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

// hidden-layer epilogue of one row: 128 accumulators (bias included) ->
// 2 GELU -> bf16 A tile (the next layer's weights are staged halved)
__device__ __forceinline__ void sur_hidden_epilogue(uint32_t tmem_row, unsigned char *A, int row)
{
#pragma unroll
    for (int c0 = 0; c0 < SUR_H; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem_row + c0, v);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint4 w;
            w.x = gelu2_bf16x2(v[8 * q + 0], v[8 * q + 1]);
            w.y = gelu2_bf16x2(v[8 * q + 2], v[8 * q + 3]);
            w.z = gelu2_bf16x2(v[8 * q + 4], v[8 * q + 5]);
            w.w = gelu2_bf16x2(v[8 * q + 6], v[8 * q + 7]);
            *reinterpret_cast<uint4 *>(A + tc::op_off(128, row, c0 + 8 * q)) = w;
        }
    }
}

// a K = 16 operand tile of R rows whose column 0 holds bf16(src[r] * scale) (or
// 1 when src is null) and whose other columns are zero
__device__ __forceinline__ void sur_stage_col(unsigned char *dst, const float *src, int R, int tid, int nthr)
{
    for (int v = tid; v < R * 2; v += nthr) {
        const int r = v >> 1, half = v & 1;
        uint4 z = make_uint4(0u, 0u, 0u, 0u);
        if (half == 0) {
            const __nv_bfloat16 b = __float2bfloat16_rn(src ? src[r] : 1.0f);
            z.x = (uint32_t)__bfloat16_as_ushort(b);
        }
        *reinterpret_cast<uint4 *>(dst + tc::op_off(R, r, 8 * half)) = z;
    }
}

template <class Src>
__global__ void __launch_bounds__(128 * SUR_NG, 1) k_sur_mlp(SurWeights W, const SurNorm *__restrict__ nrm_g, Src src,
                                                           long long ntiles, int *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int g = tid >> 7, t = tid & 127, warp = tid >> 5;
    __shared__ SurNorm nrm;
    for (int v = tid; v < EU3D_SUR_NORM_LEN; v += nthr) nrm.v[v] = nrm_g->v[v];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + SURK_MBAR);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + SURK_MBAR + SUR_NG * 8);
    unsigned char *A = sm + SURK_A + g * SURK_ATILE;

    sur_stage(sm + SURK_W1, W.Wt[0], SUR_H, SUR_IN, tid, nthr);
    sur_stage(sm + SURK_W2, W.Wt[1], SUR_H, SUR_H, tid, nthr, true);
    sur_stage(sm + SURK_W3, W.Wt[2], SUR_H, SUR_H, tid, nthr, true);
    sur_stage(sm + SURK_W4, W.Wt[3], SUR_OUT, SUR_H, tid, nthr, true);
    sur_stage_col(sm + SURK_ONES, nullptr, 128, tid, nthr);
    sur_stage_col(sm + SURK_BB2, W.p + SUR_OFF_B2, SUR_H, tid, nthr);
    sur_stage_col(sm + SURK_BB3, W.p + SUR_OFF_B3, SUR_H, tid, nthr);
    sur_stage_col(sm + SURK_BB4, W.p + SUR_OFF_B4, SUR_OUT, tid, nthr);
    __syncthreads();
    // layer 1's bias takes the place of W1's row 15 (input column 15 is held at 1)
    for (int n = tid; n < SUR_H; n += nthr)
        *reinterpret_cast<__nv_bfloat16 *>(sm + SURK_W1 + tc::op_off(SUR_H, n, 15)) =
            __float2bfloat16_rn(W.p[SUR_OFF_B1 + n]);
    if (warp == 0) tc::tmem_alloc(slot, 128 * SUR_NG);
    if (tid == 0) {
        for (int q = 0; q < SUR_NG; q++) tc::mbar_init(tc::smem_u32(mbar + q), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *slot + (uint32_t)(g * 128);
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const uint32_t mb = tc::smem_u32(mbar + g);
    const uint32_t aS = tc::smem_u32(A);
    const uint32_t w1 = tc::smem_u32(sm + SURK_W1), w2 = tc::smem_u32(sm + SURK_W2), w3 = tc::smem_u32(sm + SURK_W3),
                   w4 = tc::smem_u32(sm + SURK_W4);
    const uint32_t id128 = tc::idesc_bf16(128, SUR_H), id16 = tc::idesc_bf16(128, SUR_OUT);
    const uint32_t ones = tc::smem_u32(sm + SURK_ONES), bb2 = tc::smem_u32(sm + SURK_BB2),
                   bb3 = tc::smem_u32(sm + SURK_BB3), bb4 = tc::smem_u32(sm + SURK_BB4);
    uint32_t phase = 0;
    bool ok = true;
    ntiles = src.tiles(ntiles);  // the list form reads its length on the device

    for (long long tile = (long long)blockIdx.x * SUR_NG + g; tile < ntiles; tile += (long long)gridDim.x * SUR_NG) {
        long long idx = 0;
        float f[SUR_IN];
        const bool have = src.load(tile, t, nrm, f, idx);
        if (!have)
#pragma unroll
            for (int i = 0; i < SUR_IN; i++) f[i] = 0.f;
        f[15] = 1.0f;  // carries layer 1's bias
        uint4 w0, w1v;
        w0.x = pack_bf16(f[0], f[1]);
        w0.y = pack_bf16(f[2], f[3]);
        w0.z = pack_bf16(f[4], f[5]);
        w0.w = pack_bf16(f[6], f[7]);
        w1v.x = pack_bf16(f[8], f[9]);
        w1v.y = pack_bf16(f[10], f[11]);
        w1v.z = pack_bf16(f[12], f[13]);
        w1v.w = pack_bf16(f[14], f[15]);
        *reinterpret_cast<uint4 *>(A + tc::op_off(128, t, 0)) = w0;
        *reinterpret_cast<uint4 *>(A + tc::op_off(128, t, 8)) = w1v;
#pragma unroll
        for (int layer = 0; layer < 4; layer++) {
            tc::fence_async_smem();
            tc::fence_before();
            named_bar(1 + g, 128);
            if (t == 0) {
                tc::fence_after();
                if (layer == 0) {
                    tc::mma(tmem, tc::sdesc(aS), tc::sdesc(w1), id128, 0u);
                } else {
                    const uint32_t wb = layer == 1 ? w2 : layer == 2 ? w3 : w4;
                    const int N = layer == 3 ? SUR_OUT : SUR_H;
                    const uint32_t idd = layer == 3 ? id16 : id128;
#pragma unroll
                    for (int s = 0; s < SUR_H / 16; s++)
                        tc::mma(tmem, tc::sdesc(aS + s * 128 * 32), tc::sdesc(wb + s * N * 32), idd, s > 0 ? 1u : 0u);
                    const uint32_t bb = layer == 1 ? bb2 : layer == 2 ? bb3 : bb4;
                    tc::mma(tmem, tc::sdesc(ones), tc::sdesc(bb), idd, 1u);  // + bias
                }
                tc::commit(mb);
            }
            ok = tc::mbar_wait(mb, phase) && ok;
            phase ^= 1;
            tc::fence_after();
            if (layer < 3) {
                sur_hidden_epilogue(trow, A, t);
            } else {
                float o[SUR_OUT];
                tc::tmem_ld16(trow, o);
                if (have) src.store(tile, t, idx, o);
            }
        }
        tc::fence_before();
    }
    if (!ok && err) atomicExch(err, 1);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(*slot, 128 * SUR_NG);
}

// ------------------------------------------------------ coupled-step apply
// Fallback list entries: the cell index (below 2^30) with two flags.
constexpr unsigned SUR_AUDIT = 0x80000000u;         // an accepted cell re-run to judge the network
constexpr unsigned SUR_FROZEN_AUDIT = 0x40000000u;  // a frozen cell re-run to judge the gate
constexpr int SUR_CELL_MASK = 0x3fffffff;

struct SurQueue {
    int *list;      // cell indices with the flags above
    int *count;     // [0] list length, [1] work cursor
    double *audit;  // per list slot: the temperature to judge for audited cells
    long long cap;
    double *res;    // per list slot, field-major (cap apart): the integrated species and T
    int *info;      // per list slot: substeps | SUR_CAPPED | SUR_FORCED
};
constexpr int SUR_CAPPED = 1 << 24;  // a Newton iteration ran into its cap
constexpr int SUR_FORCED = 1 << 25;  // the substep cap lengthened a substep

struct SurApplyArgs {
    CellArgs a;
    const SurNorm *nrm;  // device copy
    const float *out;  // 10 x n network outputs (SoA)
    long long n;       // interior cells
    SurQueue qu;
    int audit_stride;  // 0: no audit
};

__device__ __forceinline__ void sur_push(const SurQueue &qu, bool push, int value, double audit_T)
{
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, push);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(qu.count, __popc(m));
    base = __shfl_sync(act, base, leader);
    if (push) {
        const int slot = base + __popc(m & ((1u << lane) - 1u));
        if (slot < qu.cap) {
            qu.list[slot] = value;
            qu.audit[slot] = audit_T;
        }
    }
}

// One thread per interior cell, after the flux update and its decode (a split
// step, as the adaptive integrator's).  The network's chemistry increment
// over dt for the cell's state is projected to element conservation, checked
// against the training envelope, for negative mass fractions and for the
// energy balance at the predicted temperature, then applied to the species
// and decoded in FP64.  Rejected cells (and audited ones) go to the fallback
// list untouched.  (i, j, k): ghosted indices; net: the cell's network outputs.
// Outcome bits of sur_apply_cell, in the order of the status counters it
// feeds: accepted, fallen back, then the rejection reasons (envelope,
// network output, energy residual, failed decode).
constexpr int SUR_NFLAGS = 6;

// SOLID false: the caller passes fluid cells only (the gate's list), so the
// wedge test and its node-coordinate loads are left out.
template <class P, bool COUNT = true, bool SOLID = true>
__device__ __forceinline__ unsigned sur_apply_cell(const SurApplyArgs &s, P *__restrict__ q, int i, int j, int k,
                                                   const float net[SUR_NOUT])
{
    const CellArgs &a = s.a;
    const Layout &L = a.L;
    if (SOLID && solid_cell(a, i, j)) return 0u;
    const long long c = L.at(i, j, k);
    const long long fs = L.fs;
    const long long idx = ((long long)(k - L.bc) * L.nj + (j - L.bc)) * L.ni + (i - L.bc);
    const unsigned qk = a.quirks;
    const SurNorm &n = *s.nrm;
    const double dt = a.scal[0];
    double cs[NV];
    load_cs(a.cs, fs, c, cs);
    const double T = a.T[c], Eold = a.E[c];
    double D = 0.0, sdiv = 0.0;
#pragma unroll
    for (int sp = 0; sp < NS; sp++) D += cs[sp];
    const double iD = 1.0 / D;
    double Y[NS];
#pragma unroll
    for (int sp = 0; sp < NS; sp++) {
        Y[sp] = cs[sp] * iD;
        sdiv += Y[sp] * cM.imw[sp];
    }
    const double p = D * R_GAS * 1000 * sdiv * T;
    // envelope and network-output arithmetic in FP32 (the network itself is BF16)
    const float Tf = (float)T;
    const float lnp = logf((float)(p * (1.0 / ATM_PA))), lndt = logf((float)dt);
    bool ok = Tf >= n.v[SN_ENV + 0] && Tf <= n.v[SN_ENV + 1] && lnp >= n.v[SN_ENV + 2] && lnp <= n.v[SN_ENV + 3] &&
              lndt >= n.v[SN_ENV + 4] && lndt <= n.v[SN_ENV + 5];
    bool ok_env;
    {
        double el[SUR_NELEM];
#pragma unroll
        for (int e = 0; e < SUR_NELEM; e++) {
            double x = 0.0;
#pragma unroll
            for (int sp = 0; sp < NS; sp++) x += c_sur_elem[e][sp] * Y[sp];
            el[e] = x;
        }
        const double tol = n.v[SN_RATIO_TOL];
        ok = ok && fabs(el[0] / (el[1] * n.v[SN_RATIO + 0]) - 1.0) <= tol &&
             fabs(el[2] / (el[1] * n.v[SN_RATIO + 1]) - 1.0) <= tol;
        ok_env = ok;
    }
    const float sc = (float)dt * expf(n.v[SN_TA] * (1.f / n.v[SN_TR] - 1.f / Tf));
    const float delta = n.v[SN_DELTA];
    double dY[NS];
#pragma unroll
    for (int sp = 0; sp < NS; sp++)
        dY[sp] = (double)sur_unscale_f(n, sp, net[sp], delta > 0.f ? sc * ((float)Y[sp] + delta) : sc);
    const double dTn = (double)sur_unscale_f(n, NS, net[NS], delta > 0.f ? sc * Tf : sc);
    sur_project(Y, dY, n.v[SN_PROJ_EPS]);
    double Yn[NS];
#pragma unroll
    for (int sp = 0; sp < NS; sp++) {
        const double y = Y[sp] + dY[sp];
        ok = ok && y >= -(double)n.v[SN_NEG_TOL] && isfinite(y);
        Yn[sp] = fmax(y, 0.0);
    }
    ok = ok && isfinite(dTn) && fabs(dTn) <= n.v[SN_DT_MAX];
    const bool ok_out = ok;
    const double Tg = T + dTn;
    Decoded o;
    int capped = 0;
    bool ok_res = ok;
    if (ok) {
        // the chemistry increment on the species (the flux update is in
        // already), decoded from the predicted temperature.  The decode's
        // first Newton correction is the energy residual of the prediction
        // at constant density and energy, (e(Y + dY, T + dT) - E) / cv; its
        // converged result stands in for it: the prediction is kept when
        // |T_decoded - (T + dT)| <= res_abs + res_rel |dT|.
#pragma unroll
        for (int v = 0; v < NS; v++) cs[v] = D * Yn[v];
        decode(cs, Tg, Eold, qk, o, capped);
        ok_res = fabs(o.T - Tg) <= n.v[SN_RES_ABS] + n.v[SN_RES_REL] * fabs(dTn);
        // a decode that fails or leaves the envelope's temperatures goes back
        // to the integrator (from the untouched old state)
        ok = ok_res && !capped && isfinite(o.T) && isfinite(o.D) && o.T >= 0.8 * n.v[SN_ENV + 0] &&
             o.T <= 1.2 * n.v[SN_ENV + 1];
    }
    // (interior cells are fewer than 2^31)
    const bool audit = ok && s.audit_stride > 0 && ((unsigned)idx % (unsigned)s.audit_stride) == 0;
    if (ok) {
        if (!audit) {
#pragma unroll
            for (int v = 0; v < NS; v++) a.cs[v * fs + c] = cs[v];  // momenta and energy are unchanged
            a.T[c] = o.T;
            a.E[c] = o.E;
            store_prims<P>(o, q, fs, c);
        }
    }
    sur_push(s.qu, !ok || audit, (int)((unsigned)c | (audit ? SUR_AUDIT : 0u)), audit ? o.T : 0.0);
    const unsigned flags = (ok && !audit ? 1u : 0u) | (!ok ? 2u : 0u) | (!ok_env ? 4u : 0u) |
                           (ok_env && !ok_out ? 8u : 0u) | (ok_out && !ok_res ? 16u : 0u) | (ok_res && !ok ? 32u : 0u);
    if (COUNT) {
        warp_count(&a.st->sur_cells, flags & 1u);
        warp_count(&a.st->sur_fallback, flags & 2u);
        warp_count(&a.st->sur_reject[0], flags & 4u);
        warp_count(&a.st->sur_reject[1], flags & 8u);
        warp_count(&a.st->sur_reject[2], flags & 16u);
        warp_count(&a.st->sur_reject[3], flags & 32u);
    }
    return flags;
}

// Block-level counting: each warp adds its lanes' flags to shared counters,
// then one thread per counter adds the block's sums to the status -- one
// global atomic per counter and block instead of per warp (the counters are
// a few hot addresses).  All threads of the block must call both.
template <int N>
struct BlockCount {
    unsigned long long *sm;  // N shared counters
    __device__ __forceinline__ void init() const
    {
        if (threadIdx.x < N) sm[threadIdx.x] = 0ull;
        __syncthreads();
    }
    __device__ __forceinline__ void add(unsigned flags) const
    {
#pragma unroll
        for (int b = 0; b < N; b++) {
            const unsigned m = __ballot_sync(0xffffffffu, (flags >> b) & 1u);
            if ((threadIdx.x & 31) == 0 && m) atomicAdd(&sm[b], (unsigned long long)__popc(m));
        }
    }
    __device__ __forceinline__ void flush(unsigned long long *const dst[N]) const
    {
        __syncthreads();
        if (threadIdx.x < N && sm[threadIdx.x]) atomicAdd(dst[threadIdx.x], sm[threadIdx.x]);
    }
};

// One thread per interior cell: the network outputs from the MLP kernel's
// output buffer.
template <class P>
__global__ void __launch_bounds__(128, 7) k_sur_apply(SurApplyArgs s, P *__restrict__ q)
{
    const Layout &L = s.a.L;
    const int i = L.bc + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = L.bc + blockIdx.y;
    const int k = L.bc + blockIdx.z;
    if (i >= L.ni + L.bc) return;
    const long long idx = ((long long)(k - L.bc) * L.nj + (j - L.bc)) * L.ni + (i - L.bc);
    float o[SUR_NOUT];
#pragma unroll
    for (int v = 0; v < SUR_NOUT; v++) o[v] = s.out[v * s.n + idx];
    sur_apply_cell<P>(s, q, i, j, k, o);
}

// Frozen-chemistry gate.  A fluid cell colder than T_frozen whose summed
// mass fraction over the species of `mask` (the radicals) is at most y_max
// keeps the state its flux update and decode left: over one flow time step
// its chemistry changes nothing the FP64 integrator would resolve (cold
// H2-air ahead of the shock has ignition delays of seconds against steps of
// tens of nanoseconds).  The other fluid cells are listed for the network.
// About one frozen cell in audit_stride (a fixed hash sample of the interior
// index, gate_sample) is also sent to the fallback queue, whose FP64
// integrator records the largest temperature change the gate ignored.
struct SurGate {
    double T_frozen;
    float y_max_f;  // compared with the FP32 sum of the radicals' mass fractions
    unsigned mask;
    int audit_stride;  // 0: no audit
    int *active;       // listed cells (ghosted indices)
    int *acount;       // list length
};

// One block of GATE_THREADS threads per x segment of GATE_ROW cells of a row,
// each thread taking GATE_CPT cells GATE_THREADS apart with all their loads
// issued before the first test; blocks over the (j, k) rows in blockIdx.x
// (no 65535 limit).  The block appends its active cells, in x order, with one
// global atomic.  A block's life is a chain of round trips (node coordinates,
// T and the radicals, the list atomic, the list stores), so the kernel is
// bound by latency: four cells a thread keep four times the loads in flight
// per resident thread.  The radical test runs in FP32 (the primitives'
// precision of the benchmark path) and the audit sample is drawn by a
// multiplicative hash instead of a division.
constexpr int GATE_THREADS = 128, GATE_CPT = 4, GATE_ROW = GATE_THREADS * GATE_CPT;

// deterministic sample of about one cell in `stride` (Knuth's multiplicative hash)
__device__ __forceinline__ bool gate_sample(long long idx, unsigned stride)
{
    return stride > 0 && (unsigned)idx * 2654435761u < 0xFFFFFFFFu / stride;
}

template <class P>
__global__ void __launch_bounds__(GATE_THREADS) k_sur_gate(CellArgs a, const P *__restrict__ q, SurGate g,
                                                           SurQueue qu)
{
    const Layout &L = a.L;
    const int r = blockIdx.x;
    const int j = L.bc + r % L.nj, k = L.bc + r / L.nj;
    const int i0 = L.bc + blockIdx.y * GATE_ROW + threadIdx.x;
    bool fluid[GATE_CPT], frozen[GATE_CPT];
    long long c[GATE_CPT];
    double T[GATE_CPT];
#pragma unroll
    for (int s = 0; s < GATE_CPT; s++) {
        const int i = i0 + s * GATE_THREADS;
        fluid[s] = i < L.ni + L.bc && !solid_cell(a, i, j);
        c[s] = L.at(min(i, L.ni + L.bc - 1), j, k);
    }
    float y[GATE_CPT];
#pragma unroll
    for (int s = 0; s < GATE_CPT; s++) {
        // T and the radicals of a cell are loaded together (the radicals of
        // hot cells are read and not needed)
        T[s] = 0.0;
        y[s] = 0.f;
        if (fluid[s]) {
            T[s] = a.T[c[s]];
            if (g.mask) {
#pragma unroll
                for (int v = 0; v < NS; v++)
                    if ((g.mask >> v) & 1u) y[s] += fmaxf((float)q[(PY + v) * L.fs + c[s]], 0.f);
            }
        }
    }
    __shared__ int wact[GATE_CPT][GATE_THREADS / 32], base_s, nfrz;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned ma[GATE_CPT];
    int nf = 0;
#pragma unroll
    for (int s = 0; s < GATE_CPT; s++) {
        frozen[s] = fluid[s] && T[s] < g.T_frozen && (!g.mask || y[s] <= g.y_max_f);
        ma[s] = __ballot_sync(0xffffffffu, fluid[s] && !frozen[s]);
        nf += __popc(__ballot_sync(0xffffffffu, frozen[s]));
        if (lane == 0) wact[s][w] = __popc(ma[s]);
    }
    if (threadIdx.x == 0) nfrz = 0;
    __syncthreads();
    if (lane == 0 && nf) atomicAdd(&nfrz, nf);
    if (threadIdx.x == 0) {
        // exclusive offsets, cell slot outer and warp inner: the x order
        int ta = 0;
        for (int s = 0; s < GATE_CPT; s++)
            for (int v = 0; v < GATE_THREADS / 32; v++) {
                const int n = wact[s][v];
                wact[s][v] = ta;
                ta += n;
            }
        base_s = ta ? atomicAdd(g.acount, ta) : 0;
    }
    __syncthreads();
    if (threadIdx.x == 0 && nfrz) atomicAdd(&a.st->sur_frozen, (unsigned long long)nfrz);
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int s = 0; s < GATE_CPT; s++)
        if ((ma[s] >> lane) & 1u) g.active[base_s + wact[s][w] + __popc(ma[s] & below)] = (int)c[s];
#pragma unroll
    for (int s = 0; s < GATE_CPT; s++) {
        const int i = i0 + s * GATE_THREADS;
        const long long idx = ((long long)(k - L.bc) * L.nj + (j - L.bc)) * L.ni + (i - L.bc);
        sur_push(qu, frozen[s] && gate_sample(idx, (unsigned)g.audit_stride),
                 (int)((unsigned)c[s] | SUR_FROZEN_AUDIT), T[s]);
    }
}

// SSP-RK2 stage 2 with the frozen-chemistry gate fused into it (tuning
// gate_fused): the stage update and decode of k_cell<M_RK_STAGE2>, then the
// gate's test on the T and radicals the decode just produced, each warp's
// active cells appended to the list in x order with one global atomic, and
// the hashed audit sample of frozen cells pushed to the fallback list -- the
// separate gate kernel's decisions and list (in another order), without
// reading T and the radicals back from memory.  Every lane reaches its
// warp's append (cell_body returns to this kernel for cells past the row or
// in the wedge).
template <class P, bool SPEC, int NB>
__global__ void __launch_bounds__(128, NB) k_rk2_gate(CellArgs a, P *__restrict__ q, SurGate g, SurQueue qu)
{
    CellGate gc{g.mask, false, 0, 0.0, 0.f};
    cell_body<P, M_RK_STAGE2, SPEC, true>(a, q, &gc);
    const Layout &L = a.L;
    const int i = L.bc + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = L.bc + blockIdx.y, k = L.bc + blockIdx.z;
    const bool frozen = gc.valid && gc.T < g.T_frozen && (!g.mask || gc.y <= g.y_max_f);
    const bool active = gc.valid && !frozen;
    // one list atomic per warp, no block barrier: a barrier would hold every
    // warp of the block for the slowest decode and the atomic's round trip
    const int lane = threadIdx.x & 31;
    const unsigned ma = __ballot_sync(0xffffffffu, active), mf = __ballot_sync(0xffffffffu, frozen);
    if (lane == 0 && mf) atomicAdd(&a.st->sur_frozen, (unsigned long long)__popc(mf));
    int base = 0;
    if (lane == 0 && ma) base = atomicAdd(g.acount, __popc(ma));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (active) g.active[base + __popc(ma & ((1u << lane) - 1u))] = (int)gc.c;
    const long long idx = ((long long)(k - L.bc) * L.nj + (j - L.bc)) * L.ni + (i - L.bc);
    sur_push(qu, frozen && gate_sample(idx, (unsigned)g.audit_stride), (int)((unsigned)gc.c | SUR_FROZEN_AUDIT),
             gc.T);
}

// Lists every fluid interior cell (the queued adaptive chemistry's work).
__global__ void __launch_bounds__(256) k_list_fluid(CellArgs a, SurQueue qu)
{
    const Layout &L = a.L;
    const int i = L.bc + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = L.bc + blockIdx.y;
    const int k = L.bc + blockIdx.z;
    if (i >= L.ni + L.bc) return;
    if (solid_cell(a, i, j)) return;
    sur_push(qu, true, (int)L.at(i, j, k), 0.0);
}

// The apply of the listed cells: one thread per list position, launched
// for the largest possible list (the length is on the device); network
// outputs by list position.
template <class P>
__global__ void __launch_bounds__(128, 7) k_sur_apply_list(SurApplyArgs s, P *__restrict__ q,
                                                           const int *__restrict__ list, const int *__restrict__ count)
{
    const Layout &L = s.a.L;
    const long long total = min((long long)*count, s.n);
    if ((long long)blockIdx.x * blockDim.x >= total) return;  // a whole block past the list
    __shared__ unsigned long long cnt[SUR_NFLAGS];
    const BlockCount<SUR_NFLAGS> bc{cnt};
    bc.init();
    const long long pos = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned flags = 0u;
    if (pos < total) {
        const int plane = L.NJ * L.px;
        const int c = list[pos];
        const int k = c / plane, r = c - k * plane;
        const int j = r / L.px, i = r - j * L.px;
        float o[SUR_NOUT];
#pragma unroll
        for (int v = 0; v < SUR_NOUT; v++) o[v] = s.out[v * s.n + pos];
        flags = sur_apply_cell<P, false, false>(s, q, i, j, k, o);  // listed cells are fluid
    }
    bc.add(flags);
    Status *st = s.a.st;
    unsigned long long *const dst[SUR_NFLAGS] = {&st->sur_cells,     &st->sur_fallback,  &st->sur_reject[0],
                                                 &st->sur_reject[1], &st->sur_reject[2], &st->sur_reject[3]};
    bc.flush(dst);
}

// The MLP kernel's source for the fused form: features from the flowfield
// (SurSrcField) and, instead of writing the outputs, the apply of each cell
// right after its output layer, so that the outputs never travel through
// HBM.  Same decisions as the network kernel followed by k_sur_apply; on the
// 33.5 M-cell ODW it takes 10.4 ms against 4.55 + 3.94 ms for the two
// kernels (the apply's memory latency has only the network kernel's 16
// warps per SM to hide behind, and the kernel spills), so it is off by
// default.
template <class P>
struct SurSrcFieldApply : SurSrcField<P> {
    SurApplyArgs ap;
    P *q;
    __device__ __forceinline__ void store(long long tile, int lane, long long, const float o[SUR_OUT]) const
    {
        const Layout &L = this->L;
        const int t = (int)tile;
        const int r = t / this->tpr;
        const int i = (t - r * this->tpr) * 128 + lane;
        sur_apply_cell<P>(ap, q, L.bc + i, L.bc + r % L.nj, L.bc + r / L.nj, o);
    }
};

// Persistent fallback queue, one listed cell per lane: a lane whose cell is
// done takes the next listed cell at once (the lanes of a warp that need one
// take them with one atomic on the global cursor), so a warp keeps stepping
// the substeps of cells with different substep counts instead of waiting for
// the slowest of a batch.  Each cell runs the FP64 adaptive split step the
// network was trained on (adapt_split_step with the flux update applied
// already: chem_increment, then the species update and a decode), one
// substep per pass.  The loop holds the substeps only: a finished cell's
// integrated species, T and counts go to its list slot, and
// k_sur_fallback_finish does the projection, update, decode and stores with
// one thread per slot -- run inside the loop, that work was executed by the
// warp in nearly every pass (some lane finishes a cell in most passes), and
// its code competed with the substep's for the instruction cache.
template <class P, bool SPEC>
__global__ void __launch_bounds__(128, 3) k_sur_fallback(CellArgs a, P *__restrict__ q, SurQueue qu)
{
    const int lane = threadIdx.x & 31;
    const int total = (int)min((long long)*qu.count, qu.cap);
    const long long fs = a.L.fs;
    const unsigned qk = a.quirks;
    const double dt = a.scal[0];
    const AdaptCfg cfg = a.acfg;
    const double hmin = dt / cfg.nmax;
    int slot = -1;  // list slot of the lane's cell; -1: needs one; >= total: none left
    double cs[NV];  // the integrator's copy of the cell's state
    double T = 0.0, Esub = 0.0, trem = 0.0;
    int k = 0, capped = 0, forced = 0;
    Decoded o;
    for (;;) {
        const bool need = slot < 0;
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(qu.count + 1, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                slot = base + __popc(m & ((1u << lane) - 1u));
                if (slot < total) {
                    const long long c = (long long)((unsigned)qu.list[slot] & (unsigned)SUR_CELL_MASK);
                    load_cs(a.cs, fs, c, cs);
                    // the decoded state (adapt_split_step without the flux
                    // update): the integrator runs at its energy from its T
                    double D = 0.0;
#pragma unroll
                    for (int s = 0; s < NS; s++) D += cs[s];
                    const double iD = 1.0 / D;
                    const double U = cs[NS] * iD, V = cs[NS + 1] * iD, W = cs[NS + 2] * iD;
                    Esub = (cs[NS + 3] - 0.5 * D * (U * U + V * V + W * W)) * iD;
                    T = a.T[c];
                    trem = dt;
                    k = 0;
                    capped = 0;
                    forced = 0;
                }
            }
        }
        if (__all_sync(0xffffffffu, slot >= total)) break;
        if (slot < total) {
            if (trem > 0.0 && k < cfg.nmax) adapt_substep<SPEC>(cs, T, Esub, qk, trem, k, hmin, cfg, o, capped, forced);
            if (!(trem > 0.0 && k < cfg.nmax)) {
#pragma unroll
                for (int sp = 0; sp < NS; sp++) qu.res[sp * qu.cap + slot] = cs[sp];
                qu.res[NS * qu.cap + slot] = T;
                qu.info[slot] = k | (capped ? SUR_CAPPED : 0) | (forced ? SUR_FORCED : 0);
                slot = -1;
            }
        }
    }
}

// The end of each fallback cell's split step, one thread per list slot:
// chem_increment's element projection of the integrated change, then
// adapt_split_step's species update and decode at the cell's density and
// energy, the stores, and the status counts (audits compared with the
// surrogate's temperature).  The same arithmetic as the end of
// adapt_split_step, on the state k_sur_fallback left in the slot.
constexpr int FALLBACK_FINISH_BLOCKS = 148 * 8;  // grid of k_sur_fallback_finish (grid-stride over the slots)

template <class P, bool SPEC>
__global__ void __launch_bounds__(128) k_sur_fallback_finish(CellArgs a, P *__restrict__ q, SurQueue qu)
{
    const int total = (int)min((long long)*qu.count, qu.cap);
    const long long fs = a.L.fs;
    const unsigned qk = a.quirks;
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < total; slot += gridDim.x * blockDim.x) {
        const unsigned ent = (unsigned)qu.list[slot];
        const bool audit = (ent & SUR_AUDIT) != 0, faudit = (ent & SUR_FROZEN_AUDIT) != 0;
        const long long c = (long long)(ent & (unsigned)SUR_CELL_MASK);
        double cs0[NV];
        load_cs(a.cs, fs, c, cs0);
        double D0 = 0.0, Dn = 0.0, cs[NS];
#pragma unroll
        for (int sp = 0; sp < NS; sp++) {
            cs[sp] = qu.res[sp * qu.cap + slot];
            D0 += cs0[sp];
            Dn += cs[sp];
        }
        const double Tc = qu.res[NS * qu.cap + slot];
        const int inf = qu.info[slot];
        // the energy the integrator ran at (as k_sur_fallback formed it)
        double Esub;
        {
            const double iD = 1.0 / D0;
            const double U = cs0[NS] * iD, V = cs0[NS + 1] * iD, W = cs0[NS + 2] * iD;
            Esub = (cs0[NS + 3] - 0.5 * D0 * (U * U + V * V + W * W)) * iD;
        }
        double Y0[NS], dY[NS];
#pragma unroll
        for (int sp = 0; sp < NS; sp++) {
            Y0[sp] = cs0[sp] / D0;
            dY[sp] = cs[sp] / Dn - Y0[sp];
        }
        elem_project(Y0, dY, a.proj_eps);
        const double iD = 1.0 / D0;
#pragma unroll
        for (int sp = 0; sp < NS; sp++) cs0[sp] = fmax(D0 * (cs0[sp] * iD + dY[sp]), 0.0);
        int cp = 0;
        Decoded o;
        decode(cs0, Tc, Esub, qk, o, cp);
        store_cs(a.cs, fs, c, cs0);
        a.T[c] = o.T;
        a.E[c] = o.E;
        store_prims<P>(o, q, fs, c);
        warp_sum(&a.st->substeps, (unsigned long long)(inf & (SUR_CAPPED - 1)));
        warp_count(&a.st->newton_capped, cp || (inf & SUR_CAPPED));
        if (inf & SUR_FORCED) atomicAdd(&a.st->substep_capped, 1);
        warp_count(&a.st->nonfinite, !(isfinite(o.D) && isfinite(o.T)));
        if (audit || faudit) {
            const double d = fabs(qu.audit[slot] - o.T);
            unsigned long long *mx = audit ? &a.st->audit_max_dT_bits : &a.st->frozen_audit_max_dT_bits;
            atomicAdd(audit ? &a.st->audit_cells : &a.st->frozen_audit_cells, 1ull);
            if (isfinite(d)) atomicMax(mx, (unsigned long long)__double_as_longlong(d));
            else atomicMax(mx, 0x7ff0000000000000ull);
        }
    }
}

}  // namespace eu3d
