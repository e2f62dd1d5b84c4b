// Ghost-cell fills and the CFL time step.
//
// Reference: Flowfield::FieldBoundary_3dRSBI (src/Flowfield.cpp:559-773),
// FieldBoundary_3dODM (:378-558), Flowfield::CFLcondition (:242-272).
// The faces are filled in the reference's order -- x, then y over every i
// (x ghosts included), then z over every i, j -- one launch per direction so
// that each launch reads only cells the previous launches have finished.
#pragma once

#include "common.cuh"

namespace eu3d {

struct GhostArgs {
    Layout L;
    unsigned quirks;
    double *T, *E;
    const double *inflow;  // ODM planes: U V W P D T H E G, then NS species planes, each nj*nk
    int kind;
};

// Every fill loads all the values it copies before its first store.  The
// destination of a fill is never a source of the same launch (ghost cells
// take interior cells; the wedge band's solid cells take fluid ones), so the
// order changes nothing but the timing: the compiler, which cannot prove
// that the stores miss the later loads, would otherwise issue each load only
// after the store before it, one memory round trip per field.
template <class P>
__device__ __forceinline__ void ghost_load(const GhostArgs &a, const P *q, long long s, P v[NPRIM], double &T,
                                           double &E)
{
    const long long fs = a.L.fs;
#pragma unroll
    for (int f = 0; f < NPRIM; f++) v[f] = q[f * fs + s];
    T = a.T[s];
    E = a.E[s];
}

template <class P>
__device__ __forceinline__ void ghost_store(const GhostArgs &a, P *q, long long d, const P v[NPRIM], double T,
                                            double E)
{
    const long long fs = a.L.fs;
#pragma unroll
    for (int f = 0; f < NPRIM; f++) q[f * fs + d] = v[f];
    a.T[d] = T;
    a.E[d] = E;
}

template <class P>
__device__ __forceinline__ void ghost_copy(const GhostArgs &a, P *q, long long d, long long s)
{
    P v[NPRIM];
    double T, E;
    ghost_load(a, q, s, v, T, E);
    ghost_store(a, q, d, v, T, E);
}

// mirror with the wall-side thermodynamic recompute of the reflective faces
// (src/Flowfield.cpp:409-436 pattern): D from P/(T Rgas), H, E, Gamma from T
template <class P>
__device__ __forceinline__ void ghost_wall(const GhostArgs &a, P *q, long long d, long long s, bool flipv, bool flipw)
{
    const long long fs = a.L.fs;
    const P u = q[PU * fs + s], v = q[PV * fs + s], w = q[PW * fs + s];
    const P Pp = q[PP * fs + s];
    P ys[NS];
#pragma unroll
    for (int sp = 0; sp < NS; sp++) ys[sp] = q[(PY + sp) * fs + s];
    const double T = a.T[s];
    q[PU * fs + d] = u;
    q[PV * fs + d] = flipv ? -v : v;
    q[PW * fs + d] = flipw ? -w : w;
    q[PP * fs + d] = Pp;
    a.T[d] = T;
    const TPow p = tpow(T, a.quirks);
    double Y[NS], rg = 0.0, cp = 0.0, h = 0.0, e = 0.0;
#pragma unroll
    for (int sp = 0; sp < NS; sp++) {
        Y[sp] = (double)ys[sp];
        q[(PY + sp) * fs + d] = ys[sp];
    }
#pragma unroll
    for (int sp = 0; sp < NS; sp++) {
        const double cpi = cM.ri[sp] * cp_r(sp, p);
        const double hi = cM.ri[sp] * h_r(sp, p);
        const double ei = hi - cM.ri[sp] * T;
        rg += Y[sp] * cM.ri[sp];
        cp += cpi * Y[sp];
        h += Y[sp] * hi;
        e += Y[sp] * ei;
    }
    const double Rgas = rg * 1000;
    const double Cp = cp * 1000;
    q[PD * fs + d] = (P)((double)Pp / (T * Rgas));
    q[PH * fs + d] = (P)(h * 1000);
    a.E[d] = e * 1000;
    q[PG * fs + d] = (P)(Cp / (Cp - Rgas));
}

// x faces: i in [0, bc) and [ni+bc, ni+2bc), j, k interior
template <class P>
__global__ void k_ghost_x(GhostArgs a, P *q)
{
    const Layout &L = a.L;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = 2 * L.bc;
    const int n = g * L.nj * L.nk;
    if (t >= n) return;
    // a warp covers the bc ghost cells of consecutive rows j on one face:
    // neighbouring lanes write neighbouring cells, the face is uniform across
    // the warp, and the inflow planes (j fastest on the device) are read in order
    const int gi = t % L.bc, j = L.bc + (t / L.bc) % L.nj;
    const bool lower = (t / (L.bc * L.nj)) % 2 == 0;
    const int k = L.bc + t / (g * L.nj);
    const int i = lower ? gi : L.ni + L.bc + gi;
    const long long d = L.at(i, j, k);
    if (a.kind == EU3D_BC_RSBI) {
        const int si = lower ? 2 * L.bc - 1 - i : 2 * (L.ni + L.bc) - 1 - i;
        ghost_copy(a, q, d, L.at(si, j, k));
    } else if (a.kind == EU3D_BC_TRANSMISSIVE) {
        const int si = lower ? L.bc : L.ni + L.bc - 1;
        ghost_copy(a, q, d, L.at(si, j, k));
    } else if (a.kind == EU3D_BC_ODM) {
        if (lower) {
            const long long p = (long long)(k - L.bc) * L.nj + (j - L.bc), pl = (long long)L.nj * L.nk;
            const long long fs = L.fs;
            // the inflow values are all loaded before the first store
            double in[9 + NS];
#pragma unroll
            for (int f = 0; f < 9 + NS; f++) in[f] = a.inflow[f * pl + p];
            q[PU * fs + d] = (P)in[0];
            q[PV * fs + d] = (P)in[1];
            q[PW * fs + d] = (P)in[2];
            q[PP * fs + d] = (P)in[3];
            q[PD * fs + d] = (P)in[4];
            a.T[d] = in[5];
            q[PH * fs + d] = (P)in[6];
            a.E[d] = in[7];
            q[PG * fs + d] = (P)in[8];
#pragma unroll
            for (int s = 0; s < NS; s++) q[(PY + s) * fs + d] = (P)in[9 + s];
        } else {
            ghost_wall(a, q, d, L.at(2 * (L.ni + L.bc) - 1 - i, j, k), false, false);
        }
    }
}

// y faces: every i, j in the ghost rows, k interior
template <class P>
__global__ void k_ghost_y(GhostArgs a, P *q)
{
    const Layout &L = a.L;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = 2 * L.bc;
    const int n = L.NI * g * L.nk;
    if (t >= n) return;
    const int i = t % L.NI, gj = (t / L.NI) % g, k = L.bc + t / (L.NI * g);
    const bool lower = gj < L.bc;
    const int j = lower ? gj : L.nj + L.bc + (gj - L.bc);
    const long long d = L.at(i, j, k);
    const int sj = lower ? 2 * L.bc - 1 - j : 2 * (L.nj + L.bc) - 1 - j;
    if (a.kind == EU3D_BC_RSBI) {
        if (lower)
            ghost_wall(a, q, d, L.at(i, sj, k), false, false);
        else
            ghost_copy(a, q, d, L.at(i, sj, k));
    } else if (a.kind == EU3D_BC_TRANSMISSIVE) {
        ghost_copy(a, q, d, L.at(i, sj, k));
    } else if (a.kind == EU3D_BC_ODM) {
        if (lower)
            ghost_wall(a, q, d, L.at(i, sj, k), true, false);
        else
            ghost_copy(a, q, d, L.at(i, sj, k));
    }
}

// z faces: every i, j, k in the ghost planes
template <class P>
__global__ void k_ghost_z(GhostArgs a, P *q)
{
    const Layout &L = a.L;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = 2 * L.bc;
    const int n = L.NI * L.NJ * g;
    if (t >= n) return;
    const int i = t % L.NI, j = (t / L.NI) % L.NJ, gk = t / (L.NI * L.NJ);
    const bool lower = gk < L.bc;
    const int k = lower ? gk : L.nk + L.bc + (gk - L.bc);
    const long long d = L.at(i, j, k);
    const int sk = lower ? 2 * L.bc - 1 - k : 2 * (L.nk + L.bc) - 1 - k;
    if (a.kind == EU3D_BC_ODM)
        ghost_wall(a, q, d, L.at(i, j, sk), false, true);
    else
        ghost_copy(a, q, d, L.at(i, j, sk));
}

// Wedge immersed boundary (new): solid cells take the state of the fluid
// cell nearest to their mirror image across the wedge surface, with the
// velocity reflected about the surface.  Only the band of solid cells that
// flux stencils reach is filled (fluid within two cells along x or y);
// band[n] = (i, j, si, sj): the solid column and its mirror source, the same
// for every k, listed on the host when the wedge is set.
template <class P>
__global__ void k_wedge_band(GhostArgs a, P *q, const int4 *__restrict__ band, int nband, double nx, double ny)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (n >= nband) return;
    const int4 b = band[n];
    const Layout &L = a.L;
    const long long d = L.at(b.x, b.y, k), s = L.at(b.z, b.w, k);
    P w[NPRIM];
    double T, E;
    ghost_load(a, q, s, w, T, E);
    const double u = (double)w[PU], v = (double)w[PV];
    const double un = u * nx + v * ny;
    w[PU] = (P)(u - 2.0 * un * nx);
    w[PV] = (P)(v - 2.0 * un * ny);
    ghost_store(a, q, d, w, T, E);
}

// CFL: block minima of min(dx/(|U|+C), dy/(|V|+C)[, dz/(|W|+C)]) over the
// interior (solid wedge cells excluded), C = sqrt(Gamma P / D) as the decode
// defines it.
// CFLcondition (src/Flowfield.cpp:242-272) as block maxima: because IEEE
// division is monotone in the divisor, the smallest dx / (|U| + C) over the
// cells is dx over the largest |U| + C, bit for bit; so each block keeps the
// largest |U| + C, |V| + C, |W| + C of its cells and k_cfl_final divides
// once.  A cell whose x time is NaN is skipped, as the reference's
// comparisons skip it; NaN y or z times drop out of fmax as they drop out of
// the reference's min.  One warp walks one (j, k) row of interior cells.
// FP64 primitives: the reference's FP64 arithmetic (C = sqrt(gamma p / rho),
// src/Flowfield.cpp:1281).  FP32 primitives: the same speeds in FP32 (the
// inputs carry FP32 precision already), widened exactly for the maxima.
__device__ __forceinline__ void cfl_speeds(double D, double Pp, double G, double U, double V, double W, double &ax,
                                           double &ay, double &az)
{
    const double C = sqrt(G * Pp / D);
    ax = fabs(U) + C;
    ay = fabs(V) + C;
    az = fabs(W) + C;
}

__device__ __forceinline__ void cfl_speeds(float D, float Pp, float G, float U, float V, float W, double &ax,
                                           double &ay, double &az)
{
    const float C = sqrtf(__fdividef(__fmul_rn(G, Pp), D));
    ax = (double)__fadd_rn(fabsf(U), C);
    ay = (double)__fadd_rn(fabsf(V), C);
    az = (double)__fadd_rn(fabsf(W), C);
}

constexpr int CFL_U = 4;  // cells a lane has in flight in k_cfl_partial

template <class P>
__global__ void k_cfl_partial(Layout L, const P *__restrict__ q, int use_z, const double *__restrict__ xn,
                              const double *__restrict__ yn, double x0, double y0, double tn, int wedge_on,
                              double *__restrict__ partial)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int rows = L.nj * L.nk;
    const long long fs = L.fs;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int r = blockIdx.x * wpb + wid; r < rows; r += gridDim.x * wpb) {
        const int j = L.bc + r % L.nj, k = L.bc + r / L.nj;
        const double y = yn[j];
        const long long base = L.at(0, j, k);
        // CFL_U cells a lane at a time, all their loads issued before the
        // first speed is formed (the maxima do not depend on the order)
        for (int i0 = L.bc + lane; i0 < L.ni + L.bc; i0 += 32 * CFL_U) {
            bool ok[CFL_U];
            P vd[CFL_U], vp[CFL_U], vg[CFL_U], vu[CFL_U], vv[CFL_U], vw[CFL_U];
#pragma unroll
            for (int u = 0; u < CFL_U; u++) {
                const int i = i0 + 32 * u;
                ok[u] = i < L.ni + L.bc;
                if (ok[u] && wedge_on) {
                    const double x = xn[i];
                    ok[u] = !(x > x0 && (y - y0) < (x - x0) * tn);
                }
                if (ok[u]) {
                    const long long c = base + i;
                    vd[u] = q[PD * fs + c];
                    vp[u] = q[PP * fs + c];
                    vg[u] = q[PG * fs + c];
                    vu[u] = q[PU * fs + c];
                    vv[u] = q[PV * fs + c];
                    vw[u] = q[PW * fs + c];
                }
            }
#pragma unroll
            for (int u = 0; u < CFL_U; u++) {
                if (!ok[u]) continue;
                double ax, ay, az;
                cfl_speeds(vd[u], vp[u], vg[u], vu[u], vv[u], vw[u], ax, ay, az);
                if (isnan(ax)) continue;
                sx = fmax(sx, ax);
                sy = fmax(sy, ay);
                if (use_z) sz = fmax(sz, az);
            }
        }
    }
    __shared__ double sm[3][32];
    for (int o = 16; o > 0; o >>= 1) {
        sx = fmax(sx, __shfl_down_sync(0xffffffffu, sx, o));
        sy = fmax(sy, __shfl_down_sync(0xffffffffu, sy, o));
        sz = fmax(sz, __shfl_down_sync(0xffffffffu, sz, o));
    }
    if (lane == 0) {
        sm[0][wid] = sx;
        sm[1][wid] = sy;
        sm[2][wid] = sz;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        sx = lane < wpb ? sm[0][lane] : 0.0;
        sy = lane < wpb ? sm[1][lane] : 0.0;
        sz = lane < wpb ? sm[2][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            sx = fmax(sx, __shfl_down_sync(0xffffffffu, sx, o));
            sy = fmax(sy, __shfl_down_sync(0xffffffffu, sy, o));
            sz = fmax(sz, __shfl_down_sync(0xffffffffu, sz, o));
        }
        if (lane == 0) {
            partial[3 * blockIdx.x + 0] = sx;
            partial[3 * blockIdx.x + 1] = sy;
            partial[3 * blockIdx.x + 2] = sz;
        }
    }
}

// advance: time += dt as well (one rank); 0 leaves time for after the
// all-ranks minimum of dt (k_advance_time).  dt_conv starts at 1e10 as in the
// reference, so a domain without fluid cells gets cfl * 1e10.
__global__ void k_cfl_final(const double *partial, int nparts, double dx, double dy, double dz, int use_z, double cfl,
                            double final_time, double *scal, int advance)
{
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int t = threadIdx.x; t < nparts; t += blockDim.x) {
        sx = fmax(sx, partial[3 * t + 0]);
        sy = fmax(sy, partial[3 * t + 1]);
        sz = fmax(sz, partial[3 * t + 2]);
    }
    __shared__ double sm[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        sx = fmax(sx, __shfl_down_sync(0xffffffffu, sx, o));
        sy = fmax(sy, __shfl_down_sync(0xffffffffu, sy, o));
        sz = fmax(sz, __shfl_down_sync(0xffffffffu, sz, o));
    }
    if (lane == 0) {
        sm[0][wid] = sx;
        sm[1][wid] = sy;
        sm[2][wid] = sz;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        sx = lane < nw ? sm[0][lane] : 0.0;
        sy = lane < nw ? sm[1][lane] : 0.0;
        sz = lane < nw ? sm[2][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            sx = fmax(sx, __shfl_down_sync(0xffffffffu, sx, o));
            sy = fmax(sy, __shfl_down_sync(0xffffffffu, sy, o));
            sz = fmax(sz, __shfl_down_sync(0xffffffffu, sz, o));
        }
        if (threadIdx.x == 0) {
            // the smallest of dx/sx, dy/sy (and dz/sz); a zero speed gives an
            // infinite time, which the reference's 1e10 start caps
            double m = 1e10;
            const double a = dx / sx, b = dy / sy;
            if (a < m) m = a;
            if (b < m) m = b;
            if (use_z) {
                const double z = dz / sz;
                if (z < m) m = z;
            }
            double dt = cfl * m;
            if (scal[1] + dt > final_time) dt = final_time - scal[1];
            scal[0] = dt;
            if (advance) scal[1] += dt;
        }
    }
}

__global__ void k_advance_time(double *scal) { scal[1] += scal[0]; }

// x-slab halo: two x planes of every field the ghost fills write (NPRIM
// primitives, T, E) over the whole y-z extent, ghost rows included, to or
// from a contiguous buffer laid out [field][plane][k][j].  The primitives
// come first in P, then T and E in FP64.  src/Flowfield.cpp:775-1083
// (Mpi_Boundary) exchanges the same planes field by field.
template <class P>
__global__ void k_halo(Layout L, P *__restrict__ q, double *__restrict__ T, double *__restrict__ E,
                       unsigned char *__restrict__ buf, int i0, int pack)
{
    const long long plane = (long long)L.NJ * L.NK;
    const long long n = 2 * plane;
    P *bp = reinterpret_cast<P *>(buf);
    double *bd = reinterpret_cast<double *>(buf + (size_t)NPRIM * n * sizeof(P));
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(t / plane);
        const long long r = t - p * plane;
        const int j = (int)(r % L.NJ), k = (int)(r / L.NJ);
        const long long c = L.at(i0 + p, j, k);
        if (pack) {
#pragma unroll
            for (int f = 0; f < NPRIM; f++) bp[f * n + t] = q[f * L.fs + c];
            bd[t] = T[c];
            bd[n + t] = E[c];
        } else {
#pragma unroll
            for (int f = 0; f < NPRIM; f++) q[f * L.fs + c] = bp[f * n + t];
            T[c] = bd[t];
            E[c] = bd[n + t];
        }
    }
}

}  // namespace eu3d
