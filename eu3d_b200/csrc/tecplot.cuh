// The reference's result file, Euler::Output (src/Euler.cpp:792-973): one
// rank's Tecplot block file.  Three header lines, then 18 blocks over the
// interior cells in k-outer, j, i-inner order -- X, Y, Z (node coordinates),
// T, D, P, U, V, Ma, Y1..Y7 (the first seven species), L (substep counts),
// WaitTime -- one value per line, printed as std::ostream prints by default
// (%.6g for doubles, %d for the counts).
//
// From the device: one gather kernel puts the 13 FP64 columns and the counts
// of the interior cells into one buffer, one copy brings it to pinned host
// memory, and host threads format it -- on the calling thread or on a
// background thread while the GPU steps on (eu3d_write_wait joins it).
#pragma once

#include <algorithm>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace eu3d {

constexpr int TP_COLS = 13;  // T D P U V Ma Y1..Y7 (FP64); the counts L apart

// Interior cells in output order: t = ((k nj) + j) ni + i.  Ma from the
// primitives as Update_after_CS computes it (src/Flowfield.cpp:1281-1282),
// with IEEE operations only, as the reference's CPU arithmetic.
template <class P>
__global__ void k_tecplot_gather(Layout L, const P *__restrict__ q, const double *__restrict__ T,
                                 const int *__restrict__ nchem, double *__restrict__ cols, int *__restrict__ lcol)
{
    const long long n = L.interior_cells();
    const long long fs = L.fs;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = L.bc + (int)(t % L.ni);
        const long long r = t / L.ni;
        const int j = L.bc + (int)(r % L.nj), k = L.bc + (int)(r / L.nj);
        const long long c = L.at(i, j, k);
        const double D = (double)q[PD * fs + c], U = (double)q[PU * fs + c], V = (double)q[PV * fs + c];
        const double W = (double)q[PW * fs + c], Pp = (double)q[PP * fs + c], G = (double)q[PG * fs + c];
        const double C = sqrt(__ddiv_rn(__dmul_rn(G, Pp), D));
        const double u2 = __dadd_rn(__dadd_rn(__dmul_rn(U, U), __dmul_rn(V, V)), __dmul_rn(W, W));
        cols[0 * n + t] = T[c];
        cols[1 * n + t] = D;
        cols[2 * n + t] = Pp;
        cols[3 * n + t] = U;
        cols[4 * n + t] = V;
        cols[5 * n + t] = __ddiv_rn(sqrt(u2), C);
#pragma unroll
        for (int s = 0; s < 7; s++) cols[(6 + s) * n + t] = (double)q[(PY + s) * fs + c];
        lcol[t] = nchem[c];
    }
}

namespace tecplot {

// Writes the block file.  xnode/ynode/znode: ghosted node coordinates (the
// mesh's arrays); cols: TP_COLS x n FP64 values and lcol: n counts, both in
// output order.  Returns an empty string or the error.
inline std::string write(const char *path, int ni, int nj, int nk, int bc, const double *xnode, const double *ynode,
                         const double *znode, const double *cols, const int *lcol, double wait_time)
{
    const long long n = (long long)ni * nj * nk;
    const long long total = 18 * n;  // values after the header
    FILE *f = fopen(path, "wb");
    if (!f) return std::string("cannot open ") + path;
    char head[256];
    const int hl = snprintf(head, sizeof head,
                            "Variables = X,Y,Z,T,D,P,U,V,Ma,Y1,Y2,Y3,Y4,Y5,Y6,Y7,L,WaitTime\n"
                            "ZONE I=%d\tJ=%d\tK=%d\ndatapacking=block\n",
                            ni, nj, nk);
    bool ok = fwrite(head, 1, (size_t)hl, f) == (size_t)hl;
    auto value = [&](long long v, char *buf) -> int {
        const long long col = v / n, t = v - col * n;
        if (col == 16) return snprintf(buf, 32, "%d\n", lcol[t]);
        double x;
        if (col == 0)
            x = xnode[bc + (int)(t % ni)];
        else if (col == 1)
            x = ynode[bc + (int)((t / ni) % nj)];
        else if (col == 2)
            x = znode[bc + (int)(t / ((long long)ni * nj))];
        else if (col == 17)
            x = wait_time;
        else
            x = cols[(col - 3) * n + t];
        return snprintf(buf, 32, "%.6g\n", x);
    };
    // format in chunks, each chunk split over the host threads
    const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const long long chunk = 1LL << 24;
    std::vector<std::string> part(nt);
    for (long long a = 0; a < total && ok; a += chunk) {
        const long long b = std::min(total, a + chunk);
        std::vector<std::thread> th;
        for (int p = 0; p < nt; p++) {
            th.emplace_back([&, p] {
                const long long lo = a + (b - a) * p / nt, hi = a + (b - a) * (p + 1) / nt;
                std::string &s = part[p];
                s.clear();
                s.reserve((size_t)(hi - lo) * 12);
                char buf[32];
                for (long long v = lo; v < hi; v++) s.append(buf, (size_t)value(v, buf));
            });
        }
        for (auto &t : th) t.join();
        for (int p = 0; p < nt && ok; p++) ok = fwrite(part[p].data(), 1, part[p].size(), f) == part[p].size();
    }
    if (fclose(f) != 0) ok = false;
    return ok ? std::string() : std::string("write failed: ") + path;
}

}  // namespace tecplot
}  // namespace eu3d
