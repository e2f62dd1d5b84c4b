// Dynamic load balancing of the adaptive trapezoid across ranks: the
// reference's DynamicLoadBalancer (src/LoadBalance.cpp:8-159) and its use in
// Euler::Trapezoid type 1 (src/Euler.cpp:380-700), on device buffers.
//
// After the prediction (k_cell<M_TRAP1_PREDICT>) a cell's chemistry is
// defined by CS, T and its substep count alone (trap1_cell), so a cell can
// be integrated on any rank and sent back bit for bit.  A rank's load is the
// sum of the predicted substep counts of its fluid cells.  The planner pairs
// overloaded with underloaded ranks (the reference's heap pairing); a sender
// gives away whole rows (j, k) of its slab, from the first row on, each
// transfer taking consecutive rows while their load fits its amount (the
// reference picks single cells first-fit).  Packets are field-major:
//   out  (owner -> guest): CS[NV], T, count            DLB_OUT fields per cell
//   back (guest -> owner): CS[NV], T, E, prims[NPRIM], count   DLB_BACK fields
// with a count of -1 marking a solid (immersed-wedge) cell that is carried
// but not integrated.
#pragma once

#include <algorithm>
#include <queue>
#include <utility>
#include <vector>

#include "cell.cuh"
#include "surrogate.cuh"

namespace eu3d {

constexpr int DLB_OUT = NV + 2;
constexpr int DLB_BACK = NV + 3 + NPRIM;
constexpr int DLB_MAXSEG = 64;  // transfers per rank and direction

// Row r = (k - bc) nj + (j - bc) of the interior; pack p of a sender holds rows
// [row[p], row[p + 1]), its field f of row-local cell s at
// buf[off[p] + f * cells(p) + s].
struct DlbSegs {
    int n;
    long long row[DLB_MAXSEG + 1];
    long long off[DLB_MAXSEG];
};

// guest-side segments: segment s holds cells [first[s], first[s + 1]) of the
// guest store at in/out offsets off[s]
struct DlbGuestSegs {
    int n;
    long long first[DLB_MAXSEG + 1];
    long long off_in[DLB_MAXSEG], off_out[DLB_MAXSEG];
};

__device__ __forceinline__ int dlb_seg(const long long *bounds, int n, long long v)
{
    int p = 0;
    while (p + 1 < n && v >= bounds[p + 1]) p++;
    return p;
}

// Substep counts of the fluid cells summed per interior row (one warp a row).
__global__ void k_dlb_rowload(CellArgs a, long long *__restrict__ rowload)
{
    const Layout &L = a.L;
    const long long nrows = (long long)L.nj * L.nk;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * blockDim.x / 32;
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32; r < nrows; r += warps) {
        const int j = L.bc + (int)(r % L.nj), k = L.bc + (int)(r / L.nj);
        long long s = 0;
        for (int i = L.bc + lane; i < L.ni + L.bc; i += 32)
            if (!solid_cell(a, i, j)) s += a.nchem[L.at(i, j, k)];
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) rowload[r] = s;
    }
}

// The owner's packets: rows [sg.row[0], sg.row[n]) into their segments; the
// fluid cells leave the work-queue bin counts that the prediction made.
__global__ void k_dlb_pack(CellArgs a, DlbSegs sg, double *__restrict__ buf, int *__restrict__ qbins)
{
    const Layout &L = a.L;
    const long long first = sg.row[0] * L.ni, total = (sg.row[sg.n] - sg.row[0]) * L.ni;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = first + t, r = g / L.ni;
        const int i = L.bc + (int)(g % L.ni), j = L.bc + (int)(r % L.nj), k = L.bc + (int)(r / L.nj);
        const int p = dlb_seg(sg.row, sg.n, r);
        const long long cells = (sg.row[p + 1] - sg.row[p]) * L.ni, s = g - sg.row[p] * L.ni;
        double *o = buf + sg.off[p] + s;
        const long long c = L.at(i, j, k), fs = L.fs;
        const bool solid = solid_cell(a, i, j);
#pragma unroll
        for (int v = 0; v < NV; v++) o[v * cells] = a.cs[v * fs + c];
        o[NV * cells] = a.T[c];
        const int n = solid ? -1 : a.nchem[c];
        o[(NV + 1) * cells] = (double)n;
        if (!solid) atomicSub(qbins + nchem_bin(n), 1);
    }
}

// Received cells into the guest store (field stride gcap), and their bins.
__global__ void k_dlb_guest_in(DlbGuestSegs sg, const double *__restrict__ in, long long gcap, double *__restrict__ cs,
                               double *__restrict__ T, int *__restrict__ nchem, int *__restrict__ bins)
{
    const long long total = sg.first[sg.n];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int p = dlb_seg(sg.first, sg.n, g);
        const long long cells = sg.first[p + 1] - sg.first[p], s = g - sg.first[p];
        const double *o = in + sg.off_in[p] + s;
#pragma unroll
        for (int v = 0; v < NV; v++) cs[v * gcap + g] = o[v * cells];
        T[g] = o[NV * cells];
        const int n = (int)o[(NV + 1) * cells];
        nchem[g] = n;
        if (n >= 0) atomicAdd(bins + nchem_bin(n), 1);
    }
}

// Lists the fluid guest cells in their bins (the queue's scatter for the store).
__global__ void k_dlb_guest_list(const int *__restrict__ nchem, long long total, ChemQueue qu)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int n = nchem[g];
        if (n < 0) continue;
        const int b = nchem_bin(n);
        const int slot = atomicAdd(qu.bins + 2 * QBINS + b, 1);
        qu.list[qu.bins[QBINS + b] + slot] = (int)g;
    }
}

// The integrated guest cells into the return packets.
template <class P>
__global__ void k_dlb_guest_out(DlbGuestSegs sg, long long gcap, const double *__restrict__ cs,
                                const double *__restrict__ T, const double *__restrict__ E, const P *__restrict__ q,
                                const int *__restrict__ nchem, double *__restrict__ out)
{
    const long long total = sg.first[sg.n];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int p = dlb_seg(sg.first, sg.n, g);
        const long long cells = sg.first[p + 1] - sg.first[p], s = g - sg.first[p];
        double *o = out + sg.off_out[p] + s;
#pragma unroll
        for (int v = 0; v < NV; v++) o[v * cells] = cs[v * gcap + g];
        o[NV * cells] = T[g];
        o[(NV + 1) * cells] = E[g];
#pragma unroll
        for (int f = 0; f < NPRIM; f++) o[(NV + 2 + f) * cells] = (double)q[f * gcap + g];
        o[(NV + 2 + NPRIM) * cells] = (double)nchem[g];
    }
}

// The returned cells back into the owner's fields (fluid cells only).
template <class P>
__global__ void k_dlb_unpack(CellArgs a, DlbSegs sg, const double *__restrict__ back, P *__restrict__ q)
{
    const Layout &L = a.L;
    const long long first = sg.row[0] * L.ni, total = (sg.row[sg.n] - sg.row[0]) * L.ni;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = first + t, r = g / L.ni;
        const int i = L.bc + (int)(g % L.ni), j = L.bc + (int)(r % L.nj), k = L.bc + (int)(r / L.nj);
        if (solid_cell(a, i, j)) continue;
        const int p = dlb_seg(sg.row, sg.n, r);
        const long long cells = (sg.row[p + 1] - sg.row[p]) * L.ni, s = g - sg.row[p] * L.ni;
        const double *o = back + sg.off[p] + s;
        const long long c = L.at(i, j, k), fs = L.fs;
#pragma unroll
        for (int v = 0; v < NV; v++) a.cs[v * fs + c] = o[v * cells];
        a.T[c] = o[NV * cells];
        a.E[c] = o[(NV + 1) * cells];
#pragma unroll
        for (int f = 0; f < NPRIM; f++) q[f * fs + c] = (P)o[(NV + 2 + f) * cells];
        a.nchem[c] = (int)o[(NV + 2 + NPRIM) * cells];
    }
}

// ---------------------------------------------------------------------------
// Load balancing of the learned chemistry's FP64 fallback (new).  The sender
// gives away the last list slots: segment p of the transfers holds slots
// keep + [first[p], first[p + 1]).  Packets, field-major per segment:
//   out  (owner -> guest): CS[NV], T, audit T, list flags     SDLB_OUT fields
//   back (guest -> owner): CS[NV], T, E, prims[NPRIM]          SDLB_BACK fields
constexpr int SDLB_OUT = NV + 3;
constexpr int SDLB_BACK = NV + 2 + NPRIM;

__global__ void k_sdlb_pack(CellArgs a, SurQueue qu, DlbGuestSegs sg, long long keep, double *__restrict__ buf)
{
    const long long total = sg.first[sg.n], fs = a.L.fs;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int p = dlb_seg(sg.first, sg.n, g);
        const long long cells = sg.first[p + 1] - sg.first[p], s = g - sg.first[p];
        const long long slot = keep + g;
        const unsigned ent = (unsigned)qu.list[slot];
        const long long c = (long long)(ent & (unsigned)SUR_CELL_MASK);
        double *o = buf + sg.off_in[p] + s;
#pragma unroll
        for (int v = 0; v < NV; v++) o[v * cells] = a.cs[v * fs + c];
        o[NV * cells] = a.T[c];
        o[(NV + 1) * cells] = qu.audit[slot];
        o[(NV + 2) * cells] = (double)(ent >> 30);
    }
}

// the owner keeps list slots [0, keep) for its own fallback work
__global__ void k_sdlb_keep(int *__restrict__ count, int keep)
{
    count[0] = keep;
    count[1] = 0;
}

// received cells into the guest store (field stride gcap) and the guest's
// fallback list (entry g with the sender's flags)
__global__ void k_sdlb_guest_in(DlbGuestSegs sg, const double *__restrict__ in, long long gcap, double *__restrict__ cs,
                                double *__restrict__ T, double *__restrict__ audit, int *__restrict__ list)
{
    const long long total = sg.first[sg.n];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int p = dlb_seg(sg.first, sg.n, g);
        const long long cells = sg.first[p + 1] - sg.first[p], s = g - sg.first[p];
        const double *o = in + sg.off_in[p] + s;
#pragma unroll
        for (int v = 0; v < NV; v++) cs[v * gcap + g] = o[v * cells];
        T[g] = o[NV * cells];
        audit[g] = o[(NV + 1) * cells];
        list[g] = (int)((unsigned)g | ((unsigned)o[(NV + 2) * cells] << 30));
    }
}

// the integrated guest cells into the return packets
template <class P>
__global__ void k_sdlb_guest_out(DlbGuestSegs sg, long long gcap, const double *__restrict__ cs,
                                 const double *__restrict__ T, const double *__restrict__ E, const P *__restrict__ q,
                                 double *__restrict__ out)
{
    const long long total = sg.first[sg.n];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int p = dlb_seg(sg.first, sg.n, g);
        const long long cells = sg.first[p + 1] - sg.first[p], s = g - sg.first[p];
        double *o = out + sg.off_out[p] + s;
#pragma unroll
        for (int v = 0; v < NV; v++) o[v * cells] = cs[v * gcap + g];
        o[NV * cells] = T[g];
        o[(NV + 1) * cells] = E[g];
#pragma unroll
        for (int f = 0; f < NPRIM; f++) o[(NV + 2 + f) * cells] = (double)q[f * gcap + g];
    }
}

// the returned cells back into the owner's fields
template <class P>
__global__ void k_sdlb_unpack(CellArgs a, SurQueue qu, DlbGuestSegs sg, long long keep, const double *__restrict__ back,
                              P *__restrict__ q)
{
    const long long total = sg.first[sg.n], fs = a.L.fs;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int p = dlb_seg(sg.first, sg.n, g);
        const long long cells = sg.first[p + 1] - sg.first[p], s = g - sg.first[p];
        const long long c = (long long)((unsigned)qu.list[keep + g] & (unsigned)SUR_CELL_MASK);
        const double *o = back + sg.off_out[p] + s;
#pragma unroll
        for (int v = 0; v < NV; v++) a.cs[v * fs + c] = o[v * cells];
        a.T[c] = o[NV * cells];
        a.E[c] = o[(NV + 1) * cells];
#pragma unroll
        for (int f = 0; f < NPRIM; f++) q[f * fs + c] = (P)o[(NV + 2 + f) * cells];
    }
}

namespace dlb {

// DynamicLoadBalancer::DLBPriorityQueue (src/LoadBalance.cpp:8-59): the
// integer mean of the loads; ranks at or above it in one max-heap of
// (load, rank), the others in a second max-heap of (load, rank) -- the
// reference's "minHeap" is a std::priority_queue as well, so the
// underloaded rank closest to the mean is filled first.  Each sender, most
// loaded first, passes min(excess, room) to receivers until its excess is
// gone; a receiver still under the mean goes back into its heap.
inline void plan(const long long *loads, int n, std::vector<int> &snd, std::vector<int> &rcv,
                 std::vector<long long> &amt)
{
    snd.clear();
    rcv.clear();
    amt.clear();
    if (n <= 0) return;
    std::vector<long long> arr(loads, loads + n);
    long long sum = 0;
    for (long long v : arr) sum += v;
    const long long average = sum / n;
    std::priority_queue<std::pair<long long, int>> over, under;
    for (int i = 0; i < n; i++) (arr[i] >= average ? over : under).push({arr[i], i});
    while (!over.empty()) {
        const int sender = over.top().second;
        long long diff = over.top().first - average;
        over.pop();
        while (!under.empty() && diff > 0) {
            const int receiver = under.top().second;
            const long long room = average - under.top().first;
            under.pop();
            const long long x = std::min(diff, room);
            arr[sender] -= x;
            arr[receiver] += x;
            snd.push_back(sender);
            rcv.push_back(receiver);
            amt.push_back(x);
            diff -= x;
            if (arr[receiver] < average) under.push({arr[receiver], receiver});
        }
    }
}

// Consecutive rows from row 0 for each transfer: a transfer takes rows while
// their summed load stays within its amount, and the next transfer starts
// at the first row not taken.  bounds: npacks + 1 row boundaries.
inline void select_rows(const long long *rowload, long long nrows, int npacks, const long long *amount,
                        long long *bounds, long long *moved)
{
    long long r = 0;
    bounds[0] = 0;
    for (int p = 0; p < npacks; p++) {
        long long acc = 0;
        while (r < nrows && acc + rowload[r] <= amount[p]) acc += rowload[r++];
        bounds[p + 1] = r;
        moved[p] = acc;
    }
}

}  // namespace dlb
}  // namespace eu3d
