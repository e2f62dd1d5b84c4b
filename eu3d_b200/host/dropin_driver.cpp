// Euler::Computing's loop body (src/Euler.cpp:256-344) driven through the
// C++ shim (flowfield_gpu.hpp) on reference-layout host buffers: a compiled
// C++ caller of include/eu3d_gpu.h.
//
//   eu3d_dropin <case.bin> <result.bin>
//
// case.bin (little-endian, written by the caller):
//   int32[18]  magic 0x44335545, version 1, ni, nj, nk, bc, NS, NR, steps,
//              react, type, timeadv, diff, bc_kind, quirks, flux_bits,
//              whole_step (0: member by member, 1: eu3d_step), has_inflow
//   double[3]  cfl, final_time, dt (used when cfl == 0)
//   double     xnode[NI], ynode[NJ], znode[NK]
//   double     stoi_f[NS*NR], stoi_b[NS*NR], react_tb[NS*NR], af[NR], bf[NR],
//              eaf[NR], coeff0[9*NS], coeff1[9*NS], mw[NS]
//   double     U, V, W, P, D, T, H, Gamma, E [NI*NJ*NK each], Yi [NI*NJ*NK*NS],
//              CS [NI*NJ*NK*(NS+4)]
//   has_inflow: double Uint..Gint [nj*nk each] (U V W P D T H E G), Yint [nj*nk*NS]
// result.bin: double CS[NI*NJ*NK*(NS+4)], T, P, D [NI*NJ*NK each], then
//   double dt, time and int64 nonfinite_cells, newton_capped, nan_step
//   (the step after which D or T went NaN, -1: none; the reference aborts there).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "flowfield_gpu.hpp"

namespace {

struct Reader {
    FILE *f;
    template <class T>
    void get(T *p, size_t n)
    {
        if (n && std::fread(p, sizeof(T), n, f) != n) {
            std::fprintf(stderr, "eu3d_dropin: case file ends early\n");
            std::exit(2);
        }
    }
    std::vector<double> vec(size_t n)
    {
        std::vector<double> v(n);
        get(v.data(), n);
        return v;
    }
};

}  // namespace

int main(int argc, char **argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s case.bin result.bin\n", argv[0]);
        return 2;
    }
    FILE *fin = std::fopen(argv[1], "rb");
    if (!fin) {
        std::perror(argv[1]);
        return 2;
    }
    Reader r{fin};
    int32_t hd[18];
    r.get(hd, 18);
    if (hd[0] != 0x44335545 || hd[1] != 1) {
        std::fprintf(stderr, "eu3d_dropin: not a version-1 case file\n");
        return 2;
    }
    const int ni = hd[2], nj = hd[3], nk = hd[4], bc = hd[5], NS = hd[6], NR = hd[7], steps = hd[8];
    const int react = hd[9], type = hd[10], timeadv = hd[11], diff = hd[12], bc_kind = hd[13];
    const unsigned quirks = (unsigned)hd[14];
    const int flux_bits = hd[15], whole_step = hd[16], has_inflow = hd[17];
    double sc[3];
    r.get(sc, 3);
    const double cfl = sc[0], final_time = sc[1], dt = sc[2];
    const size_t NI = ni + 2 * bc, NJ = nj + 2 * bc, NK = nk + 2 * bc, n3 = NI * NJ * NK;
    std::vector<double> xn = r.vec(NI), yn = r.vec(NJ), zn = r.vec(NK);
    std::vector<double> sf = r.vec(NS * NR), sb = r.vec(NS * NR), tb = r.vec(NS * NR);
    std::vector<double> af = r.vec(NR), bf = r.vec(NR), eaf = r.vec(NR);
    std::vector<double> c0 = r.vec(9 * NS), c1 = r.vec(9 * NS), mw = r.vec(NS);
    const int f3[9] = {EU3D_FIELD_U, EU3D_FIELD_V, EU3D_FIELD_W, EU3D_FIELD_P, EU3D_FIELD_D,
                       EU3D_FIELD_T, EU3D_FIELD_H, EU3D_FIELD_GAMMA, EU3D_FIELD_E};
    std::vector<std::vector<double>> prim(9);
    for (int f = 0; f < 9; f++) prim[f] = r.vec(n3);
    std::vector<double> Yi = r.vec(n3 * NS), CS = r.vec(n3 * (NS + 4));
    std::vector<std::vector<double>> inflow;
    if (has_inflow) {
        for (int f = 0; f < 9; f++) inflow.push_back(r.vec((size_t)nj * nk));
        inflow.push_back(r.vec((size_t)nj * nk * NS));
    }
    std::fclose(fin);

    // Euler::Euler(): the handle over the rank's mesh and mechanism, state uploaded
    const eu3d_host::MeshAndMechanism mm{ni,        nj,        nk,        bc,        NS,        NR,
                                         xn.data(), yn.data(), zn.data(), sf.data(), sb.data(), tb.data(),
                                         af.data(), bf.data(), eaf.data(), c0.data(), c1.data(), mw.data()};
    eu3d_host::GpuFlowfield TwoDim(mm, quirks, flux_bits, 0);
    for (int f = 0; f < 9; f++) TwoDim.Upload(f3[f], prim[f].data());
    TwoDim.Upload(EU3D_FIELD_YI, Yi.data());
    TwoDim.Upload(EU3D_FIELD_CS, CS.data());
    if (has_inflow)
        TwoDim.SetInflow(inflow[0].data(), inflow[1].data(), inflow[2].data(), inflow[3].data(), inflow[4].data(),
                         inflow[5].data(), inflow[6].data(), inflow[7].data(), inflow[8].data(), inflow[9].data());
    if (cfl == 0.0) TwoDim.SetDt(dt);

    long long nan_step = -1;
    for (int it = 0; it < steps && nan_step < 0; it++) {
        if (whole_step) {
            eu3d_step_desc s{react, type, timeadv, diff, bc_kind, cfl, final_time};
            TwoDim.Step(s);
        } else {
            // src/Euler.cpp:266-333, member by member
            if (cfl != 0.0) TwoDim.CFLcondition(cfl, final_time);
            TwoDim.FieldBoundary(bc_kind);
            TwoDim.Advection(timeadv, diff);
            if (react == EU3D_REACT_IMEX)
                TwoDim.IMEX();
            else if (react == EU3D_REACT_TRAPEZOID)
                TwoDim.Trapezoid(type);
        }
        if (TwoDim.IsNan()) nan_step = it;
    }

    TwoDim.Download(EU3D_FIELD_CS, CS.data());
    std::vector<double> T(n3), P(n3), D(n3);
    TwoDim.Download(EU3D_FIELD_T, T.data());
    TwoDim.Download(EU3D_FIELD_P, P.data());
    TwoDim.Download(EU3D_FIELD_D, D.data());
    const eu3d_status st = TwoDim.Status();
    FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) {
        std::perror(argv[2]);
        return 2;
    }
    std::fwrite(CS.data(), sizeof(double), CS.size(), fo);
    std::fwrite(T.data(), sizeof(double), n3, fo);
    std::fwrite(P.data(), sizeof(double), n3, fo);
    std::fwrite(D.data(), sizeof(double), n3, fo);
    const double tail_d[2] = {st.dt, st.time};
    const int64_t tail_i[3] = {st.nonfinite_cells, st.newton_capped, nan_step};
    std::fwrite(tail_d, sizeof(double), 2, fo);
    std::fwrite(tail_i, sizeof(int64_t), 3, fo);
    std::fclose(fo);
    return 0;
}
