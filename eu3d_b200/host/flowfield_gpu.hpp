// Host shim of the EU3D hot path for a C++ caller: the member functions of
// the reference's Flowfield / Reaction that Euler::Computing calls
// (src/Euler.cpp:256-344), each forwarding to one entry point of the C ABI in
// include/eu3d_gpu.h.  Host arrays keep the reference's layout
// (ARRAY::Array, include/Array.hpp:33-43: row-major over the ghosted extents,
// last index fastest, per-cell vectors innermost), so a caller hands over the
// buffers it already owns.  Errors follow the reference's convention: the
// message goes to stderr and the process aborts.
//
// Call shapes kept (reference declarations):
//   Flowfield::CFLcondition(double, double)          include/Flowfield.hpp:157
//   Flowfield::FieldBoundary_3dODM/_3dRSBI()          include/Flowfield.hpp:160-162
//   Flowfield::Advection(int TimeAdv, int Diff)       include/Flowfield.hpp:165
//   Flowfield::Update_after_CS()                      include/Flowfield.hpp:178
//   Euler::Trapezoid(int) / Euler::IMEX()             include/Euler.hpp:110-113 (Reaction.hpp:157-162 underneath)
//   TwoDim.D.IsNan() || TwoDim.T.IsNan()              src/Euler.cpp:319-331
#pragma once

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/eu3d_gpu.h"

namespace eu3d_host {

inline void check(int rc, const char *what)
{
    if (rc != EU3D_OK) {
        std::fprintf(stderr, "eu3d: %s failed (%d): %s\n", what, rc, eu3d_last_error());
        std::abort();
    }
}

// The mechanism and mesh as Reaction::ReactionRead and Mesh::MeshProcess
// leave them (host arrays owned by the caller).
struct MeshAndMechanism {
    int ni, nj, nk, bc, NS, NR;
    const double *xnode, *ynode, *znode;
    const double *stoi_f, *stoi_b, *react_tb, *af, *bf, *eaf, *coeff0, *coeff1, *mw;
};

class GpuFlowfield {
  public:
    GpuFlowfield(const MeshAndMechanism &m, unsigned quirks, int flux_bits, int device)
    {
        eu3d_desc d{};
        d.ni = m.ni;
        d.nj = m.nj;
        d.nk = m.nk;
        d.bc = m.bc;
        d.xnode = m.xnode;
        d.ynode = m.ynode;
        d.znode = m.znode;
        d.NS = m.NS;
        d.NR = m.NR;
        d.stoi_f = m.stoi_f;
        d.stoi_b = m.stoi_b;
        d.react_tb = m.react_tb;
        d.af = m.af;
        d.bf = m.bf;
        d.eaf = m.eaf;
        d.coeff0 = m.coeff0;
        d.coeff1 = m.coeff1;
        d.mw = m.mw;
        d.quirks = quirks;
        d.flux_bits = flux_bits;
        d.device = device;
        check(eu3d_create(&d, &h_), "eu3d_create");
    }
    ~GpuFlowfield() { eu3d_destroy(h_); }
    GpuFlowfield(const GpuFlowfield &) = delete;
    GpuFlowfield &operator=(const GpuFlowfield &) = delete;

    // host <-> device, reference layout
    void Upload(int field, const double *host) { check(eu3d_upload_field(h_, field, host), "eu3d_upload_field"); }
    void Download(int field, double *host) { check(eu3d_download_field(h_, field, host), "eu3d_download_field"); }
    // Uint .. Yint of FieldBoundary_3dODM (include/Flowfield.hpp:105-106)
    void SetInflow(const double *U, const double *V, const double *W, const double *P, const double *D,
                   const double *T, const double *H, const double *E, const double *G, const double *Y)
    {
        check(eu3d_set_inflow(h_, U, V, W, P, D, T, H, E, G, Y), "eu3d_set_inflow");
    }

    // Flowfield::CFLcondition: dt from the device reduction, time advanced there
    void CFLcondition(double cfl, double final_time) { check(eu3d_cfl(h_, cfl, final_time, &dt), "eu3d_cfl"); }
    void SetDt(double v)
    {
        dt = v;
        check(eu3d_set_dt(h_, v), "eu3d_set_dt");
    }
    void FieldBoundary(int kind) { check(eu3d_boundary(h_, kind), "eu3d_boundary"); }
    void FieldBoundary_3dRSBI() { FieldBoundary(EU3D_BC_RSBI); }
    void FieldBoundary_3dODM() { FieldBoundary(EU3D_BC_ODM); }
    void Advection(int timeadv, int diff) { check(eu3d_advection(h_, timeadv, diff), "eu3d_advection"); }
    void Update_after_CS() { check(eu3d_update_after_cs(h_), "eu3d_update_after_cs"); }
    void IMEX() { check(eu3d_react_imex(h_), "eu3d_react_imex"); }
    void Trapezoid(int type) { check(eu3d_react_trapezoid(h_, type), "eu3d_react_trapezoid"); }
    // the whole loop body as one CUDA-graph replay
    void Step(const eu3d_step_desc &s) { check(eu3d_step(h_, &s), "eu3d_step"); }
    // D.IsNan() || T.IsNan()
    bool IsNan()
    {
        eu3d_status st{};
        check(eu3d_get_status(h_, &st), "eu3d_get_status");
        return st.nonfinite_cells != 0;
    }
    eu3d_status Status()
    {
        eu3d_status st{};
        check(eu3d_get_status(h_, &st), "eu3d_get_status");
        return st;
    }

    double dt = 0.0;

  private:
    eu3d_handle *h_ = nullptr;
};

}  // namespace eu3d_host
