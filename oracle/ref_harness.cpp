// Function-level harness around the reference EU3D sources (test
// infrastructure only).  It is compiled together with the reference's own
// src/{Flowfield,Reaction,Mesh,TimeAdv,Function,FileReader,Global,LoadBalance}.cpp, left
// unmodified, into oracle/_ref/libeu3d_ref.so.  The reference's driver class
// `Euler` is a friend of Flowfield, Reaction and Mesh
// (include/Flowfield.hpp:139, include/Reaction.hpp:140, include/Mesh.hpp:57);
// this file supplies its own `Euler` so that a test can set every private
// array and call each hot-path member function in isolation, exactly as
// Euler::Computing / Euler::IMEX / Euler::Trapezoid do
// (src/Euler.cpp:256-344, :357-760) on a single rank.
//
// Deviations from the reference driver, all deliberate and documented:
//  * arrays that the reference allocates with `new T[]` and may read before
//    writing (YL_temp/YR_temp, MD, RHS, Partion_T, ...) are zero-filled after
//    construction, which is what the reference sees for mmap-backed
//    allocations; this makes the harness deterministic.
//  * Reaction::Trapezoid returns its member array by value through the
//    implicit (shallow) copy constructor (src/Reaction.cpp:484); the
//    reference then frees the member's buffer when the temporary dies
//    (src/Euler.cpp:375), a use-after-free on the next call.  The harness keeps
//    the returned shallow copy alive, so each call computes what the
//    reference computes when memory is not reused.
//  * dynamic load balancing is a no-op on one rank and is not run as part of a
//    step; its planner (DynamicLoadBalancer::DLBPriorityQueue) is exported on
//    its own (ref_dlb_plan) so the transfer plan can be compared.
#include <cstring>
#include <cstdint>
#include <string>
#include <mpi.h>

#include "Array.hpp"
#include "Mesh.hpp"
#include "Flowfield.hpp"
#include "Reaction.hpp"
#include "Global.hpp"
#include "LoadBalance.hpp"

namespace {
struct RefCase {
    Flowfield flow;
    Reaction react;
};

template <class A> void zero(A &a) { a.Fill(0); }

template <class T1>
void copy_in(Array<T1, 1> &dst, const double *src, int n)
{
    dst.Initial(n);
    for (int i = 0; i < n; i++) dst(i) = src[i];
}
}  // namespace

class Euler {
public:
    static void set_globals()
    {
        myid = 0;
        numprocs = 1;
        m_block_x = m_block_y = m_block_z = 1;
        myid_x = myid_y = myid_z = 0;
        m_left = m_right = m_up = m_down = m_front = m_back = MPI_PROC_NULL;
        num_thread = 1;
    }

    // mech tables: Stoi_F/Stoi_B/React_TB as (NS, NR) row-major, Coeff0/1 as (9, NS)
    static RefCase *create(int ni, int nj, int nk, int bc, const double *xn, const double *yn, const double *zn,
                           int NS, int NR, int TB, const double *stoi_f, const double *stoi_b, const double *react_tb,
                           const double *af, const double *bf, const double *eaf, const double *c0, const double *c1,
                           const double *mw)
    {
        set_globals();
        RefCase *c = new RefCase();
        Flowfield &F = c->flow;
        Reaction &R = c->react;
        copy_in(F.xnode, xn, ni + 2 * bc);
        copy_in(F.ynode, yn, nj + 2 * bc);
        copy_in(F.znode, zn, nk + 2 * bc);
        F.bc = bc;
        F.ni = ni;
        F.nj = nj;
        F.nk = nk;
        F.NS = NS;
        F.NR = NR;
        F.Construction();

        copy_in(R.xnode, xn, ni + 2 * bc);
        copy_in(R.ynode, yn, nj + 2 * bc);
        copy_in(R.znode, zn, nk + 2 * bc);
        R.bc = bc;
        R.ni = ni;
        R.nj = nj;
        R.nk = nk;
        R.NS = NS;
        R.NR = NR;
        R.TB = TB;
        R.ReactionConstruction();
        for (int s = 0; s < NS; s++)
            for (int r = 0; r < NR; r++) {
                R.Stoi_F(s, r) = stoi_f[s * NR + r];
                R.Stoi_B(s, r) = stoi_b[s * NR + r];
                R.React_TB(s, r) = react_tb[s * NR + r];
            }
        for (int r = 0; r < NR; r++) {
            R.Af(r) = af[r];
            R.Bf(r) = bf[r];
            R.Eaf(r) = eaf[r];
        }
        for (int k = 0; k < 9; k++)
            for (int s = 0; s < NS; s++) {
                R.Coeff0(k, s) = c0[k * NS + s];
                R.Coeff1(k, s) = c1[k * NS + s];
            }
        for (int s = 0; s < NS; s++) {
            R.Mw(s) = mw[s];
            R.Ri(s) = R.R / R.Mw(s);  // as ReactionInitial, src/Reaction.cpp:352-353
        }
        // Flowfield's copies, as FieldInitial sets them (src/Flowfield.cpp:166-169)
        F.Ri = R.Ri;
        F.Mw = R.Mw;
        F.Coeff0 = R.Coeff0;
        F.Coeff1 = R.Coeff1;

        zero(F.U); zero(F.V); zero(F.W); zero(F.P); zero(F.D); zero(F.T); zero(F.C); zero(F.Ma);
        zero(F.Wav); zero(F.Rgas); zero(F.Cp); zero(F.H); zero(F.E); zero(F.Gamma);
        zero(F.Mr); zero(F.Mc); zero(F.Mi); zero(F.Yi); zero(F.Di);
        zero(F.CS); zero(F.F); zero(F.G); zero(F.Q); zero(F.RHS); zero(F.Partion_T);
        zero(F.PLR); zero(F.DLR); zero(F.ULR); zero(F.VLR); zero(F.WLR); zero(F.HLR); zero(F.GLR); zero(F.YLR);
        zero(F.Yi_temp); zero(F.YL_temp); zero(F.YR_temp);
        zero(F.Uint); zero(F.Vint); zero(F.Wint); zero(F.Pint); zero(F.Dint); zero(F.Tint);
        zero(F.Hint); zero(F.Eint); zero(F.Gint); zero(F.Yint);
        F.Cpi.Fill(0.0); F.Hi.Fill(0.0); F.Ei.Fill(0.0); F.Yi_temp0.Fill(0.0);
        zero(R.Mr); zero(R.Mi); zero(R.Yi); zero(R.Mc); zero(R.Di); zero(R.CMS); zero(R.MD);
        F.dt = 0.0;
        F.time = 0.0;
        return c;
    }

    static double *field(RefCase *c, const char *name, size_t *len)
    {
        Flowfield &F = c->flow;
        Reaction &R = c->react;
#define EU3D_F(nm) if (!std::strcmp(name, #nm)) { *len = F.nm.GetLen(); return F.nm.Getbuf(); }
#define EU3D_R(nm) if (!std::strcmp(name, "R." #nm)) { *len = R.nm.GetLen(); return R.nm.Getbuf(); }
        EU3D_F(U) EU3D_F(V) EU3D_F(W) EU3D_F(P) EU3D_F(D) EU3D_F(T) EU3D_F(C) EU3D_F(Ma)
        EU3D_F(Wav) EU3D_F(Rgas) EU3D_F(Cp) EU3D_F(H) EU3D_F(E) EU3D_F(Gamma)
        EU3D_F(Mc) EU3D_F(Yi) EU3D_F(Di) EU3D_F(Mi)
        EU3D_F(CS) EU3D_F(RHS) EU3D_F(Partion_T) EU3D_F(F) EU3D_F(G) EU3D_F(Q)
        EU3D_F(Uint) EU3D_F(Vint) EU3D_F(Wint) EU3D_F(Pint) EU3D_F(Dint) EU3D_F(Tint)
        EU3D_F(Hint) EU3D_F(Eint) EU3D_F(Gint) EU3D_F(Yint)
        EU3D_R(Mc) EU3D_R(Di) EU3D_R(CMS) EU3D_R(MD)
#undef EU3D_F
#undef EU3D_R
        *len = 0;
        return nullptr;
    }

    static int *nchem(RefCase *c, size_t *len)
    {
        *len = c->react.Nchem.GetLen();
        return c->react.Nchem.Getbuf();
    }

    static void set_dt(RefCase *c, double dt) { c->flow.dt = dt; }
    static double get_dt(RefCase *c) { return c->flow.dt; }
    static double get_time(RefCase *c) { return c->flow.time; }
    static void set_time(RefCase *c, double t) { c->flow.time = t; }

    static void cfl(RefCase *c, double cfl, double final_time) { c->flow.CFLcondition(cfl, final_time); }
    static void boundary(RefCase *c, int kind)
    {
        if (kind == 0) c->flow.FieldBoundary_3dRSBI();
        else if (kind == 1) c->flow.FieldBoundary_3dODM();
    }
    static void advection(RefCase *c, int timeadv, int diff) { c->flow.Advection(timeadv, diff); }
    static void update_after_adv(RefCase *c) { c->flow.Update_after_Adv(); }
    static void update_after_cs(RefCase *c) { c->flow.Update_after_CS(); }
    static void explicit_field(RefCase *c) { c->flow.Explicit(); }
    static void partial_t(RefCase *c) { c->flow.GetPartial_T(); }

    // Euler::IMEX, src/Euler.cpp:748-760
    static void imex(RefCase *c)
    {
        Flowfield &F = c->flow;
        c->react.Diagonalized(F.Mc, F.Di, F.T, F.Partion_T);
        F.Update_IMEX(c->react.CMS, c->react.MD);
    }

    // Euler::Trapezoid(type) on one rank, src/Euler.cpp:357-737 (DLB inactive)
    static void trapezoid(RefCase *c, int type)
    {
        Flowfield &F = c->flow;
        Reaction &R = c->react;
        const int ni = F.ni, nj = F.nj, nk = F.nk, bc = F.bc;
        F.Update_after_Adv();
        if (type == 0) {
            // the returned shallow copy shares R.Di's buffer; it is kept alive on
            // purpose so that the buffer is never freed (see the file header)
            Array<double, 4> *shared = new Array<double, 4>(R.Trapezoid(F.Mc, F.Di, F.T, F.dt));
            F.Di = *shared;
            F.Explicit();
        } else {
            R.TrapezoidPrediction(F.Mc, F.Di, F.Yi, F.T, F.dt);
            for (int i = bc; i < (ni - 1) / 2 + bc; i++)
                for (int j = bc; j < nj + bc; j++)
                    for (int k = bc; k < nk + bc; k++)
                        for (int step = 0; step < R.Nchem(i, j, k); step++) {
                            R.Trapezoid(F.Mc, F.Di, F.Yi, F.T, F.dt, step, i, j, k);
                            F.Explicit(step, i, j, k);
                        }
            for (int i = (ni - 1) / 2 + bc; i < ni + bc; i++)
                for (int j = bc; j < nj + bc; j++)
                    for (int k = bc; k < nk + bc; k++)
                        for (int step = 0; step < R.Nchem(i, j, k); step++) {
                            R.Trapezoid(F.Mc, F.Di, F.Yi, F.T, F.dt, step, i, j, k);
                            F.Explicit(step, i, j, k);
                        }
        }
    }

    static void prediction(RefCase *c)
    {
        Flowfield &F = c->flow;
        c->react.TrapezoidPrediction(F.Mc, F.Di, F.Yi, F.T, F.dt);
    }

    static double get_temp(RefCase *c, double T, int i, int j, int k, const double *Y)
    {
        Flowfield &F = c->flow;
        Array<double, 1> y(F.NS);
        for (int s = 0; s < F.NS; s++) y(s) = Y[s];
        return F.Get_temp(T, i, j, k, y);
    }

    // which: 0 = GetCpi, 1 = GetHi, 2 = GetSi
    static double thermo(RefCase *c, int which, double T, double Rgas, int sp)
    {
        Reaction &R = c->react;
        if (which == 0) return R.GetCpi(T, Rgas, sp, R.Coeff0, R.Coeff1);
        if (which == 1) return R.GetHi(T, Rgas, sp, R.Coeff0, R.Coeff1);
        return R.GetSi(T, Rgas, sp, R.Coeff0, R.Coeff1);
    }

    // Reaction::ReactionRead on the given mechanism/thermo files, for pinning
    // the project's own reader.  Tables out in the same layouts as create().
    static int read_mechanism(const char *mech, const char *thermo, int *ns_nr_tb, double *stoi_f, double *stoi_b,
                              double *react_tb, double *af, double *bf, double *eaf, double *c0, double *c1,
                              double *mw, int cap_ns, int cap_nr)
    {
        set_globals();
        Array<double, 1> xn(5), yn(5), zn(5);
        for (int i = 0; i < 5; i++) { xn(i) = 0.01 * i; yn(i) = 0.01 * i; zn(i) = 0.01 * i; }
        Reaction *R = new Reaction();
        char m[512], t[512];
        std::strncpy(m, mech, sizeof(m) - 1); m[sizeof(m) - 1] = 0;
        std::strncpy(t, thermo, sizeof(t) - 1); t[sizeof(t) - 1] = 0;
        R->ReactionRead(m, t, xn, yn, zn, 2);
        const int NS = R->NS, NR = R->NR;
        ns_nr_tb[0] = NS; ns_nr_tb[1] = NR; ns_nr_tb[2] = R->TB;
        if (NS > cap_ns || NR > cap_nr) return -1;
        for (int s = 0; s < NS; s++)
            for (int r = 0; r < NR; r++) {
                stoi_f[s * NR + r] = R->Stoi_F(s, r);
                stoi_b[s * NR + r] = R->Stoi_B(s, r);
                react_tb[s * NR + r] = R->React_TB(s, r);
            }
        for (int r = 0; r < NR; r++) { af[r] = R->Af(r); bf[r] = R->Bf(r); eaf[r] = R->Eaf(r); }
        for (int k = 0; k < 9; k++)
            for (int s = 0; s < NS; s++) { c0[k * NS + s] = R->Coeff0(k, s); c1[k * NS + s] = R->Coeff1(k, s); }
        for (int s = 0; s < NS; s++) mw[s] = R->Mw(s);
        return 0;  // the Reaction object is leaked: its destructor frees nothing it owns
    }
};

extern "C" {
void *ref_create(int ni, int nj, int nk, int bc, const double *xn, const double *yn, const double *zn, int NS, int NR,
                 int TB, const double *stoi_f, const double *stoi_b, const double *react_tb, const double *af,
                 const double *bf, const double *eaf, const double *c0, const double *c1, const double *mw)
{
    return Euler::create(ni, nj, nk, bc, xn, yn, zn, NS, NR, TB, stoi_f, stoi_b, react_tb, af, bf, eaf, c0, c1, mw);
}
void ref_destroy(void *h) { delete static_cast<RefCase *>(h); }
double *ref_field(void *h, const char *name, size_t *len) { return Euler::field(static_cast<RefCase *>(h), name, len); }
int *ref_nchem(void *h, size_t *len) { return Euler::nchem(static_cast<RefCase *>(h), len); }
void ref_set_dt(void *h, double dt) { Euler::set_dt(static_cast<RefCase *>(h), dt); }
double ref_get_dt(void *h) { return Euler::get_dt(static_cast<RefCase *>(h)); }
double ref_get_time(void *h) { return Euler::get_time(static_cast<RefCase *>(h)); }
void ref_set_time(void *h, double t) { Euler::set_time(static_cast<RefCase *>(h), t); }
void ref_cfl(void *h, double cfl, double final_time) { Euler::cfl(static_cast<RefCase *>(h), cfl, final_time); }
void ref_boundary(void *h, int kind) { Euler::boundary(static_cast<RefCase *>(h), kind); }
void ref_advection(void *h, int timeadv, int diff) { Euler::advection(static_cast<RefCase *>(h), timeadv, diff); }
void ref_update_after_adv(void *h) { Euler::update_after_adv(static_cast<RefCase *>(h)); }
void ref_update_after_cs(void *h) { Euler::update_after_cs(static_cast<RefCase *>(h)); }
void ref_explicit(void *h) { Euler::explicit_field(static_cast<RefCase *>(h)); }
void ref_partial_t(void *h) { Euler::partial_t(static_cast<RefCase *>(h)); }
void ref_imex(void *h) { Euler::imex(static_cast<RefCase *>(h)); }
void ref_trapezoid(void *h, int type) { Euler::trapezoid(static_cast<RefCase *>(h), type); }
void ref_prediction(void *h) { Euler::prediction(static_cast<RefCase *>(h)); }
double ref_get_temp(void *h, double T, int i, int j, int k, const double *Y)
{
    return Euler::get_temp(static_cast<RefCase *>(h), T, i, j, k, Y);
}
double ref_thermo(void *h, int which, double T, double R, int sp)
{
    return Euler::thermo(static_cast<RefCase *>(h), which, T, R, sp);
}
int ref_read_mechanism(const char *mech, const char *thermo, int *ns_nr_tb, double *stoi_f, double *stoi_b,
                       double *react_tb, double *af, double *bf, double *eaf, double *c0, double *c1, double *mw,
                       int cap_ns, int cap_nr)
{
    return Euler::read_mechanism(mech, thermo, ns_nr_tb, stoi_f, stoi_b, react_tb, af, bf, eaf, c0, c1, mw, cap_ns,
                                 cap_nr);
}
// DynamicLoadBalancer::DLBPriorityQueue (src/LoadBalance.cpp:8-59) on per-rank
// loads; out receives (sender, receiver, amount) triples, at most cap of them.
// Returns the number of transfers.
int ref_dlb_plan(const int *loads, int n, int *out, int cap)
{
    Array<int, 1> arr(n);
    for (int i = 0; i < n; i++) arr(i) = loads[i];
    DynamicLoadBalancer dlb;
    dlb.DLBPriorityQueue(arr);
    const int m = (int)dlb.transferNchem.size();
    for (int t = 0; t < m && t < cap; t++) {
        out[3 * t] = std::get<0>(dlb.transferNchem[t]);
        out[3 * t + 1] = std::get<1>(dlb.transferNchem[t]);
        out[3 * t + 2] = std::get<2>(dlb.transferNchem[t]);
    }
    return m;
}
}
