/*
 * EU3D hot-path oracle: a plain-C CPU restatement of the reference solver's
 * per-step arithmetic (MUSCL/minmod reconstruction, AUSM flux sweeps, TimeAdv
 * EE update, conservative->primitive decode with Newton temperature
 * inversion, IMEX and trapezoid H2 chemistry, ghost fills, CFL).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links or calls this
 * code; tests, the smoke check and the CPU-baseline leg of bench.py use it as
 * the checker.  Each function cites the reference file:line it restates.
 *
 * Layout follows the reference's ARRAY::Array (include/Array.hpp:33-43):
 * row-major, last index fastest.  3D fields are indexed (i, j, k) over the
 * ghosted extents NI x NJ x NK, 4D fields (i, j, k, s) with s innermost.
 */
#ifndef EU3D_ORACLE_H
#define EU3D_ORACLE_H

#include <stddef.h>
#include "../include/eu3d_quirks.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXS 16
#define ORC_MAXR 24

typedef struct {
    int NS, NR;
    double stoi_f[ORC_MAXS * ORC_MAXR]; /* (s, r) -> s * NR + r */
    double stoi_b[ORC_MAXS * ORC_MAXR];
    double react_tb[ORC_MAXS * ORC_MAXR];
    double af[ORC_MAXR], bf[ORC_MAXR], eaf[ORC_MAXR];
    double c0[9 * ORC_MAXS], c1[9 * ORC_MAXS]; /* (k, s) -> k * NS + s */
    double mw[ORC_MAXS], ri[ORC_MAXS];
} orc_mech;

typedef struct {
    int ni, nj, nk, bc, NS;
    int NI, NJ, NK;
    unsigned quirks;
    double dt, time;
    double *xnode, *ynode, *znode;
    /* 3D */
    double *U, *V, *W, *P, *D, *T, *C, *Ma, *Wav, *Rgas, *Cp, *H, *E, *Gamma;
    /* 4D, NS */
    double *Mc, *Yi, *Di;
    /* 4D, NS + 4 */
    double *CS, *RHS, *Partion_T, *F, *G, *Q;
    /* reaction-side per-cell arrays */
    double *CMS;   /* 4D, NS */
    double *MDd;   /* 4D, NS + 4: diagonal of the reference's MD(i,j,k,s,s) */
    int *Nchem;    /* 3D */
    /* ODM inflow planes (nj x nk, Yint nj x nk x NS) */
    double *Uint, *Vint, *Wint, *Pint, *Dint, *Tint, *Hint, *Eint, *Gint, *Yint;
} orc_field;

/* allocation (all arrays zero-filled) */
int orc_field_alloc(orc_field *f, int ni, int nj, int nk, int bc, int NS);
void orc_field_free(orc_field *f);

/* thermo, src/Reaction.cpp:893-948 */
double orc_getcpi(const orc_mech *m, double T, double R, int sp);
double orc_gethi(const orc_mech *m, double T, double R, int sp, unsigned quirks);
double orc_getsi(const orc_mech *m, double T, double R, int sp, unsigned quirks);

/* hot path */
void orc_advection(orc_field *f, int timeadv, int diff);
void orc_update_after_adv(orc_field *f, const orc_mech *m);
void orc_update_after_cs(orc_field *f, const orc_mech *m);
double orc_get_temp(const orc_field *f, const orc_mech *m, double T, int i, int j, int k, const double *Y);
void orc_get_partial_t(orc_field *f, const orc_mech *m);
void orc_diagonalized(orc_field *f, const orc_mech *m);
void orc_update_imex(orc_field *f, const orc_mech *m);
void orc_imex(orc_field *f, const orc_mech *m);
void orc_trapezoid(orc_field *f, const orc_mech *m, int type);
void orc_prediction(orc_field *f, const orc_mech *m);
void orc_explicit(orc_field *f, const orc_mech *m);

/* ghost fills: kind EU3D_BC_* from eu3d_quirks.h */
void orc_boundary(orc_field *f, const orc_mech *m, int kind, const double *wedge);
void orc_cfl(orc_field *f, double cfl, double final_time);

/* one step of Euler::Computing's loop body (src/Euler.cpp:266-333).
   react: 0 trapezoid, 1 IMEX, 2 no chemistry; cfl == 0 uses f->dt as given. */
void orc_step(orc_field *f, const orc_mech *m, int react, int type, int timeadv, int diff, double cfl,
              double final_time, int bc_kind, const double *wedge);

/* initial condition of the shipped 3D RSBI case: ReactionInitial
   (src/Reaction.cpp:339-398) then FieldInitial (src/Flowfield.cpp:159-230) */
void orc_rsbi_initial(orc_field *f, const orc_mech *m, double P_pre, double T_pre, double M_wave);

/* conversion helpers shared with the GPU tests: fill the derived primitives
   of every cell (ghosts included) from CS and T the way FieldInitial does */
void orc_prims_from_state(orc_field *f, const orc_mech *m);

#ifdef __cplusplus
}
#endif
#endif
