/*
 * EU3D B200 hot path: C ABI.
 *
 * A device-resident flowfield for one rank of the EU3D reactive Euler solver,
 * advanced by hand-written sm_100a CUDA kernels.  Each entry point replaces
 * one member function of the reference's Flowfield / Reaction / TimeAdv
 * classes or one step of Euler::Computing; the reference interface it stands
 * in for is cited beside it.  A host C++ caller keeps its own readers and
 * arrays (Mesh, FileReader, Reaction::ReactionRead) and hands the library
 * plain pointers.
 *
 * Conventions
 *  - Every function returns 0 (EU3D_OK) or a negative EU3D_ERR_* code; no
 *    exception crosses the ABI.  eu3d_last_error() gives a text for the last
 *    failure on the calling thread.
 *  - Host arrays use the reference layout (ARRAY::Array, include/Array.hpp:33-43):
 *    row-major over the ghosted extents NI = ni + 2 bc, NJ, NK with the last
 *    index fastest; per-cell vectors (species, conserved variables) innermost.
 *  - The library owns all device memory of a handle; the caller owns every
 *    host pointer.  Calls on one handle are issued on the handle's own CUDA
 *    stream and are not thread-safe per handle (the reference's ranks are
 *    single-threaded).
 *  - The mechanism tables of all handles in one process must be identical:
 *    they live in the device's constant memory.  Quirk policies and every
 *    other setting are per handle.
 */
#ifndef EU3D_GPU_H
#define EU3D_GPU_H

#include <stddef.h>
#include "eu3d_quirks.h"

#ifdef __cplusplus
extern "C" {
#endif

#define EU3D_OK 0
#define EU3D_ERR_ARG (-1)       /* invalid argument or unsupported size */
#define EU3D_ERR_CUDA (-2)      /* a CUDA call failed */
#define EU3D_ERR_NOMEM (-3)     /* device allocation failed */
#define EU3D_ERR_MECH (-4)      /* mechanism differs from the one already loaded */
#define EU3D_ERR_STATE (-5)     /* call not valid in the handle's current state */
#define EU3D_ERR_NONFINITE (-6) /* a NaN/Inf density or temperature was found */
#define EU3D_ERR_IO (-7)        /* a result file could not be written */

/* Interior node counts, ghost width and node coordinates come from the
   reference's Mesh (include/Mesh.hpp:22-46, src/Mesh.cpp:75-130); the
   mechanism tables from Reaction::ReactionRead (src/Reaction.cpp:150-326).
   This build supports NS = 9, NR = 19 (the H2_JA919 mechanism). */
typedef struct {
    int ni, nj, nk, bc;
    const double *xnode, *ynode, *znode; /* lengths ni+2bc, nj+2bc, nk+2bc */
    int NS, NR;
    const double *stoi_f, *stoi_b, *react_tb; /* (NS, NR) row-major */
    const double *af, *bf, *eaf;             /* (NR) Arrhenius A, b, Ea[cal/mol] */
    const double *coeff0, *coeff1;           /* (9, NS): a1..a7, b1, b2 per range */
    const double *mw;                        /* (NS) g/mol */
    unsigned quirks;                         /* EU3D_Q_* bit set */
    int flux_bits;                           /* 64: FP64 reconstruction/AUSM; 32: FP32 */
    int device;                              /* CUDA device ordinal */
} eu3d_desc;

typedef struct eu3d_handle eu3d_handle;
typedef struct eu3d_surrogate eu3d_surrogate;

/* Field identifiers for upload/download.  Shapes (reference layout):
   3D fields NI*NJ*NK; EU3D_FIELD_YI/MC/DI NI*NJ*NK*NS; CS/RHS NI*NJ*NK*(NS+4).
   Host arrays are always double.  On the device the primitives (U V W P D H
   Gamma Yi) and the flux residual RHS have the flux precision (flux_bits: FP32
   or FP64); CS, T and E are FP64. */
enum {
    EU3D_FIELD_U = 0, EU3D_FIELD_V, EU3D_FIELD_W, EU3D_FIELD_P, EU3D_FIELD_D, EU3D_FIELD_T,
    EU3D_FIELD_H, EU3D_FIELD_GAMMA, EU3D_FIELD_E,
    EU3D_FIELD_YI, EU3D_FIELD_CS, EU3D_FIELD_RHS,
    /* download only: recomputed from the state */
    EU3D_FIELD_C, EU3D_FIELD_MC, EU3D_FIELD_DI, EU3D_FIELD_NCHEM /* substep counts, as doubles */,
    EU3D_FIELD_COUNT
};

typedef struct {
    int react;      /* EU3D_REACT_* */
    int type;       /* trapezoid: 0 field form, 1 adaptive substeps */
    int timeadv;    /* EU3D_ADV_* */
    int diff;       /* EU3D_DIFF_* */
    int bc_kind;    /* EU3D_BC_* */
    double cfl;     /* 0: use the dt set by eu3d_set_dt */
    double final_time;
} eu3d_step_desc;

typedef struct {
    long long nonfinite_cells;   /* cells whose D or T became NaN/Inf */
    long long newton_capped;     /* decodes that used all 10 Newton iterations */
    long long substeps;          /* adaptive-trapezoid substeps taken */
    int nchem_max;               /* largest per-cell substep count since the last reset */
    int substep_capped;          /* cells whose substep count hit the cap: the adaptive trapezoid's
                                    TrapezoidPrediction count above its cap, or an adaptive-chemistry
                                    substep lengthened by nmax (dt / nmax at least, the last allowed
                                    substep takes the time left) */
    long long surrogate_cells;   /* cells advanced by the learned surrogate */
    long long surrogate_fallback;/* cells sent back to the integrator */
    double dt, time;             /* device copies of Flowfield::dt / ::time */
    long long surrogate_audited; /* surrogate cells re-run by the integrator to judge it */
    double surrogate_audit_max_dT; /* largest |T_surrogate - T_integrator| over audited cells [K] */
    long long surrogate_rejects[4]; /* why cells fell back: outside the envelope, network output
                                       (non-finite, |dT| too large, negative fraction), energy
                                       residual, failed decode */
    long long wait_timeouts;     /* kernels that gave up a bounded wait on an asynchronous copy
                                    (their results for that launch are incomplete) */
    long long surrogate_frozen;  /* cells the frozen-chemistry gate kept out of the network */
    long long frozen_audited;    /* of those, cells also run through the FP64 integrator */
    double frozen_audit_max_dT;  /* largest |T_integrator - T| over them [K] */
    long long drain_timeouts;    /* after a timed-out wait, the bounded wait for the copies still in
                                    flight ran out as well: treat the device state as untrusted */
} eu3d_status;

const char *eu3d_last_error(void);

/* Flowfield::Construction + the member copies FieldInitial makes
   (src/Flowfield.cpp:72-150, :166-169); Reaction::ReactionConstruction. */
int eu3d_create(const eu3d_desc *desc, eu3d_handle **out);
int eu3d_destroy(eu3d_handle *h);

/* Host <-> device copies with the reference-layout transpose. */
int eu3d_upload_field(eu3d_handle *h, int field, const double *host);
int eu3d_download_field(eu3d_handle *h, int field, double *host);
/* Inflow planes of FieldBoundary_3dODM (Uint..Yint, include/Flowfield.hpp:105-106):
   nj*nk each (Y: nj*nk*NS); any pointer may be NULL to keep the old plane. */
int eu3d_set_inflow(eu3d_handle *h, const double *U, const double *V, const double *W, const double *P,
                    const double *D, const double *T, const double *H, const double *E, const double *G,
                    const double *Y);
/* Uniform state in every cell, ghosts included (new; the reference's
   FieldInitial hard-codes its RSBI state): P, T, velocity and NS mass
   fractions, completed with FieldInitial's arithmetic (src/Flowfield.cpp:193-229). */
int eu3d_init_uniform(eu3d_handle *h, double P, double T, double U, double V, double W, const double *Y);
/* Wedge immersed boundary (new): solid where x > x0 and y - y0 < (x - x0) tan. */
int eu3d_set_wedge(eu3d_handle *h, double x0, double y0, double tan_angle, int enabled);

int eu3d_set_dt(eu3d_handle *h, double dt);   /* Flowfield::dt */
int eu3d_set_time(eu3d_handle *h, double t);  /* Flowfield::time */
int eu3d_get_dt(eu3d_handle *h, double *dt);

/* Flowfield::CFLcondition, src/Flowfield.cpp:242-272 (device reduction;
   dt_out may be NULL to keep the result on the device) */
int eu3d_cfl(eu3d_handle *h, double cfl, double final_time, double *dt_out);
/* FieldBoundary_3dRSBI / _3dODM, src/Flowfield.cpp:378-773, plus the
   transmissive and wedge fills (new) */
int eu3d_boundary(eu3d_handle *h, int kind);
/* Flowfield::Advection(TimeAdv, Diff), src/Flowfield.cpp:1096-1128, with
   Flowfield::AUSM x3 (:1330-1502), MUSCL_1/MUSCL_2 (include/Differ.hpp:110-238)
   and TimeAdv::EE / TVD_RK3 (src/TimeAdv.cpp:29-67): fills RHS */
int eu3d_advection(eu3d_handle *h, int timeadv, int diff);
/* Flowfield::Update_after_Adv, src/Flowfield.cpp:1140-1157 */
int eu3d_update_after_adv(eu3d_handle *h);
/* Flowfield::Update_after_CS, src/Flowfield.cpp:1246-1284 (with Get_temp :1542-1566) */
int eu3d_update_after_cs(eu3d_handle *h);
/* Euler::IMEX = Reaction::Diagonalized + Flowfield::Update_IMEX (+ GetPartial_T),
   src/Euler.cpp:748-760, src/Reaction.cpp:736-811, src/Flowfield.cpp:1215-1234, :1578-1595 */
int eu3d_react_imex(eu3d_handle *h);
/* Euler::Trapezoid(type), src/Euler.cpp:357-737: Update_after_Adv, then
   Reaction::Trapezoid field form (type 0, src/Reaction.cpp:412-485) + Explicit(),
   or TrapezoidPrediction + per-cell substeps (type 1, :489-670) on the device
   work queue */
int eu3d_react_trapezoid(eu3d_handle *h, int type);
/* FP64 adaptive chemistry (new): the closed-reactor chemistry increment of
   each cell over dt, integrated with species-diagonal implicit substeps (the
   composition part of Reaction::Diagonalized's Jacobian, src/Reaction.cpp:
   736-811) and a decode after each, projected to element conservation and
   added with the flux residual.  Substep h: largest with h |CMS_s| <= rel
   (rho_s + 1e-9 rho) for all s and h MD_s <= amp where MD_s > 0, at least
   dt / nmax (defaults rel 0.02, amp 0.5, nmax 1024).  The reference's
   one-step IMEX and adaptive trapezoid diverge through H2-air ignition at the
   time steps of its detonation cases; this integrator does not, and it is
   the learned surrogate's teacher and fallback.  Needs the element
   composition: atoms (3, NS) = H, O, N atoms per species. */
int eu3d_set_elements(eu3d_handle *h, const double *atoms);
int eu3d_set_adaptive(eu3d_handle *h, double rel, double amp, int nmax);
int eu3d_react_adaptive(eu3d_handle *h);
/* One pass of Euler::Computing's loop body, src/Euler.cpp:266-333 (CFL, ghost
   fill, advection, chemistry), recorded once and replayed as a CUDA graph. */
int eu3d_step(eu3d_handle *h, const eu3d_step_desc *s);
/* nsteps passes; stops early once time reaches final_time (checked on the host
   after each step only when check_time is nonzero). */
int eu3d_run(eu3d_handle *h, const eu3d_step_desc *s, int nsteps, int check_time);
int eu3d_synchronize(eu3d_handle *h);
/* x-slab decomposition (replaces Flowfield::Mpi_Boundary, src/Flowfield.cpp:775-1083,
   and the MPI_Reduce/MPI_Bcast of dt in CFLcondition, :242-272).  One handle per rank
   holds a slab of the x extent; the caller moves the buffers between ranks with its
   collective library (NCCL send/recv over NVLink) on the handle's stream (eu3d_stream).
   A step of a rank, as eu3d_step does it on one rank:
     eu3d_cfl_local; all-reduce MIN of the double at eu3d_dt_device across ranks;
     eu3d_advance_time;
     eu3d_boundary; halo exchange; [wedge set: eu3d_wedge_fill; halo exchange];
     eu3d_step_part(STAGE1);
     SSP-RK2/RK3: eu3d_boundary; halo exchange; [wedge ...]; eu3d_step_part(STAGE2);
     SSP-RK3: eu3d_boundary; halo exchange; [wedge ...]; eu3d_step_part(STAGE3);
     eu3d_step_part(REACT).
   Halo exchange: eu3d_halo_pack(side) into a device buffer of eu3d_halo_bytes bytes,
   send it to the neighbour on that side, receive the neighbour's buffer and
   eu3d_halo_unpack(side) it.  Side 0 is the low-x face, 1 the high-x face; a pack
   takes the two interior planes next to the face, an unpack fills the face's two
   ghost planes (all y and z, ghosts included; primitives, T and E).  overlap 0:
   slabs partition the cells; overlap 1: neighbouring slabs share their end node, as
   the reference's mesh blocks do (src/Mesh.cpp:77-93), and the pack skips it
   (Mpi_Boundary sends planes bc+1, bc+2 and ni-1, ni).  Buffers are device memory,
   16-byte aligned. */
int eu3d_halo_bytes(eu3d_handle *h, long long *bytes);
int eu3d_halo_pack(eu3d_handle *h, int side, int overlap, void *dst);
int eu3d_halo_unpack(eu3d_handle *h, int side, const void *src);
/* CFLcondition without the time update: the rank's dt (clipped to final_time) into
   the device scalar at eu3d_dt_device; eu3d_advance_time then adds it to time. */
int eu3d_cfl_local(eu3d_handle *h, double cfl, double final_time);
double *eu3d_dt_device(eu3d_handle *h);
int eu3d_advance_time(eu3d_handle *h);
/* the immersed-wedge ghost band alone (eu3d_boundary runs it after the faces) */
int eu3d_wedge_fill(eu3d_handle *h);
/* the parts of eu3d_step after its CFL and first ghost fill */
#define EU3D_PART_STAGE1 0 /* advection (SSP-RK: with the stage-1 update and decode; the stage's
                              conserved state is held apart and CS keeps CS^n until the last stage) */
#define EU3D_PART_STAGE2 1 /* SSP-RK2/RK3 stage 2: advection, update, decode */
#define EU3D_PART_REACT 2  /* chemistry */
#define EU3D_PART_STAGE3 3 /* SSP-RK3 stage 3: advection, update, decode */
/* the adaptive trapezoid (react TRAPEZOID, type 1, work queue on) in two halves, for load
   balancing between them: PREDICT = Update_after_Adv + TrapezoidPrediction, counts binned;
   WORK = the substeps of every cell not packed away (eu3d_dlb_pack) since PREDICT.
   PREDICT then WORK equals REACT. */
#define EU3D_PART_CHEM_PREDICT 4
#define EU3D_PART_CHEM_WORK 5
/* the learned chemistry (react SURROGATE) in two halves, for load balancing of its FP64
   fallback (new): SUR_PREDICT = the flux update (unless the stages left it decoded), the
   frozen-chemistry gate, the network and its apply, ending with the fallback list;
   SUR_WORK = the fallback integration of the list slots kept (all of them unless
   eu3d_sdlb_pack sent some away).  SUR_PREDICT then SUR_WORK equals REACT. */
#define EU3D_PART_SUR_PREDICT 6
#define EU3D_PART_SUR_WORK 7
int eu3d_step_part(eu3d_handle *h, const eu3d_step_desc *s, int part);

/* Dynamic load balancing of the adaptive trapezoid across ranks (replaces the reference's
   DynamicLoadBalancer, include/LoadBalance.hpp:10-47, src/LoadBalance.cpp:8-159, and its use in
   Euler::Trapezoid, src/Euler.cpp:380-700).  A rank's load is the sum of its cells' predicted
   substep counts (React.Nchem.SumNoBoundary, src/Euler.cpp:392).  Per step, on every rank:
     eu3d_step_part(CHEM_PREDICT); eu3d_chem_load -> all-gather the loads;
     eu3d_dlb_plan (same result on every rank); the transfers whose sender is this rank:
     eu3d_dlb_select -> cells per transfer (tell each receiver its count);
     eu3d_dlb_pack into a device buffer of EU3D_DLB_OUT_FIELDS doubles per cell, one segment per
     transfer in plan order; send each segment to its receiver;
     eu3d_step_part(CHEM_WORK);
     receivers: eu3d_dlb_guest on the received segments (in plan order) -> results, sent back;
     senders: eu3d_dlb_unpack of the returned segments (same order and sizes, EU3D_DLB_BACK_FIELDS
     doubles per cell).
   The result equals the step without balancing bit for bit.  Packets are field-major per
   segment: out CS[13], T, count; back CS[13], T, E, the 16 primitives, count (-1: a solid cell,
   carried but not integrated).  All buffers are device memory; the calls run on the handle's
   stream, eu3d_chem_load synchronises it. */
#define EU3D_DLB_OUT_FIELDS 15
#define EU3D_DLB_BACK_FIELDS 32
#define EU3D_DLB_MAX_TRANSFERS 64 /* per rank and direction */
/* DynamicLoadBalancer::DLBPriorityQueue (src/LoadBalance.cpp:8-59): transfers (sender,
   receiver, amount) in the reference's order; *ntransfers is set even when cap is too small
   (EU3D_ERR_ARG).  Host only. */
int eu3d_dlb_plan(const long long *loads, int nranks, int cap, int *sender, int *receiver, long long *amount,
                  int *ntransfers);
/* the row picker of eu3d_dlb_select on host arrays: from row 0, each transfer takes
   consecutive rows while their summed load stays within its amount; bounds: npacks + 1 row
   boundaries, moved: the load each transfer takes.  Host only. */
int eu3d_dlb_select_rows(const long long *rowload, long long nrows, int npacks, const long long *amount,
                         long long *bounds, long long *moved);
/* sum of the predicted substep counts of the handle's fluid cells (after CHEM_PREDICT) */
int eu3d_chem_load(eu3d_handle *h, long long *load);
/* picks the rows of this rank's transfers (amounts in plan order); cells and moved per transfer */
int eu3d_dlb_select(eu3d_handle *h, int ntransfers, const long long *amount, long long *cells, long long *moved);
int eu3d_dlb_pack(eu3d_handle *h, double *dev_out);
/* integrates received cells: nseg segments of seg_cells[s] cells each, concatenated in dev_in;
   writes the return segments, concatenated in the same order, to dev_back */
int eu3d_dlb_guest(eu3d_handle *h, int nseg, const long long *seg_cells, const double *dev_in, double *dev_back);
int eu3d_dlb_unpack(eu3d_handle *h, const double *dev_back);

/* Load balancing of the learned chemistry's FP64 fallback across ranks (new: the reference
   has no learned chemistry; the protocol is the one above, with the fallback list in place
   of the trapezoid's rows).  The rejected and audited cells gather at the detonation front,
   so the slabs it crosses carry most of the fallback.  A rank's load is the length of its
   fallback list.  Per step, on every rank:
     eu3d_step_part(SUR_PREDICT); eu3d_sur_load -> all-gather the loads; eu3d_dlb_plan;
     senders: eu3d_sdlb_select (cells per transfer, taken from the end of the list) and
     eu3d_sdlb_pack (EU3D_SDLB_OUT_FIELDS doubles per cell, segments in plan order);
     eu3d_step_part(SUR_WORK) on the slots kept;
     receivers: eu3d_sdlb_guest -> EU3D_SDLB_BACK_FIELDS doubles per cell, sent back;
     senders: eu3d_sdlb_unpack.
   Packets are field-major per segment: out CS[13], T, the audit temperature, the list
   flags; back CS[13], T, E, the 16 primitives.  The result equals the unbalanced step bit
   for bit; the receivers' status counts the fallback work they did.  Device buffers, the
   handle's stream; eu3d_sur_load synchronises it. */
#define EU3D_SDLB_OUT_FIELDS 16
#define EU3D_SDLB_BACK_FIELDS 31
/* the fallback list length after SUR_PREDICT */
int eu3d_sur_load(eu3d_handle *h, long long *load);
/* cells per transfer (amounts in plan order), taken as consecutive list slots from its end;
   EU3D_ERR_STATE unless eu3d_sur_load ran after the step's SUR_PREDICT */
int eu3d_sdlb_select(eu3d_handle *h, int ntransfers, const long long *amount, long long *cells);
int eu3d_sdlb_pack(eu3d_handle *h, double *dev_out);
int eu3d_sdlb_guest(eu3d_handle *h, int nseg, const long long *seg_cells, const double *dev_in, double *dev_back);
int eu3d_sdlb_unpack(eu3d_handle *h, const double *dev_back);

/* Launch settings picked per handle (new): z planes walked by one flux block
   (default: 64, halved while the flux grid has fewer than four waves),
   adaptive trapezoid on the persistent work queue (1) or one thread per cell
   (0), resident queue blocks per SM, and how the FP32 flux kernel reads the
   primitives: 2 (default) tile planes brought into a shared-memory ring by
   TMA, 1 staged into shared memory by loads, 0 read through L1.  flux_stage
   2 needs the driver's tensor-map encoder and falls back to 1 without it.
   sur_fused 1: the surrogate's network and its apply in one kernel; 0
   (default, faster on B200): two kernels; the same decisions either way.
   adapt_queue 1: the FP64 adaptive chemistry (EU3D_REACT_ADAPTIVE) lists the
   fluid cells and integrates them on the persistent queue, one cell per lane
   with refill; 0 (default): one thread per cell.  cell_blocks (3, default,
   or 4): resident blocks of 128 threads per SM the SSP-RK2 stage updates of
   the FP32-flux path are compiled for (more blocks, fewer registers a
   thread; the same results).  gate_fused (1, default): in an SSP-RK2 step
   with the learned chemistry and its frozen-chemistry gate on, the gate runs
   inside stage 2 on the state the stage has just decoded, instead of as a
   kernel of its own that reads T and the radicals back (0); the same list
   and results.  Changing them drops the recorded step graphs. */
typedef struct {
    int flux_kz;
    int chem_queue;
    int queue_blocks;
    int flux_stage;
    int sur_fused;
    int adapt_queue;
    int cell_blocks;
    int gate_fused;
} eu3d_tuning;
int eu3d_set_tuning(eu3d_handle *h, const eu3d_tuning *t);
/* Bound of the waits of the TMA-fed flux kernel for its plane copies (new), in
   sleep-waits of about a microsecond each (default 524288, about half a
   second; at most 2^24).  A wait that runs out makes the kernel count
   eu3d_status.wait_timeouts, wait with the default bound for the copies it
   has in flight and return without storing the rest of its residuals; 0
   gives up at the first wait, which tests that path without a fault or a
   hang.  The residuals of such a launch are incomplete.  Drops the recorded
   step graphs. */
int eu3d_set_wait_limit(eu3d_handle *h, long long tries);
int eu3d_get_tuning(eu3d_handle *h, eu3d_tuning *t);
/* Autotuner: times `steps` steps of s for each candidate setting (flux_kz in
   {4, 8, 16, 32, 64}, the three FP32 flux kernels; for the adaptive
   trapezoid also the queue on/off and 2..4 blocks per SM; for the FP64
   adaptive chemistry adapt_queue on/off; for SSP-RK2 with FP32 flux the
   stage updates' cell_blocks 3, 4) on the handle's current state,
   restoring the state after
   each trial, and keeps the fastest.  best / best_ms may be NULL.  Needs
   temporary device memory for one copy of the state. */
int eu3d_autotune(eu3d_handle *h, const eu3d_step_desc *s, int steps, eu3d_tuning *best, double *best_ms);

/* Per-kernel timing with CUDA events on the handle's stream (replaces the
   reference's MPI_Wtime phase timers, src/Euler.cpp:256-344).  While enabled,
   eu3d_step launches its kernels directly instead of replaying its graph.
   eu3d_profile_read synchronises, then reports per kernel name (newline
   separated in `names`) the summed milliseconds and launch counts since the
   previous read. */
int eu3d_profile_enable(eu3d_handle *h, int on);
int eu3d_profile_read(eu3d_handle *h, char *names, size_t names_cap, double *ms, long long *counts,
                      int max_kernels, int *n_out);
/* Euler::Output (src/Euler.cpp:792-973): the rank's Tecplot block file at `path`
   (the caller picks the name; the reference uses output_<n>/results/Series<react><num>_<rank>.dat
   for one rank and output_<n>/results<react><num>_<rank>.dat for several).  Header
   "Variables = X,Y,Z,T,D,P,U,V,Ma,Y1,...,Y7,L,WaitTime", "ZONE I=ni<TAB>J=nj<TAB>K=nk",
   "datapacking=block", then 18 blocks over the interior cells, k outer, i inner, one
   value per line as std::ostream prints them (%.6g; L, the substep counts, as
   integers; WaitTime the caller's wait_time).  The fields are gathered on the device
   and copied to pinned host memory before the call returns; background != 0 formats
   and writes on a host thread while the caller steps on, and eu3d_write_wait returns
   its outcome (a new write waits for the previous one). */
int eu3d_write_tecplot(eu3d_handle *h, const char *path, double wait_time, int background);
int eu3d_write_wait(eu3d_handle *h);
/* The same file from host arrays (no device): ghosted node coordinates, 13 x ni*nj*nk
   columns T D P U V Ma Y1..Y7 and the counts L, both in the file's cell order. */
int eu3d_tecplot_write_host(const char *path, int ni, int nj, int nk, int bc, const double *xnode,
                            const double *ynode, const double *znode, const double *cols, const int *lcol,
                            double wait_time);
/* Status counters; a D/T NaN scan replaces D.IsNan()/T.IsNan() (src/Euler.cpp:319-331). */
int eu3d_get_status(eu3d_handle *h, eu3d_status *st);
int eu3d_reset_status(eu3d_handle *h);

/* CFL time step that allocates nothing (no counterpart in the reference).
   For callers that cannot allocate device memory -- code running while
   another framework owns the memory pool and forbids allocations, or code
   that must not call cudaMalloc/cudaFree because they synchronise the device.
   The caller passes FP64 device fields D, U, V, W, P, Gamma on the ghosted
   grid (index k*plane + j*pitch + i, x fastest) and caller-owned device
   doubles time_inout and dt_out.  The result: dt = cfl * the minimum over
   every interior cell of min(dx/(|U|+C), dy/(|V|+C)[, dz/(|W|+C) if use_z]),
   C = sqrt(Gamma P / D), shortened so that time + dt does not pass
   final_time; then time += dt.  Every interior cell counts: the caller's
   fields carry no wedge, so unlike eu3d_cfl on a handle with eu3d_set_wedge,
   solid cells are not left out.
   Scratch: a fixed 1024-double device array inside the library (kept by every
   GPU that loads it until exit); nblocks (reduction blocks, 0 = 592) above
   1024 is rejected with EU3D_ERR_ARG.  The first call on a device looks up
   that array's device address with the device current, so make it before any
   stream capture.  All calls share the array: calls that overlap on the GPU
   race.  Work is queued on `stream` (a cudaStream_t; NULL = default stream)
   and the call does not synchronise. */
int eu3d_cfl_noalloc(const double *D, const double *U, const double *V, const double *W, const double *P,
                     const double *Gamma, int ni, int nj, int nk, int bc, long long pitch, long long plane,
                     double dx, double dy, double dz, int use_z, double cfl, double final_time,
                     double *time_inout, double *dt_out, int nblocks, void *stream);

/* Learned chemistry surrogate (new; the reference's "DNN" mode has no model,
   src/Euler.cpp:773-780).  Tensor-core GEMM used by the surrogate's training:
   C (M x N, f32, row-major) = [C +] A B^T with A (M x K) and B (N x K) bf16
   row-major, all device pointers; M % 128 == 0, N % 16 == 0 with 16 <= N <= 256,
   K % 16 == 0.  *err (device int, may be NULL) is set when a tensor-core wait
   ran out of its bound.  Queued on `stream`, no synchronisation. */
int eu3d_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int accumulate, int *err,
                   void *stream);

/* ---- Learned chemistry surrogate (new; no counterpart in the reference) ----
   An MLP 12 -> 128 -> 128 -> 128 -> 10 (GELU), BF16 weights, FP32
   accumulation on the tensor cores, maps a cell's (T, ln p, Y_k, ln dt) to the
   chemistry increment (dY_k, dT) over dt.  Its training set lives on the
   device: sampled states (T, p, Y_k, dt in FP64) labelled by the project's
   own FP64 integrators.  Parameters: flat FP32 vector of EU3D_SUR_NPARAM
   values, W1[16][128] b1[128] W2[128][128] b2[128] W3[128][128] b3[128]
   W4[128][16] b4[16] (W[in][out]; rows 12..15 of W1 take the padded inputs,
   columns 10..15 of W4 are unused).  Normalisation / acceptance vector: float
   [EU3D_SUR_NORM_LEN] with the offsets below. */
#define EU3D_SUR_NPARAM 37264
#define EU3D_SUR_NORM_LEN 80
#define EU3D_SUR_N_IN_MEAN 0    /* 12 raw-feature means: T, ln(p/atm), Y_0..8, ln dt */
#define EU3D_SUR_N_IN_STD 12    /* 12 raw-feature scales */
#define EU3D_SUR_N_OUT_MEAN 24  /* 10 target means (asinh space) */
#define EU3D_SUR_N_OUT_STD 34   /* 10 target scales */
#define EU3D_SUR_N_LIN 44       /* 10 asinh linear scales */
#define EU3D_SUR_N_TA 54        /* activity temperature Ta [K] (0: no activity scaling) */
#define EU3D_SUR_N_TR 55        /* activity reference temperature Tr [K] */
#define EU3D_SUR_N_ENV 56       /* envelope: T_lo, T_hi, lnp_lo, lnp_hi, lndt_lo, lndt_hi */
#define EU3D_SUR_N_RATIO 62     /* element ratios H/O, N/O of the training set */
#define EU3D_SUR_N_RATIO_TOL 64 /* relative tolerance on those ratios */
#define EU3D_SUR_N_RES_ABS 65   /* energy-residual tolerance [K] ... */
#define EU3D_SUR_N_RES_REL 66   /* ... plus this fraction of |dT| */
#define EU3D_SUR_N_NEG_TOL 67   /* most negative mass fraction accepted (then clipped to 0) */
#define EU3D_SUR_N_PROJ_EPS 68  /* weight floor of the element projection */
#define EU3D_SUR_N_DT_MAX 69    /* largest |dT| accepted from the network [K] */
#define EU3D_SUR_N_DELTA 70     /* > 0: relative targets dY_k / (Y_k + delta), dT / T; 0: absolute */

/* Surrogate bound to h's device, quirk policy and mechanism; atoms: (3, NS)
   counts of H, O, N atoms per species; capacity: training samples. */
int eu3d_sur_create(eu3d_handle *h, long long capacity, const double *atoms, eu3d_surrogate **out);
int eu3d_sur_destroy(eu3d_surrogate *s);
int eu3d_sur_reset_dataset(eu3d_surrogate *s);
int eu3d_sur_dataset_size(eu3d_surrogate *s, long long *n);
/* n random states: T uniform in [env0, env1] K, ln(p/atm) in [env2, env3],
   ln dt in [env4, env5], composition at the element ratios of stoichiometric
   H2-air; species: indices of H, O, H2O, OH, O2, H2, H2O2, HO2, N2. */
int eu3d_sur_add_random(eu3d_surrogate *s, long long n, const double *env, const int *species,
                        unsigned long long seed);
/* n samples of src's interior cells (offset, offset + stride, ...): T, p, Y
   with T scaled by 1 + jitter_T u, p by exp(jitter_lnp u), u uniform in
   [-1, 1], and ln dt uniform in [lndt_lo, lndt_hi]. */
int eu3d_sur_add_snapshot(eu3d_surrogate *s, eu3d_handle *src, long long n, long long stride, long long offset,
                          double jitter_T, double jitter_lnp, double lndt_lo, double lndt_hi,
                          unsigned long long seed);
/* FP64 labels of every sample: kind EU3D_REACT_IMEX (one closed-reactor
   Diagonalized + Update_IMEX step, src/Reaction.cpp:736-811,
   src/Flowfield.cpp:1215-1234) or EU3D_REACT_TRAPEZOID (TrapezoidPrediction
   substeps, src/Reaction.cpp:489-670, at most cap), projected to element
   conservation (weight floor proj_eps) and decoded at constant density and
   energy.  n_valid (may be NULL) counts the usable samples. */
int eu3d_sur_label(eu3d_surrogate *s, int kind, int cap, double proj_eps, long long *n_valid);
/* rows [first, first + count) of the states (12 doubles), raw features and
   raw labels (12 floats each); any output may be NULL */
int eu3d_sur_get_dataset(eu3d_surrogate *s, long long first, long long count, double *states, float *X, float *L);
int eu3d_sur_set_norm(eu3d_surrogate *s, const float *norm);
int eu3d_sur_get_norm(eu3d_surrogate *s, float *norm);
/* parameters in and out; setting them also clears the Adam moments */
int eu3d_sur_set_params(eu3d_surrogate *s, const float *params);
int eu3d_sur_get_params(eu3d_surrogate *s, float *params);
/* steps Adam steps (beta 0.9, 0.999) on random minibatches of `batch` samples
   (a multiple of 256): linear warm-up to lr_max over `warmup` steps, then a
   cosine decay to lr_min.  losses (may be NULL): per-step MSE. */
int eu3d_sur_train(eu3d_surrogate *s, int steps, int batch, float lr_max, float lr_min, int warmup,
                   unsigned long long seed, float *losses);
/* loss and gradient (EU3D_SUR_NPARAM) for one host batch: X (batch x 16
   normalised inputs), Y (batch x 16 standardised targets, column 15 = sample
   weight); out (batch x 16, may be NULL): network outputs.  No update. */
int eu3d_sur_loss_grad(eu3d_surrogate *s, const float *X, const float *Y, int batch, float *loss, float *grad,
                       float *out);
/* inference with the fused tensor-core kernel: X (n x 16 normalised inputs)
   -> out (n x 16 outputs); host buffers (predict, synchronous) or device
   buffers on `stream` (infer, NULL = the surrogate's stream, asynchronous). */
int eu3d_sur_predict(eu3d_surrogate *s, const float *X, long long n, float *out);
int eu3d_sur_infer(eu3d_surrogate *s, const float *X_dev, long long n, float *out_dev, void *stream);
/* Use s (NULL: none) for EU3D_REACT_SURROGATE steps of h.  Every
   audit_stride-th accepted cell (0: none) also runs the FP64 integrator,
   which keeps its result and records the surrogate's temperature error. */
int eu3d_set_surrogate(eu3d_handle *h, eu3d_surrogate *s, int audit_stride);
/* Frozen-chemistry gate for EU3D_REACT_SURROGATE steps (new): a fluid cell
   colder than t_frozen [K] whose mass fractions summed over the species in
   species_mask (bit s = species s; 0: no composition test) are at most y_max
   keeps the state of its flux update and decode -- over one flow step its
   chemistry is below what the FP64 integrator resolves -- and only the other
   cells go through the network and its apply.  The radicals' mass fractions
   are summed in FP32.  About one gated cell in audit_stride (0: none; a
   fixed hash sample of the interior cell index) is integrated by the FP64
   fallback as well, which keeps its result and records the largest
   temperature change the gate ignored (eu3d_status.frozen_audit_max_dT).  t_frozen = 0 (the default) turns the
   gate off: every fluid cell takes the network.  With the gate on, sur_fused
   is ignored. */
int eu3d_set_surrogate_gate(eu3d_handle *h, double t_frozen, double y_max, unsigned species_mask, int audit_stride);
/* Learned chemistry step of h after the flux residual is in RHS: network
   increment for the previous decode's state, element projection, envelope /
   negativity / energy-residual checks, EE update + FP64 decode; rejected
   cells run the FP64 IMEX step (Euler::IMEX, src/Euler.cpp:748-760) on the
   device work queue. */
int eu3d_react_surrogate(eu3d_handle *h);

/* Pointer to the handle's CUDA stream (cudaStream_t), for callers that
   interleave their own work. */
void *eu3d_stream(eu3d_handle *h);

#ifdef __cplusplus
}
#endif
#endif
