/*
 * Constants shared by the EU3D B200 C-ABI (eu3d_gpu.h) and its oracle.
 *
 * Quirk flags.  The reference solver's arithmetic contains several defects
 * that change results.  Each flag reproduces one of them exactly when set
 * ("ref" policy, EU3D_QUIRKS_REF) and applies the evident correction when
 * clear ("fixed" policy, EU3D_QUIRKS_FIXED).
 */
#ifndef EU3D_QUIRKS_H
#define EU3D_QUIRKS_H

/* High-temperature (T >= 1000 K) enthalpy and entropy take the integration
   constants b1, b2 from the LOW range table (src/Reaction.cpp:923, :945). */
#define EU3D_Q_THERMO_B12_LOW 0x001u
/* Field trapezoid: `R_TB(r) == 1.0;` is a comparison, so reactions without
   third-body efficiencies keep R_TB = 0 (src/Reaction.cpp:449-450). */
#define EU3D_Q_TRAP_RTB_ZERO 0x002u
/* Adaptive trapezoid: `if (ip.R_TB[r] = 0.0)` assigns, so every R_TB is 0 and
   the net production rate is zero (src/Reaction.cpp:528, :634). */
#define EU3D_Q_ADAPT_RTB_ZERO 0x004u
/* AUSM copies reconstructed species states only for face index i < ni
   (src/Flowfield.cpp:1353); faces with i in [ni, ni+bc) see zero species
   states (the never-written buffer), in every sweep direction. */
#define EU3D_Q_SPECIES_FACES 0x008u
/* Field Explicit() stores total energy in the w-momentum slot and leaves the
   energy slot untouched (src/Flowfield.cpp:1183). */
#define EU3D_Q_EXPLICIT_ENERGY 0x010u
/* Update_after_Adv adds the flux residual to the species only
   (src/Flowfield.cpp:1146). */
#define EU3D_Q_ADV_SPECIES_ONLY 0x020u
/* CFLcondition ignores the z direction (src/Flowfield.cpp:254). */
#define EU3D_Q_CFL_NO_Z 0x040u
/* Update_after_CS inverts T before it recomputes E, so the Newton solve uses
   the internal energy of the PREVIOUS decode (src/Flowfield.cpp:1264-1268). */
#define EU3D_Q_STALE_E 0x080u

/* GetPartial_T adds the species enthalpy in kJ/kg to terms in J/kg
   (src/Flowfield.cpp:1590); corrected, the enthalpy is scaled to J/kg. */
#define EU3D_Q_PARTIAL_T_UNITS 0x100u

#define EU3D_QUIRKS_REF 0x1ffu
#define EU3D_QUIRKS_FIXED 0x000u

/* Ghost-fill kinds */
#define EU3D_BC_RSBI 0         /* FieldBoundary_3dRSBI, src/Flowfield.cpp:559-773 */
#define EU3D_BC_ODM 1          /* FieldBoundary_3dODM, src/Flowfield.cpp:378-558 */
#define EU3D_BC_TRANSMISSIVE 2 /* zero-gradient x ends, RSBI-style mirrors in y/z (new) */
#define EU3D_BC_NONE 3

/* Reaction schemes (include/Global.hpp:24-29 REACT) and extra modes */
#define EU3D_REACT_TRAPEZOID 0
#define EU3D_REACT_IMEX 1
#define EU3D_REACT_NONE 2      /* "DNN"/"Cantera" in the reference: no chemistry */
#define EU3D_REACT_SURROGATE 3 /* learned MLP substep with integrator fallback (new) */
#define EU3D_REACT_ADAPTIVE 4  /* FP64 adaptive species-implicit substeps (new; the surrogate's teacher) */

/* Spatial schemes (include/Global.hpp DIFF) */
#define EU3D_DIFF_MUSCL1 0
#define EU3D_DIFF_MUSCL2 1
#define EU3D_DIFF_WENO 2 /* the reference's WENO value (no scheme behind it there, src/Flowfield.cpp:1101-1109):
                            here third-order WENO, Jiang-Shu weights, epsilon 1e-6, on the same
                            three-cell stencils as MUSCL_2 (two ghost layers suffice) (new) */

/* Time schemes (include/Global.hpp ADV) */
#define EU3D_ADV_EE 0
#define EU3D_ADV_TVD_RK3 1 /* the reference's no-op: RHS is left unchanged */
#define EU3D_ADV_SSPRK2 2  /* two-stage SSP Runge-Kutta (new) */
#define EU3D_ADV_SSPRK3 3  /* three-stage SSP Runge-Kutta, Shu-Osher form (new) */

#endif
