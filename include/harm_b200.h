/*
 * harm_b200.h -- C ABI of the B200 (sm_100a) implementation of HARM's
 * per-step finite-volume update.
 *
 * This is the drop-in boundary for the reference's
 *     int step_ch(void)                        (step_ch.c:16, global.h:1383)
 * which reads and writes the reference's globals p, pk, pflag, dt, t,
 * realnstep and the geometry tables gcov/gcon/gdet/conn (defs.h:4-309).
 * A host shim that replaces step_ch() calls harm_step() on a context that
 * holds device-resident copies of those arrays.
 *
 * Array arguments use the reference's own memory layout (defs.h) over the
 * full grid including NG = 3 ghost zones per side, n1m = n1 + 6 rows of
 * n2m = n2 + 6 zones, x2 index fastest:
 *   prims   [n1m][n2m][8]            rho, u, u~1, u~2, u~3, B1, B2, B3
 *   pflag   [n1m][n2m][5]            pflag[..][0] = FLAGUTOPRIMFAIL,
 *                                    [2] = FLAGBSQORHO, [3] = FLAGBSQOU
 *   gcov    [n1m][n2m][4][4][4]      [loc][mu][nu], loc = FACE1, FACE2,
 *   gcon    [n1m][n2m][4][4][4]      CORN, CENT (global.h:645-648)
 *   gdet    [n1m][n2m][4]
 *   conn    [n1m][n2m][4][4][4]      conn[k][l][j] = Gamma^k_{l j}
 *   floors  [n1m][n2m][2]            rho and u floors at CENT, already
 *                                    clamped below by RHOMINLIMIT/UUMINLIMIT
 *                                    (fixup.c:295-307)
 *
 * Every entry point returns 0 on success or a positive HARM_E* code; no
 * entry point aborts the process.  One context = one CUDA stream = one host
 * thread.  There is no CPU fallback: without a usable CUDA device
 * harm_create() fails with HARM_ENODEVICE.
 */
#ifndef HARM_B200_H
#define HARM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define HARM_OK 0
#define HARM_EINVAL 1        /* invalid argument or configuration */
#define HARM_ENODEVICE 2     /* no CUDA device / not sm_100 */
#define HARM_ECUDA 3         /* CUDA runtime error */
#define HARM_ENOMEM 4        /* device allocation failed */
#define HARM_EGEOMETRY 5     /* geometry tables not symmetric or not uploaded */
#define HARM_EFAIL 6         /* the step hit a fatal check of the reference
                                (fail() codes, global.h:562-579, or 20 when
                                Utoprim_ffde met a space-like drift velocity,
                                phys.ffde.c:281-284); see harm_status.fail_code */

/* limiter / Riemann solver / equations of motion (step_ch.h:22-80) */
#define HARM_LIM_MC 3
#define HARM_LIM_PARA 4
#define HARM_FLUX_LAXF 0
#define HARM_FLUX_HLL 1
#define HARM_EOM_GRMHD 0
#define HARM_EOM_FFDE 1      /* force-free electrodynamics (phys.ffde.c) */

/* boundary set of the problem (the bounds*.c plugin) */
#define HARM_BC_TORUS 0      /* bounds.fishmon.c: OUTFLOW at both x1 ends,
                                polar mirror with POLEDEATH */
#define HARM_BC_STAR 1       /* bounds.ns.c: rotating stellar surface inside
                                (NSSURFACE), extrapolating OUTFLOW outside,
                                plain polar mirror */

/* arithmetic of the step */
#define HARM_PREC_FP64 0   /* everything FP64: bit-identical to the reference */
#define HARM_PREC_MIXED 1  /* reconstruction, wavespeeds and face fluxes in FP32 (FP32 face
                              geometry and flux storage); con-to-prim, conserved update,
                              geometric source, EMF and dt in FP64 */

/* Run-time knobs of the reference (initbase.c:119-243 and the problem's
   init_global), plus the grid size that the reference fixes at compile time
   (global.h:126-127). */
typedef struct harm_config {
  int n1, n2;           /* interior zones */
  int lim;              /* HARM_LIM_MC or HARM_LIM_PARA */
  int fluxmethod;       /* HARM_FLUX_HLL or HARM_FLUX_LAXF */
  int eom;              /* HARM_EOM_GRMHD or HARM_EOM_FFDE */
  int precision;        /* HARM_PREC_FP64 or HARM_PREC_MIXED */
  double cour;          /* Courant factor */
  double gam;           /* adiabatic index */
  double dx1, dx2;      /* uniform coordinate spacings dx[1], dx[2] */
  double safe;          /* SAFE: max dt growth per step */
  double defcon;
  double gammamax;      /* GAMMAMAX */
  double gammafail;     /* GAMMAFAIL */
  double bsqorholimit;  /* BSQORHOLIMIT */
  double bsqoulimit;    /* BSQOULIMIT */
  double tf;            /* end time: dt is clamped so that t + dt <= tf (a zeroed
                           config has tf = 0, which stops a run at t = 0) */
  int bc;               /* HARM_BC_TORUS or HARM_BC_STAR */
  double omegastar;     /* HARM_BC_STAR: angular frequency of the surface
                           (Omegastar, bounds.ns.c:107) */
  int currents;         /* 1: the diagnostic currents J^mu and the Faraday
                           tensor F^{mu nu} every step, as step_ch.c:143-156
                           does (WHICHCURRENTCALC 1); 0: not computed */
  int tryagain;         /* 1: the UTOPRIMTRYAGAIN retry chain (global.h:213,
                           step_ch.c:608-626): a zone whose 2D inversion fails
                           is inverted again by 5D1, 2D, 1D, 1D_OPT, 1D_FINAL,
                           2D_FINAL and 5D2_FINAL in turn until one succeeds;
                           0: the 2D inversion only (GRMHD only) */
  int fluxadjust;       /* FLUXADJUST (global.h:286-293): 0 FLUXFIXED, every face
                           uses fluxmethod; 1 FLUXBSQORHO, 2 FLUXBSQOU, 3
                           FLUXBSQORHOANDU: per zone, the hydro variables of
                           the faces a zone owns switch one step down from
                           fluxmethod (HLL -> LAXF) where b^2/rho >
                           bsqorholimit, b^2/u > bsqoulimit or the Lorentz
                           factor > 2 gammadamp (get_bsqflags' FLAGREALFLUX,
                           fixup.c:1236-1290; choose_flux with
                           HYDROFLUXADJUSTONLY 1, step_ch.c:703-738).  The
                           reference decides alike for 1, 2 and 3. */
  double gammadamp;     /* GAMMADAMP (initbase.c:215 sets 5.0); read only when
                           fluxadjust != 0, and must then be > 0 */
} harm_config;

typedef struct harm_status {
  int fail_code;                 /* reference fail() code, 0 if none */
  int fail_i, fail_j;            /* zone of the first fatal check: of the kernels
                                    that reported one, the first in the reference's
                                    order of the step (x1 faces, x2 faces, update,
                                    bound, repairs, bound; per substep), the first
                                    zone of that pass in its loop order (i outer,
                                    j inner) -- the zone and code the reference's
                                    fail() reports (fail.c:4-57) for that state,
                                    independent of thread scheduling */
  int fixups;                    /* zones repaired by fixup_utoprim since harm_set_time */
  long long realnstep;
  double t, dt;                  /* time and the next step's dt */
  unsigned long long newton_iters; /* Newton iterations since harm_set_time */
  int chk_multi;                 /* substeps since harm_set_time whose check-solution
                                    sweep (fixup.c:388-488) needed more than one
                                    parallel round */
  int deferred;                  /* inversions since harm_set_time that needed more
                                    than 16 Newton iterations (redone by the tail
                                    kernel with the reference's limit of 200) */
  long long fail_step;           /* realnstep at the start of the step whose fatal
                                    check is reported (-1 if none) */
} harm_status;

typedef struct harm_ctx harm_ctx;

/* Allocates the device state for cfg on `stream` (a cudaStream_t, or NULL
   for the default stream). */
int harm_create(const harm_config* cfg, void* stream, harm_ctx** out);

/* Uploads the geometry tables computed by set_grid() (set_grid.c:6-89) and
   the per-zone floors; once, before the first step. */
int harm_upload_geometry(harm_ctx* ctx, const double* gcov, const double* gcon, const double* gdet,
                         const double* conn, const double* floors);

/* Host -> device copy of p (and pflag, may be NULL) from the reference
   layout; also resets the device copy of fixup_checksolution's gammacheck
   table when reset_gammacheck != 0 (fixup.c:393 keeps it static). */
int harm_set_prims(harm_ctx* ctx, const double* prims, const int* pflag, int reset_gammacheck);

/* Device -> host copy of p and pflag (either may be NULL). */
int harm_get_prims(harm_ctx* ctx, double* prims, int* pflag);

/* Fills the ghost zones of the device state as bound_prim() does
   (bounds.fishmon.c:14-330 with the torus's POLEDEATH zeroing of the first
   and last active rows, or bounds.ns.c:10-355 for HARM_BC_STAR), e.g. after
   uploading an unbounded state. */
int harm_bound_prims(harm_ctx* ctx);

/* Sets t, dt and realnstep (as init() or a restart leaves them). */
int harm_set_time(harm_ctx* ctx, double t, double dt, long long realnstep);

/* Changes the end time tf of the run, e.g. to stop at a diagnostic time
   and continue.  The clamp t + dt <= tf (step_ch.c:183) is redone on the
   unclamped next dt, so a run that stopped at the old end time moves on;
   the state and the horizon accumulators are kept. */
int harm_set_end_time(harm_ctx* ctx, double tf);

/* One con-to-prim method of the reference's Utoprimgen_pick
   (step_ch.c:583-600): which = 0 5D1, 2 2D, 3 1D, 4 1D_OPT, 5 1D_FINAL,
   6 2D_FINAL, 7 5D2_FINAL (the ids of step_ch.h:39-53), or -1 for the
   whole Utoprimgen with the UTOPRIMTRYAGAIN retry chain (step_ch.c:468-640),
   run on the device at nz active zones: zones holds (i, j) pairs, U the
   evolved conserved vectors (8 per zone, with sqrt(-g), as the update
   forms them), pr the guesses in and the results out (8 per zone), pflag
   the codes out.  Host arrays; synchronous.  GRMHD only. */
int harm_invert_zones(harm_ctx* ctx, int which, int nz, const int* zones, const double* U, double* pr, int* pflag);

/* Enqueues nsteps full steps of step_ch() on the context's stream
   (asynchronous; the first call captures a CUDA graph of one step). */
int harm_step(harm_ctx* ctx, int nsteps);

/* Waits for the stream and reports the run state; returns HARM_EFAIL when a
   fatal check fired. */
int harm_sync(harm_ctx* ctx, harm_status* st);

/* Host copies of the last substep's F1, F2 after fix_flux and flux-CT, in
   the reference layout [n1m][n2m][8] (what diag_flux() reads). */
int harm_get_fluxes(harm_ctx* ctx, double* F1, double* F2);

/* Horizon accounting of the reference's diag_flux() (diag.c:576-833) for
   the inner x1 face of the whole grid, computed on the device every step:
   out[0..5] = pdot[X1DN][RHO], pdot[X1DN][UU] (face fluxes of the last step
   in diagnostic form, summed over x2), pdotterms[X1DN][3][UU] and
   pdotterms[X1DN][6][UU] (the b^2 u^r u_t and -b^r b_t parts of the energy
   flux from the zone-centred state), pcum[X1DN][RHO], pcum[X1DN][UU]
   (sum of pdot * dt since harm_set_time). */
int harm_get_horizon(harm_ctx* ctx, double* out);

/* Diagnostic currents of a context created with currents = 1, in the
   reference's layouts (phys.c:1124-1455): jcon [n1m][n2m][4] (J^mu at zone
   centres, the outermost ghost ring left 0), fcon [n1m][n2m][6]
   (F^{tr}, F^{th}, F^{tp}, F^{rh}, F^{rp}, F^{hp}), cfaraday
   [n1m][n2m][5][3] (the five time/space slots of current_precalc); any
   pointer may be NULL.  harm_set_time() performs the t = 0 evaluation of
   initbase.c:653-658 on the uploaded state. */
int harm_get_currents(harm_ctx* ctx, double* jcon, double* fcon, double* cfaraday);

/* Dump files (dump.c:24-191).  The scalars of the dump header that the step
   itself does not know (the coordinate plugin's parameters). */
typedef struct harm_dump_header {
  double startx1, startx2;  /* startx[1], startx[2] */
  double a;                 /* black-hole spin */
  double R0, Rin, Rout, hslope;
  int defcoord;
} harm_dump_header;

/* Writes the reference's text dump file (dump(): dump_header + dump_content
   through dump_gen with TEXTOUTPUT, dump.c:24-191, 641-960) of the device
   state to `path`: one header line (t, N1, N2, startx, dx, realnstep, gam,
   a, R0, Rin, Rout, hslope, dt, defcoord) and one line per active zone, x1
   fastest, of 56 "%21.15g " columns: i, j, X1, X2, r, th, p (8), divb, u^mu,
   u_mu, b^mu, b_mu, vmin/vmax in x1 and x2, sqrt(-g), J^mu, J_mu, F^{mu nu},
   F_{mu nu}.  coords [n1m][n2m][4] holds X1, X2, r, th at zone centres (the
   coordinate plugin's coord()/bl_coord()).  Needs a context created with
   currents = 1 (the current columns).  Returns HARM_EFAIL if a wavespeed
   evaluation failed (the reference's dump aborts there). */
int harm_write_dump(harm_ctx* ctx, const char* path, const harm_dump_header* hdr, const double* coords);

/* Thread-block shapes of the step's kernels (k_flux's is fixed: one warp
   along x1 by 4 rows).  update: k_update, at most 128 threads; small: the
   flag, EMF, boundary, check-solution and repair kernels, at most 1024
   threads.  Default 32 x 4 for both.  Changing them re-captures the step. */
typedef struct harm_tiles {
  int update_x, update_y;
  int small_x, small_y;
} harm_tiles;
int harm_set_tiles(harm_ctx* ctx, const harm_tiles* tiles);
int harm_get_tiles(harm_ctx* ctx, harm_tiles* tiles);

/* Ensembles: several contexts (independent grids of any sizes, e.g. tori of
   different resolutions and parameters) advanced together.  One step of
   the ensemble is one CUDA graph launch holding every member's step as an
   independent branch, so small grids run side by side on the GPU instead of
   one after another; steps_per_launch > 1 unrolls that many steps into the
   graph.  Members keep their own state and are read with the usual calls
   after harm_ensemble_sync(); a member must not be stepped on its own
   while it belongs to an ensemble. */
typedef struct harm_ensemble harm_ensemble;
int harm_ensemble_create(harm_ctx* const* members, int n, int steps_per_launch, void* stream, harm_ensemble** out);
/* Enqueues nsteps steps of every member (nsteps a multiple of
   steps_per_launch) on the ensemble's stream. */
int harm_ensemble_step(harm_ensemble* e, int nsteps);
/* Waits for the ensemble's stream; st (may be NULL) receives n statuses.
   Returns HARM_EFAIL if any member hit a fatal check. */
int harm_ensemble_sync(harm_ensemble* e, harm_status* st);
void harm_ensemble_destroy(harm_ensemble* e);

/* Reverse mode (FP64, GRMHD, torus boundaries).  The objective of a run of
   nsteps steps from the context's state p_0 is
     J = w_mass sum_n dt_n mdot_n + w_em sum_n dt_n edot_n + <lam_final, p_N>
   with mdot_n, edot_n the horizon mass flux and EM energy flux terms of
   diag_flux() (harm_get_horizon: pdot[X1DN][RHO] and pdotterms 3 + 6 of UU)
   and lam_final (reference layout [n1m][n2m][8], may be NULL) weighting the
   active zones of the final state.  dt_n is held at the run's own values
   (the derivative does not follow the Courant minimum).

   Both first fill the ghost zones of p_0 from its active zones by the
   boundary conditions (bound_prim after init, init.fishmon.c); on a state
   left by a step this changes nothing but the inflow-checked x1 ghosts of
   the two POLEDEATH rows, which then see their row's zeroed u~2.  The
   independent variables are therefore the active zones: the ghost copies
   put the MC/PARA4 limiters at their kinks (equal neighbours), where only
   derivatives along the bound's own dependence exist.

   harm_adjoint_run: runs the nsteps forward (free dt, recorded in dts_out
   if not NULL), keeping a checkpoint every checkpoint_every steps, then the
   adjoint back to p_0: grad [n1m][n2m][8] = dJ/dp_0 on the active zones
   (ghost entries 0).  Each backward step recomputes its forward
   step from the segment's states (recording the intermediate states, the
   inversion flags and the repair choices) and runs the adjoint kernels:
   floors and Lorentz limits, the con-to-prim inverse through the implicit
   function theorem on its Jacobian, the conserved update and geometric
   source, flux-CT, the face fluxes (HLL/LAXF, wavespeeds, states) and the
   MC/PARA4 reconstructions differentiated piecewise, the repairs and the
   boundary fills.  With more than one checkpoint segment the recomputation
   of a segment runs on the context's stream while the adjoint of the
   segment after it runs on a second stream (created at the device's
   highest stream priority and destroyed by the call), from two record
   sets: device memory of about 2 x checkpoint_every
   x 10 state-sized arrays (a 16-step segment of a 512^2 grid: ~3 GB a
   set) besides one checkpoint per segment.  The context is left at p_N.
   ms_out (may be NULL): the forward and the backward wall times on the
   device.

   harm_run_fixed_dt: the same objective for nsteps steps with dt_n given
   (e.g. for finite differences against the adjoint). */
int harm_adjoint_run(harm_ctx* ctx, int nsteps, int checkpoint_every, double w_mass, double w_em,
                     const double* lam_final, double* J, double* grad, double* dts_out, double* ms_out);
int harm_run_fixed_dt(harm_ctx* ctx, const double* dts, int nsteps, double w_mass, double w_em,
                      const double* lam_final, double* J);

/* Diagnostics: runs one step outside the graph with a CUDA event after
   every kernel and returns, per kernel class (harm_kernel_name(k), k <
   HARM_NKERNELS), the summed device time in ms and the launch count. */
#define HARM_NKERNELS 15
int harm_profile_step(harm_ctx* ctx, double* ms, int* launches, int nclasses);
const char* harm_kernel_name(int k);

/* Diagnostics: the device's FP64 instruction throughput (DADD, DMUL and
   DFMA per second, out3[0..2]) from independent dependency chains on every
   SM, timed with CUDA events -- the compute ceiling of the FP64 step, whose
   kernels are built without multiply-add contraction.  No counterpart in
   the reference. */
int harm_measure_fp64_peak(double* out3);

/* One step of step_ch() that allocates nothing -- no counterpart in the
   reference.  For callers that cannot call cudaMalloc (a host code that owns
   all device memory through its own pool, or that runs where allocation is
   forbidden): the caller passes its own device buffers and the scratch of
   the step lives in a static array compiled into this library (about 1.8 MB
   per device, held until the process exits).  Limit: pitch * (n2 + 6) <=
   5632 doubles per plane, i.e. at most 64 x 64 active zones; larger grids
   are rejected with HARM_EINVAL and a message on stderr.
   Inputs/outputs are device arrays in the step's structure-of-arrays layout:
   a plane holds zone (i, j), i in [-3, n1+3), j in [-3, n2+3), at
   (j+3)*pitch + (i+3) with pitch = n1+6 rounded up to a multiple of 16;
   d_prims = 8 planes (rho, u, u~1..3, B1..3), bounded, updated in place;
   d_pflag = 1 int plane (FLAGUTOPRIMFAIL), updated; d_geo = 126 planes:
   for loc = FACE1, FACE2, CORN, CENT 10 gcov + 10 gcon (packed symmetric,
   00 01 02 03 11 12 13 22 23 33) + gdet, then 40 connection planes
   Gamma^k_{(lj)} (k*10 + packed (l,j)), then the rho and u floors.
   t and dt are host values, advanced as step_ch() does; cfg->tf must be
   after *t.  The first call on a device checks that it is an sm_100 device
   (else HARM_ENODEVICE) and looks up the array's device address
   (cudaGetSymbolAddress).  Every call waits for its stream to hand t and dt
   back, so no call may be made while its stream is being captured into a
   CUDA graph (such a call returns HARM_EINVAL and leaves the capture
   intact).  Every call shares the one array: calls that overlap on the GPU
   race.  The fixup_checksolution gamma table (static in the reference,
   fixup.c:393) carries over between calls on the same grid unless
   reset_gammacheck != 0; a call on a grid other than the previous call's
   starts it from zero.  Only cfg->precision == HARM_PREC_FP64. */
int harm_step_noalloc(const harm_config* cfg, const double* d_geo, double* d_prims, int* d_pflag, double* t,
                      double* dt, int reset_gammacheck, void* stream);

void harm_destroy(harm_ctx* ctx);

const char* harm_error_string(int code);

#ifdef __cplusplus
}
#endif
#endif
