/*
 * CPU restatement of HARM's per-step finite-volume update (test
 * infrastructure only: the oracle the GPU path is checked against).
 *
 * Layout is the reference's own (defs.h): zone-major arrays over the full
 * grid including NG = 3 ghost zones per side, i (x1) slowest, j (x2), then
 * the component.  Index (i, j) with i in [-NG, n1+NG) is stored at row
 * (i+NG) of (n1+2NG) rows, column (j+NG) of (n2+2NG).
 *
 *   prims     [n1m][n2m][8]          rho, u, u~1..3, B1..3
 *   pflag     [n1m][n2m][5]          FLAGUTOPRIMFAIL, -, BSQORHO, BSQOU, -
 *   gcov/gcon [n1m][n2m][4 loc][4][4] loc = FACE1, FACE2, CORN, CENT
 *   gdet      [n1m][n2m][4 loc]
 *   conn      [n1m][n2m][4][4][4]    Gamma^k_{l j} as conn[k][l][j]
 *   floors    [n1m][n2m][2]          rho and u floors at CENT
 */
#ifndef HARM_ORACLE_H
#define HARM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n1, n2;          /* interior zones */
  int lim;             /* 3 = MC, 4 = PARA (PPM "para4") */
  int fluxmethod;      /* 0 = LAXF (Rusanov), 1 = HLL */
  int eom;             /* 0 = GRMHD, 1 = force-free */
  double cour, gam, dx1, dx2;
  double safe, defcon, gammamax, gammafail, bsqorholimit, bsqoulimit;
  double tf;
  int bc;              /* 0 = torus (bounds.fishmon.c), 1 = rotating star (bounds.ns.c) */
  double omegastar;    /* bc 1: angular frequency of the stellar surface */
  int fluxadjust;      /* FLUXADJUST (global.h:286-293): 0 = FLUXFIXED, 1-3 = per-zone HLL/LAXF switch */
  double gammadamp;    /* GAMMADAMP (initbase.c:215): Lorentz-factor threshold of the switch */
} ho_config;

typedef struct ho_state ho_state;

ho_state *ho_create(const ho_config *cfg, const double *gcov, const double *gcon,
                    const double *gdet, const double *conn, const double *floors);
void ho_destroy(ho_state *s);

/* One full RK2 step of the reference (step_ch.c:35-188) on prims/pflag in
   place.  t and dt are advanced as step_ch() does.  Returns 0, or a
   nonzero FAIL_* code of the reference when a fatal check fired. */
int ho_step(ho_state *s, double *prims, int *pflag, double *t, double *dt);

/* moves the end time tf of the run and redoes the clamp t + dt <= tf
   (step_ch.c:183) on the last step's unclamped dt (on *dt before any step) */
void ho_set_end_time(ho_state *s, double tf, double t, double *dt);

/* Boundary fill of a prims array (bounds.fishmon.c:14) and pre_fixup flags
   (fixup.c:1197), as init() leaves them. */
void ho_bound(ho_state *s, double *prims);
void ho_bsqflags(ho_state *s, const double *prims, int *pflag);

/* last substep's fluxes F1, F2 [n1m][n2m][8] (after flux-CT) */
void ho_get_fluxes(const ho_state *s, double *f1, double *f2);

/* horizon accounting of diag_flux() (diag.c:576-833) after the last step:
   pdot[X1DN][RHO], pdot[X1DN][UU], pdotterms[X1DN][3][UU] and [6][UU],
   pcum[X1DN][RHO], pcum[X1DN][UU] (cumulative since creation) */
void ho_get_horizon(const ho_state *s, double *out);

/* diagnostic currents, WHICHCURRENTCALC 1: ho_init_currents() is the t = 0
   call of initbase.c:653-658 on the initial state; every ho_step() then
   updates them as step_ch.c:143-156 does.  jcon [n1m][n2m][4], fcon
   [n1m][n2m][6], cfaraday [n1m][n2m][5][3] (any may be NULL). */
void ho_init_currents(ho_state *s, const double *p, double dt);
void ho_get_currents(const ho_state *s, double *jcon, double *fcon, double *cfaraday);

/* count of Newton cycle-break events since creation */
long ho_ncyclebreak(const ho_state *s);

/* single-zone inversion of an evolved U (with sqrt(-g)) at zone (i,j) */
int ho_utoprim(ho_state *s, int i, int j, const double *U, double *pr);

/* from now on, record the zone, evolved U and guess of up to max failed 2D
   inversions of the steps (inputs for the retry chain's tests) */
int ho_record_failures(ho_state *s, int max);

/* copies the recorded failures out (ij: 2 ints, U and pr: 8 doubles each per
   failure; arrays sized for the max given); returns their number */
int ho_get_failures(const ho_state *s, int *ij, double *U, double *pr);

/* the first fatal check of the last ho_step: out[0] = FAIL_* code (0 if
   none), out[1..2] = the zone or face (i, j) being worked on, as the
   reference's fail() reports it (fail.c:4-57) */
void ho_get_fail(const ho_state *s, int *out);

/* the deterministic cycle-break factor (shared with the GPU kernel) */
double ho_cycle_break_uniform(double x0, double x1, int n_iter);

#ifdef __cplusplus
}
#endif
#endif
