/*
 * CPU restatement of HARM's per-step finite-volume update.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle that the CUDA path is checked
 * against.  Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * it; the product never links or calls it.
 *
 * Parity pinning: this restatement is checked against the reference itself,
 * compiled from its own sources (oracle/build_ref.py, oracle/ref_harness.c),
 * on identical seeded inputs; see tests/test_oracle_vs_reference.py.
 *
 * Every function states the reference function it restates (file:line in the
 * pseudotensor/harm_ramt tree).  The arithmetic keeps the reference's
 * evaluation order term by term (left-to-right C semantics, no contraction:
 * build with -ffp-contract=off) so that results can agree bit for bit.
 * Configuration covered: 2D, NG = 3 ghost zones, WHICHVEL = VELREL4,
 * REMOVERESTMASSFROMUU = 1, WHICHEOM = WITHGDET (e = sqrt(-g) for every
 * equation), FLUXB = FLUXCTTOTH with CORNGDETVERSION 1, BDIRCONT 1,
 * TIMEORDER 2 (midpoint RK2), UTOPRIMVERSION 2D, CHECKSOLUTION 1,
 * UTOPRIMADJUST = UTOPRIMAVG.  Physics: EOMGRMHD (Utoprim_2d) or EOMFFDE
 * (Utoprim_ffde, phys.ffde.c:141-372).  Boundaries: the torus's
 * (bounds.fishmon.c: OUTFLOW at both x1 ends, polar mirror with POLEDEATH)
 * or the rotating star's (bounds.ns.c: NSSURFACE inside, extrapolating
 * OUTFLOW outside, plain polar mirror).
 *
 * The UTOPRIMTRYAGAIN retry chain (step_ch.c:608-626) is not restated here:
 * its inversion methods are pinned directly against the reference built
 * with the chain on (oracle/build_ref.py --problem torusta).  This file
 * supplies their test inputs: ho_record_failures()/ho_get_failures() keep
 * the zone, U and guess of every 2D inversion that fails.
 */
#include "harm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NG 3
#define NPR 8
#define NFL 5
enum { RHO = 0, UU, U1, U2, U3, B1, B2, B3 };
enum { FACE1 = 0, FACE2 = 1, CORN = 2, CENT = 3 };
enum { F_FAIL = 0, F_BSQORHO = 2, F_BSQOU = 3, F_REALFLUX = 4 };
enum { LIM_MC = 3, LIM_PARA = 4 };
enum { FLUX_LAXF = 0, FLUX_HLL = 1 };

#define DBL_EPS_REF 2.2204460492503131e-16 /* global.h:710 */

/* Newton settings, utoprim_1d2d.h:1-36 with PRECISEINVERSION 1 */
#define MAX_NEWT_ITER 200
#define NEWT_TOL 1.0e-15
#define MIN_NEWT_TOL 1.0e-10
#define CYCLE_BREAK_PERIOD 10
#define W_TOO_BIG 1.e9
#define FAIL_VAL 1.e30

/* pflag codes, global.h:547-559 */
#define PF_FIXED (-1)
#define PF_CONVUTSQ 2
#define PF_CONVW 3
#define PF_CONVUTSQ2 4
#define PF_RHONEG 5
#define PF_UNEG 6
#define PF_RHOUNEG 7
#define PF_GAMMAPERC 8
#define PF_UPERC 9

/* fatal fail codes, global.h:562-579 */
#define FAIL_VCHAR_DISCR 3
#define FAIL_COEFF_NEG 4
#define FAIL_COEFF_SUP 5
#define FAIL_UTCALC_DISCR 6
#define FAIL_VSQ_NEG 9
/* Utoprim_ffde's space-like velocity (phys.ffde.c:281-284) aborts the step
   through MYFUN; it has no FAIL_* number in the reference */
#define FAIL_FFDE_SPACELIKE 20

enum { BC_TORUS = 0, BC_STAR = 1 };

struct ho_state {
  ho_config c;
  int n1m, n2m;
  const double *gcov, *gcon, *gdet, *conn, *floors;
  double *pk0, *dq, *pl, *pr, *F1, *F2, *emf, *prc, *ulast, *unew;
  double *gammacheck; /* persistent, [n1+2][n2+2] like fixup.c:393 */
  double hz[6];       /* horizon accounting, see ho_get_horizon */
  double dt_free;     /* the last step's next dt before the end-time clamp */
  const double *pcur; /* the step's p (bounds.ns.c reads the global p's field) */
  const int *pfcur;   /* the step's pflag (fluxcalc reads FLAGREALFLUX) */
  double *cfar;       /* current_precalc slots, [n1m][n2m][5][3] like cfaraday */
  double *fcon;       /* [n1m][n2m][6] */
  double *jcon;       /* [n1m][n2m][4] */
  long ccalls;        /* current_calc_1's static call count */
  double clastdt;     /* and its static lastdt */
  long ncb;
  int fail, fail_i, fail_j; /* first fatal check of the last ho_step: code and zone (fail.c:4-57 reports
                               the zone of the last get_geometry call, i.e. the zone or face being worked on) */
  /* inputs of the inversions that failed (test fixtures for the retry
     chain): zone, U in the evolved form, the guess; up to rec_max */
  int rec_max, rec_n;
  int *rec_ij;
  double *rec_U, *rec_pr;
};

/* ---------------------------------------------------------------- indexing */
static inline long zid(const ho_state *s, int i, int j) { return (long)(i + NG) * s->n2m + (j + NG); }
#define P(arr, i, j) ((arr) + zid(s, (i), (j)) * NPR)
#define FL(arr, i, j) ((arr) + zid(s, (i), (j)) * NFL)
/* records the first fatal check (code rc at zone or face i, j) and passes rc on */
static int failat(ho_state *s, int rc, int i, int j)
{
  if (rc && !s->fail) {
    s->fail = rc;
    s->fail_i = i;
    s->fail_j = j;
  }
  return rc;
}

typedef struct {
  const double *gcov; /* 16, row-major */
  const double *gcon;
  double g;
  int i, j, loc;
} geo;

static inline geo getgeo(const ho_state *s, int i, int j, int loc)
{
  geo g;
  long z = zid(s, i, j);
  g.gcov = s->gcov + (z * 4 + loc) * 16;
  g.gcon = s->gcon + (z * 4 + loc) * 16;
  g.g = s->gdet[z * 4 + loc];
  g.i = i;
  g.j = j;
  g.loc = loc;
  return g;
}
#define GCOV(g, a, b) ((g)->gcov[(a) * 4 + (b)])
#define GCON(g, a, b) ((g)->gcon[(a) * 4 + (b)])

/* the reference's max/min/sign helpers, phys.c:1562-1591 */
static inline double rmax(double a, double b) { return (a > b) ? a : b; }
static inline double rmin(double a, double b) { return (a > b) ? b : a; }
static inline double rsign(double a) { return (a > 0.0) ? 1.0 : ((a < 0.0) ? -1.0 : 0.0); }

/* ----------------------------------------------------------- cycle break */
static uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

double ho_cycle_break_uniform(double x0, double x1, int n_iter)
{
  uint64_t a, b;
  memcpy(&a, &x0, 8);
  memcpy(&b, &x1, 8);
  uint64_t h = mix64(a ^ mix64(b ^ (uint64_t)(uint32_t)n_iter));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------ state math */
typedef struct {
  double ucon[4], ucov[4], bcon[4], bcov[4];
} ostate;

/* gamma_calc, phys.c:848-877 */
static double gamma_of(const double *pr, const geo *g)
{
  double qsq = GCOV(g, 1, 1) * pr[U1] * pr[U1] + GCOV(g, 2, 2) * pr[U2] * pr[U2] + GCOV(g, 3, 3) * pr[U3] * pr[U3] +
               2. * (GCOV(g, 1, 2) * pr[U1] * pr[U2] + GCOV(g, 1, 3) * pr[U1] * pr[U3] + GCOV(g, 2, 3) * pr[U2] * pr[U3]);
  return sqrt(1. + qsq);
}

/* ucon_calc_rel4vel, phys.c:830-845 */
static void ucon_of(const double *pr, const geo *g, double *ucon)
{
  double alpha = 1. / sqrt(-GCON(g, 0, 0));
  double beta1 = GCON(g, 0, 1) * alpha * alpha;
  double beta2 = GCON(g, 0, 2) * alpha * alpha;
  double beta3 = GCON(g, 0, 3) * alpha * alpha;
  double gamma = gamma_of(pr, g);
  ucon[0] = gamma / alpha;
  ucon[1] = pr[U1] - gamma * beta1 / alpha;
  ucon[2] = pr[U2] - gamma * beta2 / alpha;
  ucon[3] = pr[U3] - gamma * beta3 / alpha;
}

/* lower, phys.c:633 (upper-triangle access as written there) */
static void lower_v(const double *v, const geo *g, double *w)
{
  w[0] = GCOV(g, 0, 0) * v[0] + GCOV(g, 0, 1) * v[1] + GCOV(g, 0, 2) * v[2] + GCOV(g, 0, 3) * v[3];
  w[1] = GCOV(g, 0, 1) * v[0] + GCOV(g, 1, 1) * v[1] + GCOV(g, 1, 2) * v[2] + GCOV(g, 1, 3) * v[3];
  w[2] = GCOV(g, 0, 2) * v[0] + GCOV(g, 1, 2) * v[1] + GCOV(g, 2, 2) * v[2] + GCOV(g, 2, 3) * v[3];
  w[3] = GCOV(g, 0, 3) * v[0] + GCOV(g, 1, 3) * v[1] + GCOV(g, 2, 3) * v[2] + GCOV(g, 3, 3) * v[3];
}

/* raise, phys.c:690 */
static void raise_v(const double *v, const geo *g, double *w)
{
  w[0] = GCON(g, 0, 0) * v[0] + GCON(g, 0, 1) * v[1] + GCON(g, 0, 2) * v[2] + GCON(g, 0, 3) * v[3];
  w[1] = GCON(g, 0, 1) * v[0] + GCON(g, 1, 1) * v[1] + GCON(g, 1, 2) * v[2] + GCON(g, 1, 3) * v[3];
  w[2] = GCON(g, 0, 2) * v[0] + GCON(g, 1, 2) * v[1] + GCON(g, 2, 2) * v[2] + GCON(g, 2, 3) * v[3];
  w[3] = GCON(g, 0, 3) * v[0] + GCON(g, 1, 3) * v[1] + GCON(g, 2, 3) * v[2] + GCON(g, 3, 3) * v[3];
}

static inline double dot4(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }

/* get_state, phys.c:716-727 (+ bcon_calc phys.c:285-294) */
static void state_of(const double *pr, const geo *g, ostate *q)
{
  int j;
  ucon_of(pr, g, q->ucon);
  lower_v(q->ucon, g, q->ucov);
  q->bcon[0] = pr[B1] * q->ucov[1] + pr[B2] * q->ucov[2] + pr[B3] * q->ucov[3];
  for (j = 1; j <= 3; j++) q->bcon[j] = (pr[B1 - 1 + j] + q->bcon[0] * q->ucon[j]) / q->ucon[0];
  lower_v(q->bcon, g, q->bcov);
}

/* mhd_calc_0, phys.c:381-406: row dir of T^mu_nu */
static void mhd_row(const double *pr, int dir, const ostate *q, double gam, int ffde, double *mhd)
{
  double r, u, P, w;
  int j;
  if (!ffde) {
    r = pr[RHO];
    u = pr[UU];
    P = (gam - 1.) * u;
    w = P + r + u;
  } else {
    r = u = P = w = 0.0;
  }
  double bsq = dot4(q->bcon, q->bcov);
  double eta = w + bsq;
  double ptot = P + bsq * 0.5;
  for (j = 0; j < 4; j++) mhd[j] = eta * q->ucon[dir] * q->ucov[j] + ptot * ((dir == j) ? 1. : 0.) - q->bcon[dir] * q->bcov[j];
}

/* primtoflux(UEVOLVE), phys.c:16-56 with massflux_calc (59), the PRIMMAXWELL
   dualfullfaraday_calc (155-185) and UtoU(UNOTHING->UEVOLVE) (219-265) */
static void flux_of(const double *pr, const ostate *q, int dir, const geo *g, double gam, int ffde, double *F)
{
  double fin[NPR];
  int k;
  fin[RHO] = pr[RHO] * q->ucon[dir];
  mhd_row(pr, dir, q, gam, ffde, &fin[UU]);
  if (dir > 0) {
    fin[B1] = (pr[B1] * q->ucon[dir] - pr[B1 + dir - 1] * q->ucon[1]) / q->ucon[0];
    fin[B2] = (pr[B2] * q->ucon[dir] - pr[B1 + dir - 1] * q->ucon[2]) / q->ucon[0];
    fin[B3] = (pr[B3] * q->ucon[dir] - pr[B1 + dir - 1] * q->ucon[3]) / q->ucon[0];
  } else {
    fin[B1] = pr[B1];
    fin[B2] = pr[B2];
    fin[B3] = pr[B3];
  }
  if (!ffde) fin[UU] += fin[RHO];
  for (k = 0; k < NPR; k++) F[k] = fin[k] * g->g;
}

/* vchar + simplefast, vchar.c:37-135 and 166-234.  Returns a fail code. */
static int vchar_of(const double *pr, const ostate *q, int dir, const geo *g, double gam, int ffde, double *vmax, double *vmin)
{
  double bsq = dot4(q->bcon, q->bcov);
  double rho = pr[RHO];
  double u = pr[UU];
  double WW, cs2, EF, va2, cms2;
  (void)ffde;
  WW = rho + gam * u;
  if (WW > 0.0) cs2 = gam * (gam - 1.) * u / WW;
  else WW = cs2 = 0.0;
  EF = bsq + WW;
  if (EF > 0.0) va2 = bsq / EF;
  else EF = va2 = 0.0;
  cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < 0.0) {
    if (cms2 / (cs2 + va2) > -DBL_EPS_REF * 100.0) cms2 = 0.0;
    else return FAIL_COEFF_NEG;
  }
  if (cms2 > 1.) {
    if (cms2 < 1.0 + DBL_EPS_REF * 100.0) cms2 = 1.0;
    else return FAIL_COEFF_SUP;
  }
  double Acov[4] = {0., 0., 0., 0.}, Bcov[4] = {1., 0., 0., 0.}, Acon[4], Bcon[4];
  Acov[dir] = 1.;
  raise_v(Acov, g, Acon);
  raise_v(Bcov, g, Bcon);
  double Asq = dot4(Acon, Acov), Bsq = dot4(Bcon, Bcov);
  double Au = dot4(Acov, q->ucon), Bu = dot4(Bcov, q->ucon), AB = dot4(Acon, Bcov);
  double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  double A = Bu2 - (Bsq + Bu2) * cms2;
  double B = 2. * (AuBu - (AB + AuBu) * cms2);
  double C = Au2 - (Asq + Au2) * cms2;
  double discr = B * B - 4. * A * C;
  if ((discr < 0.0) && (discr > -1E-10)) discr = 0.0;
  else if (discr < -1E-10) return FAIL_VCHAR_DISCR;
  discr = sqrt(discr);
  double vm = -(-B + discr) / (2. * A);
  double vp = -(-B - discr) / (2. * A);
  if (vp < vm) {
    *vmax = vm;
    *vmin = vp;
  } else {
    *vmax = vp;
    *vmin = vm;
  }
  return 0;
}

/* limit_gamma, fixup.c:1298-1354.  Returns a fail code. */
static int limit_gamma(double gammamax, double *pr, const geo *g)
{
  if (gammamax <= 1.0) return 0;
  double gamma = gamma_of(pr, g);
  if (gamma > gammamax && gamma != 1.0) {
    double pref = (gammamax * gammamax - 1.) / (gamma * gamma - 1.);
    if (pref < 0.0) return FAIL_UTCALC_DISCR;
    double f = sqrt(pref);
    pr[U1] *= f;
    pr[U2] *= f;
    pr[U3] *= f;
  }
  return 0;
}

/* inflow_check_rel4vel for dir = 1 at CENT, fixup.c:1733-1830; the inner
   x1 end is OUTFLOW for the torus and NSSURFACE (never fixed) for the star,
   the outer end OUTFLOW for both.  Returns a fail code. */
static int inflow_check_x1(const ho_state *s, double *pr, const geo *g)
{
  double ucon[4];
  ucon_of(pr, g, ucon);
  const int inner_outflow = (s->c.bc == BC_TORUS);
  int dofix = ((g->i <= -1) && inner_outflow && (ucon[1] > 0.)) || ((g->i >= s->c.n1) && (ucon[1] < 0.));
  if (!dofix) return 0;
  double gamma = gamma_of(pr, g);
  pr[U1] /= gamma;
  pr[U2] /= gamma;
  pr[U3] /= gamma;
  double alpha = 1. / sqrt(-GCON(g, 0, 0));
  double betacon = GCON(g, 0, 1) * alpha * alpha;
  pr[U1] = betacon / alpha;
  double vsq = 0.;
  int j, k;
  for (j = 1; j < 4; j++)
    for (k = 1; k < 4; k++) vsq += GCOV(g, j, k) * pr[U1 + j - 1] * pr[U1 + k - 1];
  if (vsq < 0.0) {
    if (vsq > -DBL_EPS_REF * 100.0) vsq = 0.0;
    else return FAIL_VSQ_NEG;
  }
  if (vsq >= 1.0) vsq = 1.0 - 1.0 / (s->c.gammamax * s->c.gammamax);
  gamma = 1. / sqrt(1. - vsq);
  pr[U1] *= gamma;
  pr[U2] *= gamma;
  pr[U3] *= gamma;
  return 0;
}

/* ------------------------------------------------------- reconstruction */
/* slope_lim_3points MC branch, interp.c:106-118 with MINMOD interp.h:13-14 */
static inline double minmod(double a, double b) { return (a * b <= 0) ? 0.0 : ((fabs(a) < fabs(b)) ? a : b); }
static double mc_slope(double yl, double yc, double yr)
{
  double Dqm = 2.0 * (yc - yl);
  double Dqp = 2.0 * (yr - yc);
  double Dqc = 0.5 * (yr - yl);
  return minmod(Dqc, minmod(Dqm, Dqp));
}

/* para4 with the MC sub-limiter, interp.c:444-538 */
static void para4(double x1, double x2, double x3, double x4, double x5, double *lout, double *rout)
{
  double y[5] = {x1, x2, x3, x4, x5}, dq[5];
  int i;
  for (i = 1; i < 4; i++) {
    double Dqm = 2.0 * (y[i] - y[i - 1]);
    double Dqp = 2.0 * (y[i + 1] - y[i]);
    double Dqc = 0.5 * (y[i + 1] - y[i - 1]);
    double aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
    double sgn = Dqm * Dqp;
    if (sgn <= 0.) dq[i] = 0.;
    else dq[i] = rmin(aDqc, rmin(aDqm, aDqp)) * rsign(Dqc);
  }
  double l = 0.5 * (y[2] + y[1]) - (dq[2] - dq[1]) / 8.0;
  double r = 0.5 * (y[3] + y[2]) - (dq[3] - dq[2]) / 8.0;
  l = rmax(rmin(y[2], y[1]), l);
  l = rmin(rmax(y[2], y[1]), l);
  r = rmax(rmin(y[2], y[3]), r);
  r = rmin(rmax(y[2], y[3]), r);
  double qa = (r - y[2]) * (y[2] - l);
  double qd = (r - l);
  double qe = 8.0 * (y[2] - 0.5 * (l + r));
  if (qa <= 0.) {
    l = y[2];
    r = y[2];
  } else {
    if (qd * (qd - qe) < 0.0) l = 3.0 * y[2] - 2.0 * r;
    if (qd * (qd + qe) < 0.0) r = 3.0 * y[2] - 2.0 * l;
  }
  *lout = l;
  *rout = r;
}

/* ------------------------------------------------------------ flux calc */
/* fluxcalc, step_ch.c:741-1069 (+ cminmax_calc 1095-1148).  Returns fail. */
static int fluxcalc(ho_state *s, const double *pb, double *F, int dir, double *ndt)
{
  const int idel = (dir == 1), jdel = (dir == 2);
  const int face = (dir == 1) ? FACE1 : FACE2;
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j, k, rc;
  const double dxd = (dir == 1) ? s->c.dx1 : s->c.dx2;
  const int ffde = s->c.eom;

  /* DQZLOOP: slopes over i in [-1,N1], j in [-1,N2] */
  for (i = -1; i <= n1; i++)
    for (j = -1; j <= n2; j++)
      for (k = 0; k < NPR; k++) {
        double yll = P(pb, i - 2 * idel, j - 2 * jdel)[k], yl = P(pb, i - idel, j - jdel)[k];
        double yc = P(pb, i, j)[k], yr = P(pb, i + idel, j + jdel)[k], yrr = P(pb, i + 2 * idel, j + 2 * jdel)[k];
        if (s->c.lim == LIM_PARA) para4(yll, yl, yc, yr, yrr, &P(s->pl, i, j)[k], &P(s->pr, i, j)[k]);
        else P(s->dq, i, j)[k] = mc_slope(yl, yc, yr);
      }

  *ndt = 1.e9;
  /* FZLOOP(-jdel, -idel): i from -jdel..N1, j from -idel..N2 */
  for (i = -jdel; i <= n1; i++)
    for (j = -idel; j <= n2; j++) {
      double p_l[NPR], p_r[NPR], F_l[NPR], F_r[NPR], U_l[NPR], U_r[NPR];
      for (k = 0; k < NPR; k++) {
        if (s->c.lim != LIM_PARA) {
          p_l[k] = P(pb, i - idel, j - jdel)[k] + 0.5 * P(s->dq, i - idel, j - jdel)[k];
          p_r[k] = P(pb, i, j)[k] - 0.5 * P(s->dq, i, j)[k];
        } else {
          p_l[k] = P(s->pr, i - idel, j - jdel)[k];
          p_r[k] = P(s->pl, i, j)[k];
        }
      }
      geo g = getgeo(s, i, j, face);
      if (dir == 1) p_l[B1] = p_r[B1] = 0.5 * (p_l[B1] + p_r[B1]);
      else p_l[B2] = p_r[B2] = 0.5 * (p_l[B2] + p_r[B2]);
      if ((rc = limit_gamma(s->c.gammamax, p_l, &g))) return failat(s, rc, i, j);
      if ((rc = limit_gamma(s->c.gammamax, p_r, &g))) return failat(s, rc, i, j);
      ostate ql, qr;
      state_of(p_l, &g, &ql);
      state_of(p_r, &g, &qr);
      flux_of(p_l, &ql, dir, &g, s->c.gam, ffde, F_l);
      flux_of(p_r, &qr, dir, &g, s->c.gam, ffde, F_r);
      flux_of(p_l, &ql, 0, &g, s->c.gam, ffde, U_l);
      flux_of(p_r, &qr, 0, &g, s->c.gam, ffde, U_r);
      double cmax_l, cmin_l, cmax_r, cmin_r;
      if ((rc = vchar_of(p_l, &ql, dir, &g, s->c.gam, ffde, &cmax_l, &cmin_l))) return failat(s, rc, i, j);
      if ((rc = vchar_of(p_r, &qr, dir, &g, s->c.gam, ffde, &cmax_r, &cmin_r))) return failat(s, rc, i, j);
      double lmin = rmin(cmin_l, cmin_r);
      double lmax = rmax(cmax_l, cmax_r);
      lmin = fabs(rmax(0., -lmin));
      lmax = fabs(rmax(0., lmax));
      double cmin = lmin, cmax = lmax, ctop = rmax(lmax, lmin);
      /* choose_flux, step_ch.c:703-738: with FLUXADJUST and
         HYDROFLUXADJUSTONLY 1 the hydro variables follow FLAGREALFLUX of
         zone (i, j), the field ones fluxmethod */
      const int rf = s->c.fluxadjust ? FL(s->pfcur, i, j)[F_REALFLUX] : s->c.fluxmethod;
      double *Fo = P(F, i, j);
      if (cmax + cmin != 0.0) {
        for (k = 0; k < NPR; k++) {
          const int m = (k < B1) ? rf : s->c.fluxmethod;
          const double hllfrac = (m == FLUX_HLL) ? 1.0 : 0.0;
          const double laxffrac = (m == FLUX_HLL) ? 0.0 : 1.0;
          Fo[k] = hllfrac * ((cmax * F_l[k] + cmin * F_r[k] - cmax * cmin * (U_r[k] - U_l[k])) / (cmax + cmin)) +
                  laxffrac * (0.5 * (F_l[k] + F_r[k] - ctop * (U_r[k] - U_l[k])));
        }
      } else {
        for (k = 0; k < NPR; k++) Fo[k] = (0.5 * (F_l[k] + F_r[k] - ctop * (U_r[k] - U_l[k])));
      }
      cmax = rmax(cmax, cmin);
      double dtij = s->c.cour * dxd / cmax;
      if (dtij < *ndt) *ndt = dtij;
    }
  return 0;
}

/* fix_flux, fixup.c:1357-1410 (both x2 ends POLARAXIS; the x1 inner mass
   flux clamp only where that end is OUTFLOW) */
static void fix_flux(ho_state *s)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j, k;
  for (i = -1; i < n1; i++) {
    P(s->F1, i, -1)[B2] = -P(s->F1, i, 0)[B2];
    for (k = 0; k < NPR; k++)
      if (k != U2) P(s->F2, i, 0)[k] = 0.;
  }
  for (i = -1; i < n1; i++) {
    P(s->F1, i, n2)[B2] = -P(s->F1, i, n2 - 1)[B2];
    for (k = 0; k < NPR; k++)
      if (k != U2) P(s->F2, i, n2)[k] = 0.;
  }
  /* the reference zeroes F2 on the row j = (N2-1)/2 (integer division) */
  j = (n2 - 1) / 2;
  for (i = 0; i < n1; i++)
    for (k = 0; k < NPR; k++)
      if (k != U2) P(s->F2, i, j)[k] = 0.;
  if (s->c.bc == BC_TORUS)
    for (j = -1; j < n2; j++)
      if (P(s->F1, 0, j)[RHO] > 0) P(s->F1, 0, j)[RHO] = 0;
  for (j = -1; j < n2; j++)
    if (P(s->F1, n1, j)[RHO] < 0) P(s->F1, n1, j)[RHO] = 0;
}

/* flux_ct FLUXCTTOTH with CORNGDETVERSION 1, step_ch.c:1214-1241, 1403-1413 */
static void flux_ct(ho_state *s)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j;
  for (i = 0; i <= n1; i++)
    for (j = 0; j <= n2; j++) {
      double gc = s->gdet[zid(s, i, j) * 4 + CORN];
      double g1 = s->gdet[zid(s, i, j) * 4 + FACE1], g2 = s->gdet[zid(s, i, j - 1) * 4 + FACE1];
      double g3 = s->gdet[zid(s, i, j) * 4 + FACE2], g4 = s->gdet[zid(s, i - 1, j) * 4 + FACE2];
      s->emf[zid(s, i, j)] = 0.25 * (gc) * (P(s->F1, i, j)[B2] / (g1) + P(s->F1, i, j - 1)[B2] / (g2) -
                                           P(s->F2, i, j)[B1] / (g3) - P(s->F2, i - 1, j)[B1] / (g4));
    }
  for (i = 0; i <= n1; i++)
    for (j = 0; j <= n2 - 1; j++) {
      P(s->F1, i, j)[B1] = 0.;
      P(s->F1, i, j)[B2] = 0.5 * (s->emf[zid(s, i, j)] + s->emf[zid(s, i, j + 1)]);
    }
  for (i = 0; i <= n1 - 1; i++)
    for (j = 0; j <= n2; j++) {
      P(s->F2, i, j)[B1] = -0.5 * (s->emf[zid(s, i, j)] + s->emf[zid(s, i + 1, j)]);
      P(s->F2, i, j)[B2] = 0.;
    }
}

/* ---------------------------------------------------- con-to-prim (2D) */
typedef struct {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, wglobal, gam;
} u2pctx;

/* utsq_calc, utoprim_2d.c:318-338 */
static double utsq_calc(const u2pctx *c, double W)
{
  double Wsq = W * W, W4 = Wsq * Wsq;
  return (c->Bsq * c->QdotBsq + W * (2. * c->QdotBsq + c->Qtsq * W)) /
         (W4 + 2. * c->Bsq * Wsq * W + Wsq * (c->Bsq * c->Bsq - c->Qtsq) - c->QdotBsq * (2. * W + c->Bsq));
}

/* func_vsq, utoprim_2d.c:748-798 (Newton step only; f/df are unused with
   dodamp = 0 and the reference's is_nan_inf never firing) */
static void func_vsq(const u2pctx *c, const double *x, double *dx)
{
  const double Bsq = c->Bsq, QdotBsq = c->QdotBsq, Qtsq = c->Qtsq, Qdotn = c->Qdotn, D = c->D, gam = c->gam;
  double W = x[0], vsq = x[1], Wsq = W * W;
  double gtmp = 1. - vsq;
  double p_tmp = (gam - 1.) * (W * gtmp - D * sqrt(gtmp)) / gam;
  double dPdW = (gam - 1.) * (1. - vsq) / gam;
  double dPdvsq = (gam - 1.) * (0.5 * D / sqrt(1. - vsq) - W) / gam;
  dx[0] = (-Bsq / 2. + dPdvsq) * (Qtsq - vsq * ((Bsq + W) * (Bsq + W)) + (QdotBsq * (Bsq + 2 * W)) / Wsq) +
          ((Bsq + W) * (Bsq + W)) * (Qdotn - (Bsq * (1 + vsq)) / 2. + QdotBsq / (2. * Wsq) - W + p_tmp);
  dx[1] = -((-1 + dPdW - QdotBsq / (Wsq * W)) * (Qtsq - vsq * ((Bsq + W) * (Bsq + W)) + (QdotBsq * (Bsq + 2 * W)) / Wsq)) -
          2 * (vsq + QdotBsq / (Wsq * W)) * (Bsq + W) * (Qdotn - (Bsq * (1 + vsq)) / 2. + QdotBsq / (2. * Wsq) - W + p_tmp);
  double detJ = (Bsq + W) * ((-1 + dPdW - QdotBsq / (Wsq * W)) * (Bsq + W) +
                             ((Bsq - 2 * dPdvsq) * (QdotBsq + vsq * (Wsq * W))) / (Wsq * W));
  dx[0] /= -(detJ);
  dx[1] /= -(detJ);
}

/* general_newton_raphson with validate_x(vartype 3), utoprim_2d.c:606-740
   and 556-600.  Returns 0 (converged / accepted) or 1. */
static int newton(const u2pctx *c, double *x, double gammafail, long *ncb)
{
  double dx[2], x_old[2], errx = 1., errx_old = 2., errx_oldest;
  int n_iter = 0, id;
  const double vsq_too_big = (1.0 - 1.0 / (gammafail - 1.0));
  while ((errx > NEWT_TOL) && (n_iter < MAX_NEWT_ITER)) {
    func_vsq(c, x, dx);
    if (((n_iter + 1) % CYCLE_BREAK_PERIOD) == 0) {
      double randtmp = ho_cycle_break_uniform(x[0], x[1], n_iter);
      (*ncb)++;
      for (id = 0; id < 2; id++) dx[id] *= randtmp;
    }
    errx_oldest = errx_old;
    errx_old = errx;
    errx = 0.;
    for (id = 0; id < 2; id++) {
      x_old[id] = x[id];
      x[id] += dx[id] * 1.0;
      errx += (x[id] == 0.) ? fabs(dx[id]) : fabs(dx[id] / x[id]);
    }
    errx /= 1. * 2;
    /* validate_x */
    x[0] = fabs(x[0]);
    x[0] = (x[0] / c->wglobal > W_TOO_BIG) ? x_old[0] : x[0];
    x[1] = (x[1] < 0.) ? 0.0 : x[1];
    x[1] = (x[1] > 1.) ? vsq_too_big : x[1];
    if (((errx_old == errx) || (errx_oldest == errx)) && (errx < MIN_NEWT_TOL)) errx = -errx;
    n_iter++;
  }
  if (n_iter >= MAX_NEWT_ITER) return (errx > MIN_NEWT_TOL) ? 1 : 0;
  return 0;
}

static void lower_g(const double *v, const geo *g, double *w)
{
  int i, j;
  for (i = 0; i < 4; i++) {
    w[i] = 0.;
    for (j = 0; j < 4; j++) w[i] += GCOV(g, i, j) * v[j];
  }
}
static void raise_g(const double *v, const geo *g, double *w)
{
  int i, j;
  for (i = 0; i < 4; i++) {
    w[i] = 0.;
    for (j = 0; j < 4; j++) w[i] += GCON(g, i, j) * v[j];
  }
}

/* Utoprim_new_body, utoprim_2d.c:128-310.  U and prim in the rescaled form
   of Utoprim_2d.  Returns the pflag code. */
/* ucon_calc_3vel, phys.c:885-957: u^mu from v^i = u^i/u^t; nonzero when
   the velocity is not time-like */
static int ucon_3vel(const double *vcon, const geo *g, double *ucon)
{
  double discr = +GCOV(g, 0, 0) + GCOV(g, 1, 1) * vcon[1] * vcon[1] + GCOV(g, 2, 2) * vcon[2] * vcon[2] +
                 GCOV(g, 3, 3) * vcon[3] * vcon[3] +
                 2. * (GCOV(g, 0, 1) * vcon[1] + GCOV(g, 0, 2) * vcon[2] + GCOV(g, 0, 3) * vcon[3] +
                       GCOV(g, 1, 2) * vcon[1] * vcon[2] + GCOV(g, 1, 3) * vcon[1] * vcon[3] +
                       GCOV(g, 2, 3) * vcon[2] * vcon[3]);
  int j;
  if (discr > 0.) return 1;
  ucon[0] = 1. / sqrt(-discr);
  for (j = 1; j < 4; j++) ucon[j] = vcon[j] * ucon[0];
  return 0;
}

static int u2p_body(const double *U, const geo *g, double *prim, double gam, double gammafail, long *ncb)
{
  u2pctx c;
  double Bcon[4], Bcov[4], Qcov[4], Qcon[4], ncov[4], ncon[4], Qtcon[4];
  double QdotB, Qsq, utsq, rho0, u, p, w, W;
  const double utsq_too_big = ((gammafail - 1.0) * (gammafail - 1.0));
  int i, j, pfl = 0;
  c.gam = gam;
  for (i = B1; i <= B3; i++) prim[i] = U[i];
  Bcon[0] = 0.;
  for (i = 1; i < 4; i++) Bcon[i] = U[B1 + i - 1];
  lower_g(Bcon, g, Bcov);
  for (i = 0; i < 4; i++) Qcov[i] = U[UU + i];
  raise_g(Qcov, g, Qcon);
  c.Bsq = 0.;
  for (i = 1; i < 4; i++) c.Bsq += Bcon[i] * Bcov[i];
  QdotB = 0.;
  for (i = 0; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
  c.QdotBsq = QdotB * QdotB;
  double lapse = sqrt(-1. / GCON(g, 0, 0));
  ncov[0] = -lapse;
  ncov[1] = ncov[2] = ncov[3] = 0.;
  raise_g(ncov, g, ncon);
  c.Qdotn = Qcon[0] * ncov[0];
  Qsq = 0.;
  for (i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
  c.Qtsq = Qsq + c.Qdotn * c.Qdotn;
  c.D = U[RHO];
  utsq = 0.;
  for (i = 1; i < 4; i++)
    for (j = 1; j < 4; j++) utsq += GCOV(g, i, j) * prim[U1 + i - 1] * prim[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > utsq_too_big) return PF_CONVUTSQ;
  rho0 = prim[RHO];
  u = prim[UU];
  p = (gam - 1.) * u;
  w = rho0 + u + p;
  W = w * (1. + utsq);
  c.wglobal = w;
  /* find_root_2D_gen, utoprim_2d.c:471-511 (MAX_NEWT_RETRIES = 0) */
  {
    double x[2], ut;
    int ret;
    x[0] = fabs(W);
    ut = fabs(utsq_calc(&c, W));
    x[1] = (ut > 0.) ? (ut / (ut + 1.)) : 0.0;
    ret = newton(&c, x, gammafail, ncb);
    if (ret != 0) return ret * 100 + 1;
    W = x[0];
  }
  if (W == FAIL_VAL) return 0 * 100 + 1;
  {
    double Wtest = W / c.wglobal;
    if (Wtest <= 0. || Wtest > W_TOO_BIG) return PF_CONVW;
  }
  utsq = utsq_calc(&c, W);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > utsq_too_big) return PF_CONVUTSQ2;
  double gamma = sqrt(1. + utsq);
  rho0 = c.D / gamma;
  w = W / (gamma * gamma);
  p = (gam - 1.) * (w - rho0) / gam;
  u = w - (rho0 + p);
  if ((rho0 <= 0.) || (u <= 0.)) {
    if ((rho0 <= 0.) && (u >= 0.)) pfl = PF_RHONEG;
    if ((rho0 >= 0.) && (u <= 0.)) pfl = PF_UNEG;
    if ((rho0 <= 0.) && (u <= 0.)) pfl = PF_RHOUNEG;
  }
  prim[RHO] = rho0;
  prim[UU] = u;
  for (i = 1; i < 4; i++) Qtcon[i] = Qcon[i] + ncon[i] * c.Qdotn;
  for (i = 1; i < 4; i++)
    prim[U1 + i - 1] = -gamma * Qtcon[i] / (W + c.Bsq) - gamma * QdotB * Bcon[i] / (W * (W + c.Bsq));
  for (i = B1; i <= B3; i++) prim[i] = U[i];
  return pfl;
}

/* Utoprimgen(UEVOLVE) -> UtoU -> Utoprim_2d, step_ch.c:468-552,
   phys.c:219-265, utoprim_2d.c:25-94.  Returns the pflag code. */
static int utoprimgen(const ho_state *s, const double *U, const geo *g, double *pr, long *ncb)
{
  double Ug[NPR], Ut[NPR], pt[NPR];
  int k;
  for (k = 0; k < NPR; k++) Ug[k] = U[k] / g->g;
  Ug[UU] += -Ug[RHO];
  double alpha = 1.0 / sqrt(-GCON(g, 0, 0));
  Ut[RHO] = Ug[RHO] * alpha;
  for (k = UU; k <= U3; k++) Ut[k] = -alpha * Ug[k];
  for (k = B1; k <= B3; k++) Ut[k] = alpha * Ug[k];
  for (k = 0; k < B1; k++) pt[k] = pr[k];
  for (k = B1; k <= B3; k++) pt[k] = alpha * pr[k];
  int pfl = u2p_body(Ut, g, pt, s->c.gam, s->c.gammafail, ncb);
  for (k = 0; k < B1; k++) pr[k] = pt[k];
  for (k = B1; k <= B3; k++) pr[k] = pt[k] / alpha;
  return pfl;
}

/* Utoprimgen(UEVOLVE) for EOMFFDE, step_ch.c:544-546 -> UtoU (phys.c:228-233,
   no rest-mass term) -> Utoprim_ffde, phys.ffde.c:141-372 with
   CHECKBSQMINUSESQ 1, AVOIDUTINF 2, REMOVET 0, AVOIDCS 0, FIXB3 0:
   U2BBsq (1261-1284), TtoEconOalpha (1287-1318), EBcovtovcon (551-560),
   vcon2pr(VELREL4) (transforms.c:348-393, whose active branch stores
   u^i) -> ucon_calc_3vel (phys.c:885-957).  diss_account is accounting
   only.  pr[RHO], pr[UU] keep the guess; pflag is not written. */
static int utoprim_ffde(const ho_state *s, const double *Uin, const geo *g, double *pr)
{
  double U[NPR], Bcon[4], Bcov[4], Econ[4], Ecov[4], T[4], vcon[4];
  double alphasq, Bsq, Esq, BsqmEsq, realBsq, gammasq, Gsq, o;
  int j, k;
  for (k = 0; k < NPR; k++) U[k] = Uin[k] / g->g;
  alphasq = 1. / (-GCON(g, 0, 0));
  Bcon[0] = 0.0;
  for (j = 1; j < 4; j++) Bcon[j] = U[B1 + j - 1];
  lower_v(Bcon, g, Bcov);
  Bsq = 0.0;
  for (j = 1; j < 4; j++) Bsq += Bcov[j] * Bcon[j];
  for (j = 0; j < 4; j++) T[j] = U[UU + j];
  o = 1.0 / (Bsq * g->g);
  Econ[0] = 0;
  Econ[1] = (Bcov[2] * T[3] - Bcov[3] * T[2]) * (o);
  Econ[2] = (Bcov[3] * T[1] - Bcov[1] * T[3]) * (o);
  Econ[3] = (Bcov[1] * T[2] - Bcov[2] * T[1]) * (o);
  realBsq = Bsq;
  lower_v(Econ, g, Ecov);
  Esq = 0.0;
  for (j = 1; j < 4; j++) Esq += Econ[j] * Ecov[j];
  BsqmEsq = Bsq - Esq;
  gammasq = Bsq / BsqmEsq;
  if ((gammasq > s->c.gammamax * s->c.gammamax) || (gammasq < 1.0)) {
    Gsq = 1.0 - 1.0 / (s->c.gammamax * s->c.gammamax);
    realBsq = (sqrt(Esq * Bsq / Gsq));
  }
  o = 1.0 / (realBsq * g->g);
  vcon[1] = alphasq * (-GCON(g, 0, 1) + (Ecov[2] * Bcov[3] - Ecov[3] * Bcov[2]) * o);
  vcon[2] = alphasq * (-GCON(g, 0, 2) + (Ecov[3] * Bcov[1] - Ecov[1] * Bcov[3]) * o);
  vcon[3] = alphasq * (-GCON(g, 0, 3) + (Ecov[1] * Bcov[2] - Ecov[2] * Bcov[1]) * o);
  double ucon[4];
  if (ucon_3vel(vcon, g, ucon)) return FAIL_FFDE_SPACELIKE;
  pr[U1] = ucon[1];
  pr[U2] = ucon[2];
  pr[U3] = ucon[3];
  pr[B1] = U[B1];
  pr[B2] = U[B2];
  pr[B3] = U[B3];
  return 0;
}

/* source -> source_conn, phys.c:475-619 (cooling off, numerical
   connection): dU[UU+l] = e * sum_j sum_k T^j_k Gamma^k_{l j} */
static void geom_source(const ho_state *s, const double *pb, const geo *g, double *dU)
{
  ostate q;
  double mhd[4][4], dUconn[NPR];
  const double *cn = s->conn + zid(s, g->i, g->j) * 64;
  int j, k, l;
  state_of(pb, g, &q);
  for (j = 0; j < 4; j++) mhd_row(pb, j, &q, s->c.gam, s->c.eom, mhd[j]);
  for (k = 0; k < NPR; k++) dUconn[k] = 0;
  for (l = 0; l < 4; l++)
    for (j = 0; j < 4; j++)
      for (k = 0; k < 4; k++) dUconn[UU + l] += mhd[j][k] * cn[(k * 4 + l) * 4 + j];
  for (k = 0; k < NPR; k++) dU[k] = 0. + g->g * dUconn[k];
}

/* ------------------------------------------------------------ boundaries */
/* bound_prim of the rotating star, bounds.ns.c:10-355 with EXTRAP 1:
   NSSURFACE inside (densities scaled by sqrt(-g), velocity of a surface
   rotating at omegastar through vcon2pr, field held at the step's p),
   extrapolating OUTFLOW outside, plain polar mirror (the "sign flips" are
   multiplications by 1).  Returns a fail code. */
static int bound_prims_star(ho_state *s, double *pv)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  const double dx1 = s->c.dx1;
  int i, j, k, rc, ri;
#define GD(i, j) (s->gdet[zid(s, (i), (j)) * 4 + CENT])
  for (j = 0; j < n2; j++) {
    ri = 0;
    for (i = -1; i >= -NG; i--) {
      for (k = RHO; k <= UU; k++) P(pv, i, j)[k] = P(pv, ri, j)[k] * GD(ri, j) / GD(i, j);
      double vcon[4] = {0., 0., 0., s->c.omegastar}, ucon[4];
      geo g = getgeo(s, i, j, CENT);
      if (!ucon_3vel(vcon, &g, ucon)) {
        P(pv, i, j)[U1] = ucon[1];
        P(pv, i, j)[U2] = ucon[2];
        P(pv, i, j)[U3] = ucon[3];
      }
      for (k = B1; k <= B3; k++) P(pv, i, j)[k] = P(s->pcur, i, j)[k];
    }
    for (i = -1; i >= -NG; i--) {
      geo g = getgeo(s, i, j, CENT);
      if ((rc = inflow_check_x1(s, P(pv, i, j), &g))) return failat(s, rc, i, j);
      if ((rc = limit_gamma(s->c.gammamax, P(pv, i, j), &g))) return failat(s, rc, i, j);
    }
  }
  for (j = 0; j < n2; j++) {
    ri = n1 - 1;
    for (i = n1; i <= n1 - 1 + NG; i++) {
      for (k = RHO; k <= UU; k++) P(pv, i, j)[k] = P(pv, ri, j)[k] * GD(ri, j) / GD(i, j);
      P(pv, i, j)[U1] = P(pv, ri, j)[U1] * (1. - 2 * (i - ri) * dx1);
      for (k = U2; k <= U3; k++) P(pv, i, j)[k] = P(pv, ri, j)[k] * (1. - (i - ri) * dx1);
      P(pv, i, j)[B1] = P(pv, ri, j)[B1] * GD(ri, j) / GD(i, j);
      for (k = B2; k <= B3; k++) P(pv, i, j)[k] = P(pv, ri, j)[k] * (1. - (i - ri) * dx1);
    }
    for (i = n1; i <= n1 - 1 + NG; i++) {
      geo g = getgeo(s, i, j, CENT);
      if ((rc = inflow_check_x1(s, P(pv, i, j), &g))) return failat(s, rc, i, j);
      if ((rc = limit_gamma(s->c.gammamax, P(pv, i, j), &g))) return failat(s, rc, i, j);
    }
  }
#undef GD
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = -NG; j <= -1; j++)
      for (k = 0; k < NPR; k++) P(pv, i, j)[k] = P(pv, i, -j - 1)[k];
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = n2; j <= n2 - 1 + NG; j++)
      for (k = 0; k < NPR; k++) P(pv, i, j)[k] = P(pv, i, 2 * n2 - 1 - j)[k];
  return 0;
}

/* bound_prim, bounds.fishmon.c:14-330 with EXTRAP 0, POSDEFMETRIC 0 and
   POLEDEATH 1 (the torus), or the rotating star's.  Returns a fail code. */
static int bound_prims(ho_state *s, double *pv)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j, k, rc;
  if (s->c.bc == BC_STAR) return bound_prims_star(s, pv);
  for (j = 0; j < n2; j++) {
    for (i = -1; i >= -NG; i--)
      for (k = 0; k < NPR; k++) P(pv, i, j)[k] = P(pv, 0, j)[k];
    for (i = -1; i >= -NG; i--) {
      geo g = getgeo(s, i, j, CENT);
      if ((rc = inflow_check_x1(s, P(pv, i, j), &g))) return failat(s, rc, i, j);
      if ((rc = limit_gamma(s->c.gammamax, P(pv, i, j), &g))) return failat(s, rc, i, j);
    }
  }
  for (j = 0; j < n2; j++) {
    for (i = n1; i <= n1 - 1 + NG; i++)
      for (k = 0; k < NPR; k++) P(pv, i, j)[k] = P(pv, n1 - 1, j)[k];
    for (i = n1; i <= n1 - 1 + NG; i++) {
      geo g = getgeo(s, i, j, CENT);
      if ((rc = inflow_check_x1(s, P(pv, i, j), &g))) return failat(s, rc, i, j);
      if ((rc = limit_gamma(s->c.gammamax, P(pv, i, j), &g))) return failat(s, rc, i, j);
    }
  }
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = -NG; j <= -1; j++)
      for (k = 0; k < NPR; k++) P(pv, i, j)[k] = P(pv, i, -j - 1)[k];
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = n2; j <= n2 - 1 + NG; j++)
      for (k = 0; k < NPR; k++) P(pv, i, j)[k] = P(pv, i, 2 * n2 - 1 - j)[k];
  /* sign "flips" are multiplications by 1 with POSDEFMETRIC 0 (no-ops) */
  for (i = -NG; i <= n1 - 1 + NG; i++) {
    for (j = -NG; j < 0 + 1; j++) {
      P(pv, i, j)[U2] *= 0;
      P(pv, i, j)[B2] *= 0.;
    }
    for (j = n2 - 1; j <= n2 - 1 + NG; j++) {
      P(pv, i, j)[U2] *= 0.;
      P(pv, i, j)[B2] *= 0.;
    }
  }
  return 0;
}

/* bound_pflag, boundsint.c:4-60 (FLAGUTOPRIMFAIL only) */
static void bound_pflag(ho_state *s, int *pf)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j;
  for (j = -NG; j <= n2 - 1 + NG; j++)
    for (i = -1; i >= -NG; i--) FL(pf, i, j)[F_FAIL] = FL(pf, 0, j)[F_FAIL];
  for (j = -NG; j <= n2 - 1 + NG; j++)
    for (i = n1; i <= n1 - 1 + NG; i++) FL(pf, i, j)[F_FAIL] = FL(pf, n1 - 1, j)[F_FAIL];
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = -NG; j <= -1; j++) FL(pf, i, j)[F_FAIL] = FL(pf, i, -j - 1)[F_FAIL];
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = n2; j <= n2 - 1 + NG; j++) FL(pf, i, j)[F_FAIL] = FL(pf, i, 2 * n2 - 1 - j)[F_FAIL];
}

/* get_bsqflags, fixup.c:1197-1295 (only the two stored flags matter) */
static void bsqflags(ho_state *s, const double *pv, int *pf)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j;
  for (i = -1; i <= n1; i++)
    for (j = -1; j <= n2; j++) {
      geo g = getgeo(s, i, j, CENT);
      ostate q;
      const double *pr = P(pv, i, j);
      int f0 = 0, f3 = 0;
      if (!s->c.eom) { /* the b^2 checks are GRMHD-only (fixup.c:1214-1233) */
        state_of(pr, &g, &q);
        double bsq = dot4(q.bcon, q.bcov);
        if (bsq / pr[RHO] > s->c.bsqorholimit) f0 = 2;
        else if (bsq / pr[RHO] > 0.9 * s->c.bsqorholimit) f0 = 1;
        else f0 = 0;
        if (bsq / pr[UU] > s->c.bsqoulimit) f3 = 2;
        else if (bsq / pr[UU] > 0.9 * s->c.bsqoulimit) f3 = 1;
        else f3 = 0;
      }
      FL(pf, i, j)[F_BSQORHO] = f0;
      FL(pf, i, j)[F_BSQOU] = f3;
      if (s->c.fluxadjust) {
        /* FLAGREALFLUX (fixup.c:1236-1245, 1284-1290): the Lorentz-factor
           flag, then one step down from fluxmethod (HLL -> LAXF, not below
           0) where any flag is 2 */
        const double gamma = gamma_of(pr, &g);
        const int f1 = (gamma > 2.0 * s->c.gammadamp) ? 2 : ((gamma > s->c.gammadamp) ? 1 : 0);
        int rf = (f0 == 2 || f1 == 2 || f3 == 2) ? s->c.fluxmethod - 1 : s->c.fluxmethod;
        FL(pf, i, j)[F_REALFLUX] = (rf < 0) ? 0 : rf;
      }
    }
}

/* fixup_checksolution, fixup.c:388-488 (sequential in ZLOOP order: a zone
   flagged here changes what later zones see) */
static void checksolution(ho_state *s, const double *pv, int *pf)
{
  const int n1 = s->c.n1, n2 = s->c.n2, gw = n2 + 2;
  int i, j, l;
  double *gc = s->gammacheck;
  for (i = -1; i <= n1; i++)
    for (j = -1; j <= n2; j++) {
      const int *f = FL(pf, i, j);
      if ((f[F_BSQORHO] || f[F_BSQOU]) && (f[F_FAIL] == 0)) {
        geo g = getgeo(s, i, j, CENT);
        gc[(i + 1) * gw + (j + 1)] = gamma_of(P(pv, i, j), &g);
      }
    }
  for (i = 0; i < n1; i++)
    for (j = 0; j < n2; j++) {
      int *f = FL(pf, i, j);
      if (!((f[F_BSQORHO] || f[F_BSQOU]) && (f[F_FAIL] == 0))) continue;
      static const int di[8] = {0, 0, 1, -1, 1, 1, 1, -1};
      static const int dj[8] = {1, -1, 0, 0, 1, -1, 1, -1};
      double pd[8], pd2[8];
      double g0 = gc[(i + 1) * gw + (j + 1)];
      double u0 = P(pv, i, j)[UU];
      for (l = 0; l < 8; l++) {
        int ok = (FL(pf, i + di[l], j + dj[l])[F_FAIL] == 0);
        pd[l] = ok ? (gc[(i + 1 + di[l]) * gw + (j + 1 + dj[l])] / g0) : -1;
        pd2[l] = ok ? (P(pv, i + di[l], j + dj[l])[UU] / u0) : -1;
      }
      int v0 = 0, v1 = 0, nv = 0;
      for (l = 0; l < 8; l++) {
        if (pd[0] >= 0.0) {
          if ((fabs(pd[l]) > 2.0) || (fabs(pd[l]) < 1.0 / 2.0)) v0++;
          if ((fabs(pd2[l]) > 10.0) || (fabs(pd2[l]) < 1.0 / 10.0)) v1++;
          nv++;
        }
      }
      if (v0 > nv * 0.5) f[F_FAIL] = PF_GAMMAPERC;
      if (v1 > nv * 0.5) f[F_FAIL] = PF_UPERC;
    }
}

/* fixup_utoprim, fixup.c:527-928 with UTOPRIMAVG, NOGOODAVERAGE,
   HANDLEUNEG 0, STEPOVERNEGU 0, order-independent snapshot prc */
static int fixup_utoprim(ho_state *s, double *pv, int *pf)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j, k, rc;
  memcpy(s->prc, pv, sizeof(double) * (size_t)s->n1m * s->n2m * NPR);
  const double *pa = s->prc;
#define GOOD(ii, jj) (FL(pf, (ii), (jj))[F_FAIL] == 0)
#define PA(ii, jj) (P(pa, (ii), (jj)))
  for (i = 0; i < n1; i++)
    for (j = 0; j < n2; j++) {
      int mypflag = FL(pf, i, j)[F_FAIL];
      if (mypflag == 0) continue;
      double *pr = P(pv, i, j);
      geo g = getgeo(s, i, j, CENT);
      double gamma = gamma_of(pr, &g);
      if (gamma > s->c.gammamax) gamma = s->c.gammamax;
      if (GOOD(i, j + 1) && GOOD(i, j - 1) && GOOD(i + 1, j) && GOOD(i - 1, j)) {
        for (k = 0; k <= U3; k++) pr[k] = 0.25 * (PA(i, j + 1)[k] + PA(i, j - 1)[k] + PA(i - 1, j)[k] + PA(i + 1, j)[k]);
      } else if (GOOD(i + 1, j + 1) && GOOD(i + 1, j - 1) && GOOD(i - 1, j + 1) && GOOD(i - 1, j - 1)) {
        for (k = 0; k <= U3; k++)
          pr[k] = 0.25 * (PA(i + 1, j + 1)[k] + PA(i + 1, j - 1)[k] + PA(i - 1, j + 1)[k] + PA(i - 1, j - 1)[k]);
      } else if (GOOD(i, j + 1) && GOOD(i, j - 1)) {
        for (k = 0; k <= U3; k++) pr[k] = 0.5 * (PA(i, j + 1)[k] + PA(i, j - 1)[k]);
      } else if (GOOD(i + 1, j) && GOOD(i - 1, j)) {
        for (k = 0; k <= U3; k++) pr[k] = 0.5 * (PA(i + 1, j)[k] + PA(i - 1, j)[k]);
      } else if (GOOD(i + 1, j + 1) && GOOD(i - 1, j - 1)) {
        for (k = 0; k <= U3; k++) pr[k] = 0.5 * (PA(i + 1, j + 1)[k] + PA(i - 1, j - 1)[k]);
      } else if (GOOD(i + 1, j - 1) && GOOD(i - 1, j + 1)) {
        for (k = 0; k <= U3; k++) pr[k] = 0.5 * (PA(i + 1, j - 1)[k] + PA(i - 1, j + 1)[k]);
      } else {
        static const int oi[8] = {1, 1, 1, 0, -1, -1, -1, 0};
        static const int oj[8] = {1, 0, -1, -1, -1, 0, 1, 1};
        int m, done = 0;
        for (m = 0; m < 8 && !done; m++)
          if (GOOD(i + oi[m], j + oj[m])) {
            for (k = 0; k <= U3; k++) pr[k] = PA(i + oi[m], j + oj[m])[k];
            done = 1;
          }
        if (!done)
          for (k = 0; k <= U3; k++)
            pr[k] = 0.5 * (0.25 * (PA(i, j + 1)[k] + PA(i, j - 1)[k] + PA(i - 1, j)[k] + PA(i + 1, j)[k]) +
                           0.25 * (PA(i + 1, j + 1)[k] + PA(i + 1, j - 1)[k] + PA(i - 1, j + 1)[k] + PA(i - 1, j - 1)[k]));
      }
      if ((rc = limit_gamma(gamma, pr, &g))) return failat(s, rc, i, j);
      FL(pf, i, j)[F_FAIL] = PF_FIXED;
    }
#undef GOOD
#undef PA
  return 0;
}

/* ------------------------------------------------------------- advance */
/* advance_standard, advance.c:46-197 for one RK2 substep */
static int advance(ho_state *s, const double *pi, const double *pb, double *pf, int *pflag, const double *CUf,
                   const double *Cunew, int timeorder, int last, double dt, double *ndt)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  double ndt1, ndt2;
  int i, j, k, rc;
  if ((rc = fluxcalc(s, pb, s->F1, 1, &ndt1))) return rc;
  if ((rc = fluxcalc(s, pb, s->F2, 2, &ndt2))) return rc;
  fix_flux(s);
  flux_ct(s);
  const double idx1 = 1.0 / s->c.dx1, idx2 = 1.0 / s->c.dx2;
  for (i = 0; i < n1; i++)
    for (j = 0; j < n2; j++) {
      double Ui[NPR], Uf[NPR], dUg[NPR], dUr[NPR];
      double *ul = P(s->ulast, i, j), *un = P(s->unew, i, j);
      double pfz[NPR];
      for (k = 0; k < NPR; k++) pfz[k] = P(pi, i, j)[k];
      if (timeorder == 0)
        for (k = 0; k < NPR; k++) ul[k] = un[k] = 0.0;
      geo g = getgeo(s, i, j, CENT);
      ostate q;
      state_of(P(pi, i, j), &g, &q);
      flux_of(P(pi, i, j), &q, 0, &g, s->c.gam, s->c.eom, Ui);
      geom_source(s, P(pb, i, j), &g, dUg);
      for (k = 0; k < NPR; k++) {
        double d1 = (-(P(s->F1, i + 1, j)[k] - P(s->F1, i, j)[k]) * idx1);
        double d2 = (-(P(s->F2, i, j + 1)[k] - P(s->F2, i, j)[k]) * idx2);
        dUr[k] = d1 + d2;
      }
      for (k = 0; k < NPR; k++) ul[k] = Uf[k] = CUf[0] * Ui[k] + CUf[1] * ul[k] + CUf[2] * dt * (dUr[k] + dUg[k]);
      for (k = 0; k < NPR; k++) un[k] += Cunew[0] * Ui[k] + Cunew[1] * dt * (dUr[k] + dUg[k]) + Cunew[2] * Uf[k];
      if (s->c.eom) {
        if ((rc = utoprim_ffde(s, last ? un : Uf, &g, pfz))) return failat(s, rc, i, j);
      } else {
        double guess[NPR];
        for (k = 0; k < NPR; k++) guess[k] = pfz[k];
        int pfl = utoprimgen(s, last ? un : Uf, &g, pfz, &s->ncb);
        FL(pflag, i, j)[F_FAIL] = pfl;
        if (pfl != 0 && s->rec_n < s->rec_max) {
          s->rec_ij[2 * s->rec_n] = i;
          s->rec_ij[2 * s->rec_n + 1] = j;
          for (k = 0; k < NPR; k++) {
            s->rec_U[NPR * s->rec_n + k] = (last ? un : Uf)[k];
            s->rec_pr[NPR * s->rec_n + k] = guess[k];
          }
          s->rec_n++;
        }
        /* fixup1zone, fixup.c:274-377 (floors are GRMHD-only, 293) */
        const double *fl = s->floors + zid(s, i, j) * 2;
        if (fl[0] > pfz[RHO]) pfz[RHO] = fl[0];
        if (fl[1] > pfz[UU]) pfz[UU] = fl[1];
      }
      if ((rc = limit_gamma(s->c.gammamax, pfz, &g))) return failat(s, rc, i, j);
      for (k = 0; k < NPR; k++) P(pf, i, j)[k] = pfz[k];
    }
  *ndt = s->c.defcon * 1. / (1. / ndt1 + 1. / ndt2);
  return 0;
}

/* ------------------------------------------------------------ currents */
/* current_doprecalc(0..3, p) with WHICHCURRENTCALC 1 (phys.c:1124-1218,
   all at CENT over FULLLOOP): slot 3 <- 4 <- 0 and the new f^{it} in slot
   0, f^{ir} in 1, f^{ih} in 2, and fcon (the six f^{mu nu}). */
static void currents_precalc(ho_state *s, const double *p)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  int i, j, c;
  for (i = -NG; i <= n1 - 1 + NG; i++)
    for (j = -NG; j <= n2 - 1 + NG; j++) {
      geo g = getgeo(s, i, j, CENT);
      ostate q;
      const double *b, *u;
      double *f = s->cfar + zid(s, i, j) * 15, *fc = s->fcon + zid(s, i, j) * 6;
      state_of(P(p, i, j), &g, &q);
      b = q.bcov;
      u = q.ucov;
      for (c = 0; c < 3; c++) {
        f[3 * 3 + c] = f[4 * 3 + c];
        f[4 * 3 + c] = f[0 * 3 + c];
      }
      f[0] = -1.0 / g.g * (-b[3] * u[2] + b[2] * u[3]);
      f[1] = -1.0 / g.g * (b[3] * u[1] - b[1] * u[3]);
      f[2] = -1.0 / g.g * (-b[2] * u[1] + b[1] * u[2]);
      f[3] = -1.0 / g.g * (b[3] * u[2] - b[2] * u[3]);
      f[4] = -1.0 / g.g * (-b[3] * u[0] + b[0] * u[3]);
      f[5] = -1.0 / g.g * (b[2] * u[0] - b[0] * u[2]);
      f[6] = -1.0 / g.g * (-b[3] * u[1] + b[1] * u[3]);
      f[7] = -1.0 / g.g * (b[3] * u[0] - b[0] * u[3]);
      f[8] = -1.0 / g.g * (-b[1] * u[0] + b[0] * u[1]);
      fc[0] = -1.0 / g.g * (b[3] * u[2] - b[2] * u[3]);
      fc[1] = -1.0 / g.g * (-b[3] * u[1] + b[1] * u[3]);
      fc[2] = -1.0 / g.g * (b[2] * u[1] - b[1] * u[2]);
      fc[3] = -1.0 / g.g * (b[3] * u[0] - b[0] * u[3]);
      fc[4] = -1.0 / g.g * (-b[2] * u[0] + b[0] * u[2]);
      fc[5] = -1.0 / g.g * (b[1] * u[0] - b[0] * u[1]);
    }
}

/* current_calc_1, phys.c:1335-1455: J^mu = (1/g) d_nu (g F^{mu nu}) with
   centred space differences over LOOPP11 x LOOPP12 and, from the third call
   on, a second-order one-sided time derivative through the last three
   slots.  J^h's x1 difference uses the zone's own g at i-1 (geomr), as the
   reference does. */
static void currents_calc(ho_state *s, double dt)
{
  const int n1 = s->c.n1, n2 = s->c.n2;
  const double dtl = s->clastdt, dtr = dt;
  const double idx1 = 1.0 / (2.0 * s->c.dx1), idx2 = 1.0 / (2.0 * s->c.dx2);
  int i, j;
#define GC(i, j) (s->gdet[zid(s, (i), (j)) * 4 + CENT])
#define CF(i, j, slot, c) (s->cfar[zid(s, (i), (j)) * 15 + (slot) * 3 + (c)])
  for (i = -NG + 1; i < n1 + NG - 1; i++)
    for (j = -NG + 1; j < n2 + NG - 1; j++) {
      double *J = s->jcon + zid(s, i, j) * 4;
      const double gt = GC(i, j), grp = GC(i + 1, j), ghp = GC(i, j + 1), grm = GC(i - 1, j), ghm = GC(i, j - 1);
      J[0] = 1. / gt * (grp * CF(i + 1, j, 1, 0) - grm * CF(i - 1, j, 1, 0)) * idx1 +
             1. / gt * (ghp * CF(i, j + 1, 2, 0) - ghm * CF(i, j - 1, 2, 0)) * idx2;
      if (s->ccalls >= 2) {
        double d[3];
        int c;
        for (c = 0; c < 3; c++) {
          double fl = CF(i, j, 3, c), f0 = CF(i, j, 4, c), fr = CF(i, j, 0, c);
          double AA = (dtr * (fl - f0) + dtl * (fr - f0)) / (dtl * dtr * (dtl + dtr));
          double BB = (-dtr * dtr * (fl - f0) + dtl * dtl * (fr - f0)) / (dtl * dtr * (dtl + dtr));
          d[c] = 2.0 * AA * dtr + BB;
        }
        J[1] = d[0] + 1. / gt * (ghp * CF(i, j + 1, 2, 1) - ghm * CF(i, j - 1, 2, 1)) * idx2;
        J[2] = d[1] + 1. / gt * (grp * CF(i + 1, j, 1, 1) - gt * CF(i - 1, j, 1, 1)) * idx1;
        J[3] = d[2] + 1. / gt * (grp * CF(i + 1, j, 1, 2) - grm * CF(i - 1, j, 1, 2)) * idx1 +
               1. / gt * (ghp * CF(i, j + 1, 2, 2) - ghm * CF(i, j - 1, 2, 2)) * idx2;
      } else {
        J[1] = 0 + 1. / gt * (ghp * CF(i, j + 1, 2, 1) - ghm * CF(i, j - 1, 2, 1)) * idx2;
        J[2] = 0 + 1. / gt * (grp * CF(i + 1, j, 1, 1) - gt * CF(i - 1, j, 1, 1)) * idx1;
        J[3] = 0 + 1. / gt * (grp * CF(i + 1, j, 1, 2) - grm * CF(i - 1, j, 1, 2)) * idx1 +
               1. / gt * (ghp * CF(i, j + 1, 2, 2) - ghm * CF(i, j - 1, 2, 2)) * idx2;
      }
    }
#undef GC
#undef CF
  s->ccalls++;
  s->clastdt = dt;
}

void ho_init_currents(ho_state *s, const double *p, double dt)
{
  currents_precalc(s, p);
  currents_calc(s, dt);
}

void ho_get_currents(const ho_state *s, double *jcon, double *fcon, double *cfaraday)
{
  const size_t nz = (size_t)s->n1m * s->n2m;
  if (jcon) memcpy(jcon, s->jcon, nz * 4 * sizeof(double));
  if (fcon) memcpy(fcon, s->fcon, nz * 6 * sizeof(double));
  if (cfaraday) memcpy(cfaraday, s->cfar, nz * 15 * sizeof(double));
}

/* ------------------------------------------------------------ public */
ho_state *ho_create(const ho_config *cfg, const double *gcov, const double *gcon, const double *gdet, const double *conn,
                    const double *floors)
{
  ho_state *s = (ho_state *)calloc(1, sizeof(ho_state));
  size_t nz;
  s->c = *cfg;
  s->n1m = cfg->n1 + 2 * NG;
  s->n2m = cfg->n2 + 2 * NG;
  nz = (size_t)s->n1m * s->n2m;
  s->gcov = gcov;
  s->gcon = gcon;
  s->gdet = gdet;
  s->conn = conn;
  s->floors = floors;
  s->pk0 = (double *)calloc(nz * NPR, sizeof(double));
  s->dq = (double *)calloc(nz * NPR, sizeof(double));
  s->pl = (double *)calloc(nz * NPR, sizeof(double));
  s->pr = (double *)calloc(nz * NPR, sizeof(double));
  s->F1 = (double *)calloc(nz * NPR, sizeof(double));
  s->F2 = (double *)calloc(nz * NPR, sizeof(double));
  s->emf = (double *)calloc(nz, sizeof(double));
  s->prc = (double *)calloc(nz * NPR, sizeof(double));
  s->ulast = (double *)calloc(nz * NPR, sizeof(double));
  s->unew = (double *)calloc(nz * NPR, sizeof(double));
  s->gammacheck = (double *)calloc((size_t)(cfg->n1 + 2) * (cfg->n2 + 2), sizeof(double));
  s->cfar = (double *)calloc(nz * 15, sizeof(double));
  s->fcon = (double *)calloc(nz * 6, sizeof(double));
  s->jcon = (double *)calloc(nz * 4, sizeof(double));
  return s;
}

void ho_set_end_time(ho_state *s, double tf, double t, double *dt)
{
  double base = (s->dt_free > 0.) ? s->dt_free : *dt;
  s->c.tf = tf;
  *dt = (t + base > tf) ? tf - t : base;
}

void ho_destroy(ho_state *s)
{
  if (!s) return;
  free(s->pk0); free(s->dq); free(s->pl); free(s->pr); free(s->F1); free(s->F2);
  free(s->emf); free(s->prc); free(s->ulast); free(s->unew); free(s->gammacheck);
  free(s->cfar); free(s->fcon); free(s->jcon);
  free(s->rec_ij); free(s->rec_U); free(s->rec_pr);
  free(s);
}

void ho_bound(ho_state *s, double *prims)
{
  s->pcur = prims;
  bound_prims(s, prims);
}
void ho_bsqflags(ho_state *s, const double *prims, int *pflag) { bsqflags(s, prims, pflag); }

void ho_get_fluxes(const ho_state *s, double *f1, double *f2)
{
  size_t n = (size_t)s->n1m * s->n2m * NPR * sizeof(double);
  memcpy(f1, s->F1, n);
  memcpy(f2, s->F2, n);
}

long ho_ncyclebreak(const ho_state *s) { return s->ncb; }

/* records the inputs of up to max failed inversions from now on */
int ho_record_failures(ho_state *s, int max)
{
  free(s->rec_ij);
  free(s->rec_U);
  free(s->rec_pr);
  s->rec_max = max;
  s->rec_n = 0;
  s->rec_ij = (int *)calloc((size_t)2 * max, sizeof(int));
  s->rec_U = (double *)calloc((size_t)NPR * max, sizeof(double));
  s->rec_pr = (double *)calloc((size_t)NPR * max, sizeof(double));
  return (s->rec_ij && s->rec_U && s->rec_pr) ? 0 : 1;
}

/* copies the recorded failures out (each array sized for max); returns
   their number */
int ho_get_failures(const ho_state *s, int *ij, double *U, double *pr)
{
  if (s->rec_n) {
    memcpy(ij, s->rec_ij, sizeof(int) * 2 * s->rec_n);
    memcpy(U, s->rec_U, sizeof(double) * NPR * s->rec_n);
    memcpy(pr, s->rec_pr, sizeof(double) * NPR * s->rec_n);
  }
  return s->rec_n;
}

int ho_utoprim(ho_state *s, int i, int j, const double *U, double *pr)
{
  geo g = getgeo(s, i, j, CENT);
  return utoprimgen(s, U, &g, pr, &s->ncb);
}

/* diag_flux() for the global region's inner x1 face, diag.c:576-833: the
   fluxes in diagnostic form summed over j, the stress terms 3 and 6 of the
   energy equation from the zone-centred state, and pcum += pdot * Dt */
static void horizon_flux(ho_state *s, const double *p, double Dt)
{
  const int n2 = s->c.n2;
  const double surface = s->c.dx2 * (2.0 * M_PI);
  double pr = 0, pu = 0, t3 = 0, t6 = 0;
  int j;
  for (j = 0; j < n2; j++) {
    geo gf = getgeo(s, 0, j, FACE1);
    const double *F = P(s->F1, 0, j);
    double Fr = F[RHO] * surface, Fu = F[UU] * surface;
    double gr = Fr / gf.g, gu = Fu / gf.g;
    gu += -gr;
    pr += gr * gf.g;
    pu += gu * gf.g;
    geo gc = getgeo(s, 0, j, CENT);
    ostate q;
    state_of(P(p, 0, j), &gc, &q);
    double bsq = 0;
    int l;
    for (l = 0; l < 4; l++) bsq += (q.bcon[l]) * (q.bcov[l]);
    double surgdet = (gc.g) * surface;
    t3 += bsq * (q.ucon[1]) * (q.ucov[0]) * surgdet;
    t6 += -(q.bcon[1]) * (q.bcov[0]) * surgdet;
  }
  s->hz[0] = pr;
  s->hz[1] = pu;
  s->hz[2] = t3;
  s->hz[3] = t6;
  s->hz[4] += pr * Dt;
  s->hz[5] += pu * Dt;
}

void ho_get_horizon(const ho_state *s, double *out) { memcpy(out, s->hz, sizeof(s->hz)); }

/* step_ch_simplempi with the midpoint RK2 of setup_rktimestep,
   step_ch.c:35-188 and 412-429 */
int ho_step(ho_state *s, double *p, int *pflag, double *t, double *dt)
{
  static const double CUf[2][3] = {{1.0, 0.0, 0.5}, {1.0, 0.0, 1.0}};
  static const double Cunew[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 1.0}};
  double ndt = 0.0;
  int to, rc, moved;
  s->pcur = p;
  s->pfcur = pflag;
  s->fail = s->fail_i = s->fail_j = 0;
  for (to = 0; to < 2; to++) {
    const double *pi = p;
    const double *pb = (to == 0) ? p : s->pk0;
    double *pf = (to == 0) ? s->pk0 : p;
    bsqflags(s, pi, pflag);
    if ((rc = advance(s, pi, pb, pf, pflag, CUf[to], Cunew[to], to, to == 1, *dt, &ndt))) return rc;
    if ((rc = bound_prims(s, pf))) return rc;
    bound_pflag(s, pflag);
    checksolution(s, pf, pflag);
    if (!s->c.eom)
      if ((rc = fixup_utoprim(s, pf, pflag))) return rc;
    if ((rc = bound_prims(s, pf))) return rc;
  }
  /* step_ch.c:143-156: Faraday slots and currents at the new time */
  currents_precalc(s, p);
  currents_calc(s, *dt);
  horizon_flux(s, p, *dt);
  moved = *dt > 0.;
  *t += *dt;
  if (ndt > s->c.safe * *dt) ndt = s->c.safe * *dt;
  *dt = ndt;
  if (moved) s->dt_free = ndt; /* a step at dt = 0 (past the end time) keeps the last one */
  if (*t + *dt > s->c.tf) *dt = s->c.tf - *t;
  return 0;
}

void ho_get_fail(const ho_state *s, int *out)
{
  out[0] = s->fail;
  out[1] = s->fail_i;
  out[2] = s->fail_j;
}
