// The UTOPRIMTRYAGAIN retry chain of con-to-prim inversions
// (Utoprimgen_tryagain, step_ch.c:608-626): when the primary inversion
// (Utoprim_2d) leaves a nonzero pflag, the zone's U and guess are restored
// and the next method of the chain runs, until one succeeds:
//   5D1 (utoprim.c + mnewt.c + dudp_calc.c), 2D again, 1D, 1D_OPT,
//   1D_FINAL, 2D_FINAL, 5D2_FINAL.
// A cold path: the chain runs only on the zones whose 2D inversion failed
// (a compacted list), one thread per zone.  Every method is restated with
// the reference's evaluation order so that the chain's result is the
// reference's bit for bit.  Host-and-device, so that the same code can be
// compared with the reference build on the CPU.
#pragma once
#include <string.h>

#include "harm_device.cuh"

namespace harm {
namespace ta {

// method ids of Utoprimgen_pick, step_ch.h:39-53
enum { M_5D1 = 0, M_LDZ = 1, M_2D = 2, M_1D = 3, M_1DOPT = 4, M_1DFINAL = 5, M_2DFINAL = 6, M_5D2 = 7 };
constexpr int PF_CONV = 1;  // UTOPRIMFAILCONV, global.h:550

HD_INLINE double gcov_at(const Geo<double>& g, int j, int k) { return g.gcov[sym(j, k)]; }
HD_INLINE double kdelta(int a, int b) { return (a == b) ? 1.0 : 0.0; }

// primtoU(UNOTHING), phys.c:16-56 and 219-265 (dir 0, no sqrt(-g), T^t_t
// without the rest mass)
HD_INLINE void primtoU_nothing(const double* pr, const State<double>& q, double gam, double* U)
{
  U[RHO] = pr[RHO] * q.ucon[0];
  mhd_row<double, false>(pr, 0, q, gam, &U[UU]);
  U[B1] = pr[B1];
  U[B2] = pr[B2];
  U[B3] = pr[B3];
}

// ------------------------------------------------------------------ 5D1
// dudp_calc_gen, dudp_calc.c:33-225 (REMOVERESTMASSFROMUU < 2, energy
// equation), with dPtodP for the relative 4-velocity (229-272) and the
// helpers of 278-425.  A[r][c] = dU_r/dp_c, r, c over rho, u, u~1..3.
HD_INLINE void dudp_calc_gen(const double* pr, const State<double>& q, const Geo<double>& g, double gam,
                             double A[5][5])
{
  double dutdui[4], dbtdui[4], dbiduj[4][4], dbsqdui[4], dudduu[4][4], dbdiduj[4][4];
  for (int j = 0; j < 5; j++)
    for (int k = 0; k < 5; k++) A[j][k] = 0.;
  const double bsq = dot4(q.bcon, q.bcov);
  // dutdui_calc (308-318): lower(ucon) is q.ucov
  for (int j = 1; j < 4; j++) dutdui[j] = -q.ucov[j] / q.ucov[0];
  // dbtdui_calc (321-333)
  {
    const double B[4] = {0., pr[B1], pr[B2], pr[B3]};
    double Bcov[4];
    lower_v(B, g.gcov, Bcov);
    for (int j = 1; j < 4; j++) dbtdui[j] = Bcov[j] + Bcov[0] * dutdui[j];
  }
  // dbiduj_calc (336-349)
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) dbiduj[j][k] = 0.;
  for (int j = 1; j < 4; j++)
    for (int k = 1; k < 4; k++)
      dbiduj[j][k] = -q.bcon[j] * dutdui[k] / q.ucon[0] + q.ucon[j] * dbtdui[k] / q.ucon[0];
  for (int j = 1; j < 4; j++) dbiduj[j][j] += q.bcon[0] / q.ucon[0];
  for (int j = 1; j < 4; j++) dbiduj[0][j] = dbtdui[j];
  // dbsqdui_calc (352-361): lower(b) is q.bcov
  for (int j = 0; j < 4; j++) dbsqdui[j] = 0.;
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) dbsqdui[j] += 2. * q.bcov[k] * dbiduj[k][j];
  // dudduu_calc (395-401)
  for (int j = 0; j < 4; j++)
    for (int k = 1; k < 4; k++) dudduu[j][k] = gcov_at(g, j, k) + gcov_at(g, j, 0) * dutdui[k];
  // dbdiduj_calc (405-414)
  for (int j = 0; j < 4; j++)
    for (int k = 1; k < 4; k++) {
      dbdiduj[j][k] = 0.0;
      for (int l = 0; l < 4; l++) dbdiduj[j][k] += gcov_at(g, j, l) * dbiduj[l][k];
    }
  const double rho = pr[RHO], ie = pr[UU], P = (gam - 1.0) * ie;
  const double eta = P + rho + ie + bsq;
  A[0][0] = q.ucon[0];
  for (int j = 0; j < 4; j++) A[1 + j][0] = q.ucon[0] * q.ucov[j];
  A[0][1] = 0.0;
  for (int j = 0; j < 4; j++) A[1 + j][1] = gam * q.ucon[0] * q.ucov[j] + kdelta(0, j) * (gam - 1.0);
  for (int j = 1; j < 4; j++) A[0][2 + j - 1] = pr[RHO] * dutdui[j];
  for (int j = 0; j < 4; j++)
    for (int k = 1; k < 4; k++)
      A[1 + j][2 + k - 1] = dbsqdui[k] * q.ucon[0] * q.ucov[j] +
                            eta * (dutdui[k] * q.ucov[j] + q.ucon[0] * dudduu[j][k]) +
                            kdelta(j, 0) * 0.5 * dbsqdui[k] - (dbtdui[k] * q.bcov[j] + q.bcon[0] * dbdiduj[j][k]);
  // dPtodP, VELREL4: dgdvi_calc (278-290), duidvj_calc (293-305)
  double dgdvi[4], duidvj[4][4];
  const double gamma = gamma_of(pr, g);
  for (int j = 1; j < 4; j++) {
    dgdvi[j] = 0.0;
    for (int k = 1; k < 4; k++) dgdvi[j] += 1.0 / gamma * gcov_at(g, j, k) * pr[U1 + k - 1];
  }
  {
    const double alpha = 1.0 / sqrt(-g.gcon[0]);
    double betacon[4];
    for (int j = 1; j < 4; j++) betacon[j] = g.gcon[j] * alpha * alpha;
    for (int j = 1; j < 4; j++)
      for (int k = 1; k < 4; k++) duidvj[j][k] = kdelta(j, k) - betacon[j] / alpha * dgdvi[k];
  }
  for (int i = 0; i < 5; i++) {
    double t[3];
    for (int j = 1; j < 4; j++) {
      double s = 0.;
      for (int l = 1; l < 4; l++) s += A[i][2 + l - 1] * duidvj[l][j];
      t[j - 1] = s;
    }
    for (int j = 0; j < 3; j++) A[i][2 + j] = t[j];
  }
}

// usrfun, utoprim.c:444-575 (GRMHD, NORMMETHOD 1): the normalised residual
// beta = (U(pr) - U_target) norm and Jacobian alpha = dU/dp norm
HD_INLINE void usrfun5(const double* pr, const Geo<double>& g, double gam, const double* Utarget, double beta[5],
                       double alpha[5][5], double* norm)
{
  State<double> q;
  state_of(pr, g, q);
  double Ucur[NPR];
  primtoU_nothing(pr, q, gam, Ucur);
  dudp_calc_gen(pr, q, g, gam, alpha);
  double nrm = 0.0;
  int nterms = 0;
  for (int j = 0; j < 5; j++)
    for (int k = 0; k < 5; k++)
      if (alpha[j][k] > DBL_EPS_REF) {
        nrm += fabs(alpha[j][k]);
        nterms++;
      }
  nrm = (double)nterms / nrm;
  for (int j = 0; j < 5; j++)
    for (int k = 0; k < 5; k++) alpha[j][k] *= nrm;
  for (int k = 0; k < 5; k++) beta[k] = (Ucur[k] - Utarget[k]) * nrm;
  *norm = nrm;
}

// ludcmp + lubksb (Crout LU with implicit row scaling and partial
// pivoting), ludcmp.c:4-62 and lubksb.c:3-24, on a 5 x 5 system (0-based
// here).  A singular row leaves the decomposition unfinished as the
// reference's early return does; the pivots of unfinished columns are then
// the identity (the reference reuses stale static state there).
HD_INLINE void lu_solve5(double a[5][5], double b[5], int indx[5])
{
  double vv[5];
  int singular = 0;
  for (int i = 0; i < 5; i++) {
    double big = 0.0, temp;
    for (int j = 0; j < 5; j++)
      if ((temp = fabs(a[i][j])) > big) big = temp;
    if (big == 0.0) {
      singular = 1;
      break;
    }
    vv[i] = 1.0 / big;
  }
  if (!singular) {
    for (int j = 0; j < 5; j++) {
      int imax = -1;
      for (int i = 0; i < j; i++) {
        double sum = a[i][j];
        for (int k = 0; k < i; k++) sum -= a[i][k] * a[k][j];
        a[i][j] = sum;
      }
      double big = 0.0, dum;
      for (int i = j; i < 5; i++) {
        double sum = a[i][j];
        for (int k = 0; k < j; k++) sum -= a[i][k] * a[k][j];
        a[i][j] = sum;
        if ((dum = vv[i] * fabs(sum)) >= big) {
          big = dum;
          imax = i;
        }
      }
      if (imax < 0) imax = j;  // a NaN column: no pivot found
      if (j != imax) {
        for (int k = 0; k < 5; k++) {
          dum = a[imax][k];
          a[imax][k] = a[j][k];
          a[j][k] = dum;
        }
        vv[imax] = vv[j];
      }
      indx[j] = imax;
      if (a[j][j] == 0.0) a[j][j] = 1.0e-30;
      if (j != 4) {
        dum = 1.0 / (a[j][j]);
        for (int i = j + 1; i < 5; i++) a[i][j] *= dum;
      }
    }
  }
  int ii = -1;
  for (int i = 0; i < 5; i++) {
    const int ip = indx[i];
    double sum = b[ip];
    b[ip] = b[i];
    if (ii >= 0)
      for (int j = ii; j <= i - 1; j++) sum -= a[i][j] * b[j];
    else if (sum != 0.0)
      ii = i;
    b[i] = sum;
  }
  for (int i = 4; i >= 0; i--) {
    double sum = b[i];
    for (int j = i + 1; j < 5; j++) sum -= a[i][j] * b[j];
    b[i] = sum / a[i][i];
  }
}

// mnewt, mnewt.c:13-420 with DODAMP 2, for the 5D inversion (n = 5,
// startp = RHO): damped Newton on x = pr[0..4].  Returns 0 when converged
// (or within the allowed tolerances), 1 otherwise.
HD_INLINE int mnewt5(int ntrial, int mintrial, double* x, const Geo<double>& g, double gam, const double* Utarget,
                     double tolx, double tolf, double tolxallowed, double tolfallowed)
{
  const double abstol = DBL_EPS_REF * 50.0, abstolhard = DBL_EPS_REF;
  if (tolx < abstol) tolx = abstol;
  if (tolf < abstol) tolf = abstol;
  double errx = 1.E30, errf = 1.E30, lasterrf = 0.;
  double dampfactor = 1.0;
  const double dampfactorchange = 0.5;
  int allownewdamp = 0, countstable = 0, countdamped = 0, dampdeath = 0;
  const int numstabletot = 5, numdampedtot = 5;
  int lowtol[2] = {0, 0};
  int indx[5] = {0, 1, 2, 3, 4};
  double xold[5], fvec[5], fjac[5][5], pp[5], pptest[5], normf;
  for (int i = 0; i < 5; i++) xold[i] = x[i];
  for (int k = 1; k <= ntrial; k++) {
    usrfun5(x, g, gam, Utarget, fvec, fjac, &normf);
    errf = 0.0;
    for (int i = 0; i < 5; i++) errf += fabs(fvec[i]);
    errf /= normf;
    if (errf <= abstolhard) lowtol[1] = 2;
    else if (errf <= tolf) lowtol[1] = 1;
    else lowtol[1] = 0;
    if (allownewdamp && (k > 1) && (lasterrf < errf)) {
      // the error grew: halve the damping factor and step back
      countdamped++;
      if (countdamped >= numdampedtot) {
        allownewdamp = 0;
        countdamped = 0;
        countstable = 0;
      }
      dampfactor *= dampfactorchange;
      dampdeath = 0;
      if ((dampfactor < 1E-5) && (errf < tolf * 100.0)) dampdeath = 1;
      else if (dampfactor < 1E-7) dampdeath = 1;
      if (dampdeath == 0) {
        for (int i = 0; i < 5; i++) x[i] = xold[i];
        k--;
      }
    } else {
      if (allownewdamp == 0) countstable++;
      if (allownewdamp) countdamped++;
      if (countstable >= numstabletot) {
        allownewdamp = 1;
        countdamped = 0;
        countstable = 0;
      }
      if (countdamped >= numdampedtot) {
        allownewdamp = 0;
        countdamped = 0;
        countstable = 0;
      }
      lasterrf = errf;
      for (int i = 0; i < 5; i++) xold[i] = x[i];
      for (int i = 0; i < 5; i++) pp[i] = -fvec[i];
      lu_solve5(fjac, pp, indx);
      for (int i = 0; i < 5; i++) pptest[i] = dampfactor * pp[i];
      // keep rho and u positive (a smaller step instead)
      const double testrho = x[RHO] + pptest[RHO], testu = x[UU] + pptest[UU];
      int redamp = 0;
      double redampfactor, redampfactorrho, redampfactoru;
      redampfactor = redampfactorrho = redampfactoru = dampfactor;
      if (testrho < 0) {
        redampfactorrho = -x[RHO] / pp[RHO] * 0.1;
        redamp = 1;
      }
      if (testu < 0) {
        redampfactoru = -x[UU] / pp[UU] * 0.1;
        redamp = 1;
      }
      if (redamp) {
        if (redampfactorrho < redampfactoru) redampfactor = redampfactorrho;
        else redampfactor = redampfactoru;
        for (int i = 0; i < 5; i++) pptest[i] = redampfactor * pp[i];
        if (redampfactor < 1E-7) {
          dampdeath = 1;
          break;
        }
      }
      for (int i = 0; i < 5; i++) pp[i] = pptest[i];
      errx = 0.0;
      for (int i = 0; i < 5; i++) {
        errx += fabs(pp[i]);
        x[i] += pp[i];
      }
      if (errx <= abstolhard) lowtol[0] = 2;
      else if (errx <= tolx) lowtol[0] = 1;
      else lowtol[0] = 0;
    }
    if (dampdeath) break;
    if (k > mintrial)
      if ((lowtol[0] >= 1) && (lowtol[1] >= 1)) break;
  }
  if ((lowtol[0] >= 1) && (lowtol[1] >= 1)) return 0;
  if ((errf <= tolfallowed) && (errx <= tolxallowed)) return 0;
  return 1;
}

// Utoprim (5D1), utoprim.c:24-318 with EVOLVENOENTROPY, PRECISEINVERSION 1
// and nutoprims = 1.  Ug: geometry-free U (UNOTHING); pr: guess in, result
// out.  Returns the pflag code.
HD_INLINE int utoprim_5d1(const double* Ug, const Geo<double>& g, double gam, double* pr)
{
  for (int k = B1; k <= B3; k++) pr[k] = Ug[k];
  double pr0[NPR], priter[NPR], Utarget[NPR], Ustart[NPR], dU[NPR];
  for (int k = 0; k < NPR; k++) pr0[k] = priter[k] = pr[k];
  for (int k = 0; k < NPR; k++) Utarget[k] = Ug[k];
  {
    State<double> q;
    state_of(pr, g, q);
    primtoU_nothing(pr, q, gam, Ustart);
  }
  for (int k = 0; k < NPR; k++) dU[k] = Utarget[k] - Ustart[k];
  // one pass of the backing-off loop (countutoprims = 1, frac = 1)
  const int countutoprims = 1;
  const double frac = 1.0 / ((double)1);
  for (int k = 0; k < NPR; k++) Utarget[k] = Ustart[k] + dU[k] * (double)countutoprims * frac;
  const int failed = mnewt5(200, 3, priter, g, gam, Utarget, 1.e-11, 1.e-11, 1.e-8, 1.e-8);
  for (int k = 0; k < NPR; k++) pr[k] = priter[k];
  if (failed) {
    for (int k = 0; k < NPR; k++) pr[k] = pr0[k];
    return PF_CONV;
  }
  if ((pr[RHO] < 0.0) || (pr[UU] < 0.0)) {
    int code = 0;
    if ((pr[RHO] <= 0.) && (pr[UU] >= 0.)) code = PF_RHONEG;
    if ((pr[RHO] >= 0.) && (pr[UU] <= 0.)) code = PF_UNEG;
    if ((pr[RHO] <= 0.) && (pr[UU] <= 0.)) code = PF_RHOUNEG;
    return code;
  }
  return PF_NOFAIL;
}

// ------------------------------------------------------------------ Noble et al.
// The 1D / 1D_OPT / 1D_FINAL / 2D_FINAL inversions share the scalars of
// their Utoprim_new_body (utoprim_1d.c:124-212 and the same lines of the
// other files): B^2, (Q.B)^2, Q~^2, Q.n, D, and w of the guess.
struct Noble {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, wglobal, gam, gammafail;
  double QdotB, Bcon[4], Qcon[4], ncon[4];
};

constexpr double N_W_TOO_BIG = 1.e9, N_FAIL_VAL = 1.e30, N_MAXNEGUTSQ = 1E-10;
constexpr double N_NEWT_TOL = 1.0e-15, N_MIN_NEWT_TOL = 1.0e-10, N_GRADMIN = 1.0e-10, N_NEWT_FUNC_TOL = 1.0e-5;
constexpr double N_SCALEMAX = 1.0e2;
constexpr int N_MAX_NEWT_ITER = 200, N_EXTRA_NEWT_ITER = 2;
// the line search of the 1D solvers gives up after this many halvings
// (the reference loops until its step is below its minimum, which any
// finite input reaches long before)
constexpr int N_LNSRCH_MAX = 4000;

// the deterministic cycle-break factor (the same hash as the 2D solver's)
HD_INLINE double cycle_break_hd(double x0, double x1, int n_iter)
{
  uint64_t a, b;
  memcpy(&a, &x0, 8);
  memcpy(&b, &x1, 8);
  const uint64_t h = mix64(a ^ mix64(b ^ (uint64_t)(uint32_t)n_iter));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// Utoprim_new_body's set-up of the shared scalars from U (the rescaled
// conserved vector: alpha rho u^t, +-alpha T^t_mu, alpha B^i)
HD_INLINE void noble_setup(const double* U, const Geo<double>& g, double gam, double gammafail, Noble& c)
{
  double Bcov[4], Qcov[4], ncov[4];
  c.Bcon[0] = 0.;
  for (int i = 1; i < 4; i++) c.Bcon[i] = U[B1 + i - 1];
  lower_g(c.Bcon, g.gcov, Bcov);
  for (int i = 0; i < 4; i++) Qcov[i] = U[UU + i];
  lower_g(Qcov, g.gcon, c.Qcon);  // raise_g: the same sums with g^{mu nu}
  c.Bsq = 0.;
  for (int i = 1; i < 4; i++) c.Bsq += c.Bcon[i] * Bcov[i];
  c.QdotB = 0.;
  for (int i = 0; i < 4; i++) c.QdotB += Qcov[i] * c.Bcon[i];
  c.QdotBsq = c.QdotB * c.QdotB;
  const double lapse = sqrt(-1. / g.gcon[0]);
  ncov[0] = -lapse;
  ncov[1] = ncov[2] = ncov[3] = 0.;
  lower_g(ncov, g.gcon, c.ncon);
  c.Qdotn = c.Qcon[0] * ncov[0];
  double Qsq = 0.;
  for (int i = 0; i < 4; i++) Qsq += Qcov[i] * c.Qcon[i];
  c.Qtsq = Qsq + c.Qdotn * c.Qdotn;
  c.D = U[RHO];
  c.gam = gam;
  c.gammafail = gammafail;
}

// u~^2 of the guess (the sums of utoprim_1d.c:190-192)
HD_INLINE double guess_utsq(const double* prim, const Geo<double>& g)
{
  double utsq = 0.;
  for (int i = 1; i < 4; i++)
    for (int j = 1; j < 4; j++) utsq += gcov_at(g, i, j) * prim[U1 + i - 1] * prim[U1 + j - 1];
  return utsq;
}

// --- 1D and 1D_OPT (utoprim_1d.c, utoprim_1d_opt.c): Newton on W
// utsq_calc, utoprim_1d.c:324-358
HD_INLINE double n1_utsq(const Noble& c, double W)
{
  const double Wsq = W * W;
  const double tmp = c.QdotBsq * (c.Bsq + 2 * W) + c.Qtsq * Wsq;
  return tmp / (Wsq * (W + c.Bsq) * (W + c.Bsq) - tmp);
}

// func_1d_orig and res_sq_1d_orig, utoprim_1d.c:846-932 (the opt file's
// only differ in the unreachable utsq < 0 branch)
HD_INLINE double n1_resid(const Noble& c, double W, double* gamma_out, double* gamma_sq_out)
{
  const double Wsq = W * W;
  const double utsq = fabs(n1_utsq(c, W));
  const double gamma = (utsq < 0.) ? (1. + 1.0e-15) : sqrt(1. + utsq);
  const double gamma_sq = gamma * gamma;
  const double rho0 = c.D / gamma;
  const double w = W / gamma_sq;
  const double p_tmp = (c.gam - 1.) * (w - rho0) / c.gam;
  *gamma_out = gamma;
  *gamma_sq_out = gamma_sq;
  return +W + c.Bsq * (1. - 0.5 / gamma_sq) - 0.5 * c.QdotBsq / Wsq - c.Qdotn - p_tmp;
}

// dgamma_dW and dpress_dW, utoprim_1d.c:935-983
HD_INLINE double n1_dgamma_dW(const Noble& c, double W, double gamma)
{
  const double Wsq = W * W;
  const double tmp = -c.QdotBsq * (c.Bsq + 2 * W) + Wsq * (c.Bsq * (c.Bsq + 2 * W) - c.Qtsq + Wsq);
  const double tmp3 = W * (c.Bsq + W);
  if (tmp > 0.) {
    const double tmp2 = tmp3 * sqrt(tmp);
    return -((W * (c.Bsq + W) * (c.Bsq * c.QdotBsq * (c.Bsq + 3 * W) + Wsq * (3 * c.QdotBsq + c.Qtsq * W))) /
             (tmp * tmp2));
  }
  return 0.5 * gamma / W;
}

HD_INLINE void n1_func(const Noble& c, double W, double& dx, double& resid, double& jac, double& f, double& df)
{
  double gamma, gamma_sq;
  resid = n1_resid(c, W, &gamma, &gamma_sq);
  const double Wsq = W * W;
  const double dg = n1_dgamma_dW(c, W, gamma);
  const double dpdW = ((c.gam - 1.) * (-2 * dg * W + gamma * (1.0 + c.D * dg))) / (gamma * gamma * gamma * c.gam);
  const double drdW = 1. - dpdW + c.QdotBsq / (Wsq * W) + c.Bsq * dg / (gamma * gamma_sq);
  jac = drdW;
  dx = -resid / drdW;
  f = 0.5 * resid * resid;
  df = -2. * f;
}

HD_INLINE double n1_res_sq(const Noble& c, double W)
{
  double gamma, gamma_sq;
  const double r = n1_resid(c, W, &gamma, &gamma_sq);
  return 0.5 * r * r;
}

// my_lnsrch, utoprim_1d.c:1003-1134 (n = 1): backtracking line search
// along p from xold.  check: 0 ok, 1 step too small, 2 bad step.
template <bool FINAL>
HD_INLINE void n1_lnsrch(const Noble& c, double xold, double fold, double g, double p, double& x, double& f,
                         double TOLX, double stpmax, int& check)
{
  double a, alam, alam2 = 0., alamin, b, disc, f2 = 0., fold2 = 0., rhs1, rhs2, slope, sum, temp, test, tmplam = 0.;
  check = 0;
  sum = 0.0;
  sum += p * p;
  sum = sqrt(sum);
  if (sum > stpmax) p *= stpmax / sum;
  slope = 0.0;
  slope += g * p;
  test = 0.0;
  temp = (xold == 0.) ? fabs(p) : fabs(p / xold);
  if (temp > test) test = temp;
  alamin = TOLX / test;
  alam = 1.0;
  for (int it = 0; it < N_LNSRCH_MAX; it++) {
    x = xold + alam * p;
    f = n1_res_sq(c, x);
    const int bad_step = FINAL ? (isfinite(f) == 0) : (x <= 0.);
    if (bad_step) {
      check = 2;
      return;
    }
    if (alam < alamin) {
      x = xold;
      check = 1;
      return;
    } else if (f <= fold + 1.0e-4 * alam * slope) {
      return;
    } else {
      if (alam == 1.0) {
        tmplam = -slope / (2.0 * (f - fold - slope));
      } else {
        rhs1 = f - fold - alam * slope;
        rhs2 = f2 - fold2 - alam2 * slope;
        a = (rhs1 / (alam * alam) - rhs2 / (alam2 * alam2)) / (alam - alam2);
        b = (-alam2 * rhs1 / (alam * alam) + alam * rhs2 / (alam2 * alam2)) / (alam - alam2);
        if (a == 0.0) tmplam = -slope / (2.0 * b);
        else {
          disc = b * b - 3.0 * a * slope;
          if (disc < 0.0) disc = 0.;
          else tmplam = (-b + sqrt(disc)) / (3.0 * a);
        }
        if (tmplam > 0.5 * alam) tmplam = 0.5 * alam;
      }
    }
    alam2 = alam;
    f2 = f;
    fold2 = fold;
    alam = rmax(tmplam, 0.1 * alam);
  }
  check = 1;
}

// general_newton_raphson of utoprim_1d.c:496-716 (OPT = false) and
// utoprim_1d_opt.c:560-870 (OPT = true), n = 1.  LS: line search (the retry
// after a failed plain solve).
template <bool OPT, int LS>
HD_INLINE int n1_gnr(const Noble& c, double& x)
{
  double f, df, dx, resid, jac, errx, errx_old, errx_oldest, x_old, x_orig, resid_norm = 1.0;
  int retval = 0, n_iter = 0, i_extra = 0, doing_extra = 0;
  errx = 1.;
  errx_old = 2.;
  df = f = 1.;
  x_old = x_orig = x;
  bool keep_iterating = true;
  while (keep_iterating) {
    n1_func(c, x, dx, resid, jac, f, df);
    if (n_iter == 0) {
      resid_norm = 0.0e0;
      resid_norm += fabs(resid);
      resid_norm /= 1.0 * 1;
      if (resid_norm == 0.0) resid_norm = 1.0;
    }
    if (!OPT) {
      // the cycle break every 10th iteration (CYCLE_BREAK_PERIOD of
      // utoprim_1d2d.h; the opt file compiles it out)
      if (((n_iter + 1) % 10) == 0) dx *= cycle_break_hd(x, 0.0, n_iter);
    }
    errx_oldest = errx_old;
    errx_old = errx;
    errx = 0.;
    const double f_old = f;
    x_old = x;
    if (LS == 1) {
      double tmp = 0.;
      tmp += jac * resid;
      const double del_f = tmp;
      const double dn = dx;
      n1_lnsrch<false>(c, x_old, f_old, del_f, dn, x, f, N_NEWT_TOL, N_SCALEMAX, retval);
      dx = x - x_old;
      if (retval == 1) {
        double resid_check = 0.0e0;
        resid_check += fabs(resid);
        resid_check /= 1.0 * 1;
        if (resid_check <= resid_norm * N_NEWT_FUNC_TOL) retval = 0;
      }
      if (retval == 1) {
        double grad_check = 0.0e0;
        double resid_check = (x == 0.) ? 1.0 : fabs(x);
        grad_check += del_f * resid_check;
        resid_check = (f == 0.) ? 1.0 : fabs(f);
        grad_check /= resid_check;
        if (grad_check > N_GRADMIN) retval = -1;
      }
    } else {
      x += dx;
    }
    errx += (x == 0.) ? fabs(dx) : fabs(dx / x);
    errx /= 1. * 1;
    x = fabs(x);
    if (!OPT) x = (x > N_W_TOO_BIG) ? x_old : x;
    if (((errx_old == errx) || (errx_oldest == errx)) && (errx <= N_MIN_NEWT_TOL)) errx = -errx;
    if ((retval == 1) || (retval == -1)) errx = -errx;
    if ((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0) && (N_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0)) || (i_extra > N_EXTRA_NEWT_ITER) ||
        (n_iter >= (N_MAX_NEWT_ITER - 1)))
      keep_iterating = false;
    n_iter++;
  }
  if (OPT) x = (x > N_W_TOO_BIG) ? x_old : x;
  if ((fabs(errx) > N_MIN_NEWT_TOL) && (i_extra == 0)) {
    if (LS != 0) return 1;
    // the plain solve failed: again from the start with line searching
    double xo = x_orig;
    const int retval2 = n1_gnr<OPT, (LS == 0) ? 1 : 0>(c, xo);
    x = xo;
    return retval2;
  }
  return 0;
}

// Utoprim_1d / Utoprim_1d_opt with their Utoprim_new_body (utoprim_1d.c:19-321,
// utoprim_1d_opt.c:19-375).  Ug: geometry-free U; prim: guess in, result out.
template <bool OPT>
HD_INLINE int utoprim_1d_family(const double* Ug, const Geo<double>& g, double gam, double gammafail, double* prim)
{
  const double alpha = 1.0 / sqrt(-g.gcon[0]);
  double U[NPR], pr[NPR];
  U[RHO] = alpha * Ug[RHO];
  for (int i = UU; i <= U3; i++) U[i] = -alpha * Ug[i];
  for (int i = B1; i <= B3; i++) U[i] = alpha * Ug[i];
  for (int i = 0; i < B1; i++) pr[i] = prim[i];
  for (int i = B1; i <= B3; i++) pr[i] = alpha * prim[i];
  int pfl = PF_NOFAIL;
  // body
  do {
    for (int i = B1; i <= B3; i++) pr[i] = U[i];
    Noble c;
    noble_setup(U, g, gam, gammafail, c);
    const double utsq_too_big = (gammafail - 1.0) * (gammafail - 1.0);
    double utsq = guess_utsq(pr, g);
    if (!OPT) {
      if ((utsq < 0.) && (fabs(utsq) < N_MAXNEGUTSQ)) utsq = 0.0;
      if (utsq < 0. || utsq > utsq_too_big) {
        pfl = PF_CONVUTSQ;
        break;
      }
    }
    double rho0 = pr[RHO], u = pr[UU];
    double p = (gam - 1.) * u;
    double w = rho0 + u + p;
    double gammasq = 1. + utsq;
    double x = w * gammasq;
    c.wglobal = w;
    const int ret = n1_gnr<OPT, 0>(c, x);
    const double W = x;
    if ((ret != 0) || (W == N_FAIL_VAL)) {
      pfl = ret * 100 + 1;
      break;
    }
    const double Wtest = W / c.wglobal;
    if (Wtest <= 0. || Wtest > N_W_TOO_BIG) {
      pfl = PF_CONVW;
      break;
    }
    utsq = n1_utsq(c, W);
    if ((utsq < 0.) && (fabs(utsq) < N_MAXNEGUTSQ)) utsq = 0.0;
    if (utsq < 0. || utsq > utsq_too_big) {
      if (OPT || fabs(utsq) > 1.0e-14) {
        pfl = PF_CONVUTSQ2;
        break;
      }
    }
    double gamma;
    if (!OPT) {
      gammasq = 1. + utsq;
      gamma = sqrt(gammasq);
      rho0 = sqrt(c.D * c.D / gammasq);
      w = W / gammasq;
      p = (gam - 1.) * (w - rho0) / gam;
      u = w - rho0 - p;
      if ((rho0 <= 0.) || (u <= 0.)) {
        if ((rho0 <= 0.) && (u >= 0.)) pfl = PF_RHONEG;
        if ((rho0 >= 0.) && (u <= 0.)) pfl = PF_UNEG;
        if ((rho0 <= 0.) && (u <= 0.)) pfl = PF_RHOUNEG;
      }
    } else {
      gamma = sqrt(1. + utsq);
      rho0 = c.D / gamma;
      w = W / (gamma * gamma);
      p = (gam - 1.) * (w - rho0) / gam;
      u = w - (rho0 + p);
      if ((rho0 <= 0.) || (u < 0.)) {
        if ((rho0 <= 0.) && (u >= 0.)) pfl = PF_RHONEG;
        if ((rho0 >= 0.) && (u < 0.)) pfl = PF_UNEG;
        if ((rho0 <= 0.) && (u < 0.)) pfl = PF_RHOUNEG;
      }
    }
    pr[RHO] = rho0;
    pr[UU] = u;
    double Qtcon[4];
    for (int i = 1; i < 4; i++) Qtcon[i] = c.Qcon[i] + c.ncon[i] * c.Qdotn;
    for (int i = 1; i < 4; i++)
      pr[U1 + i - 1] = -gamma * Qtcon[i] / (W + c.Bsq) - gamma * c.QdotB * c.Bcon[i] / (W * (W + c.Bsq));
    for (int i = B1; i <= B3; i++) pr[i] = U[i];
  } while (0);
  for (int i = 0; i < B1; i++) prim[i] = pr[i];
  for (int i = B1; i <= B3; i++) prim[i] = pr[i] / alpha;
  return pfl;
}

// --- 1D_FINAL and 2D_FINAL (utoprim_1d_final.c, utoprim_2d_final.c): Newton
// on W (1D) or (W, v^2) (2D), the "final" residuals of u2p_defs.h's family
HD_INLINE double nf_vsq(const Noble& c, double W)
{
  const double Wsq = W * W;
  const double Xsq = (c.Bsq + W) * (c.Bsq + W);
  return (Wsq * c.Qtsq + c.QdotBsq * (c.Bsq + 2. * W)) / (Wsq * Xsq);
}

HD_INLINE double nf_dvsq_dW(const Noble& c, double W)
{
  const double X = c.Bsq + W;
  const double Wsq = W * W;
  const double W3 = Wsq * W;
  const double X3 = X * X * X;
  return -2. * (c.Qtsq / X3 + c.QdotBsq * (3 * W * X + c.Bsq * c.Bsq) / (W3 * X3));
}

HD_INLINE double nf_pressure_W_vsq(const Noble& c, double W, double vsq)
{
  const double gtmp = 1. - vsq;
  return (c.gam - 1.) * (W * gtmp - c.D * sqrt(gtmp)) / c.gam;
}
HD_INLINE double nf_dpdW(const Noble& c, double vsq) { return (c.gam - 1.) * (1. - vsq) / c.gam; }
HD_INLINE double nf_dpdvsq(const Noble& c, double W, double vsq)
{
  return (c.gam - 1.) * (0.5 * c.D / sqrt(1. - vsq) - W) / c.gam;
}

HD_INLINE double nf_vsq_too_big(const Noble& c) { return 1.0 - 1.0 / ((c.gammafail - 1.0) + 1.0); }
constexpr double NF_MAXNEGVSQ = (1.0 - 1.0 / (N_MAXNEGUTSQ + 1.0));

// func_1d_orig, utoprim_1d_final.c:907-1001 (OPTIMIZED)
HD_INLINE void nf1_func(const Noble& c, double W, double& dx, double& f, double& df)
{
  const double Wsq = W * W;
  double vsq = nf_vsq(c, W);
  vsq = (vsq < -NF_MAXNEGVSQ) ? 0.0 : fabs(vsq);
  vsq = (vsq > 1.) ? nf_vsq_too_big(c) : vsq;
  const double p_tmp = nf_pressure_W_vsq(c, W, vsq);
  const double dvsq = nf_dvsq_dW(c, W);
  const double dp1 = nf_dpdW(c, vsq);
  const double dp2 = nf_dpdvsq(c, W, vsq);
  const double dpdW = dp1 + dp2 * dvsq;
  const double resid = +W + 0.5 * c.Bsq * (1. + vsq) - 0.5 * c.QdotBsq / Wsq + c.Qdotn - p_tmp;
  const double drdW = 1. - dpdW + c.QdotBsq / (Wsq * W) + 0.5 * c.Bsq * dvsq;
  dx = -resid / drdW;
  f = 0.5 * resid * resid;
  df = -2. * f;
}

// general_newton_raphson, utoprim_1d_final.c:511-900 with USE_LINE_SEARCH
// -2 (no line search), NEWCONVERGE 1, CHECK_FOR_STALL 0
HD_INLINE int nf1_gnr(const Noble& c, double& x)
{
  double f = 1., df = 1., dx, errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep_iterating = true;
  while (keep_iterating) {
    nf1_func(c, x, dx, f, df);
    errx = 0.;
    x += dx;
    int i_increase = 0;
    while (((x * x * x * (x + 2. * c.Bsq) - c.QdotBsq * (2. * x + c.Bsq)) <= x * x * (c.Qtsq - c.Bsq * c.Bsq)) &&
           (i_increase < 10)) {
      x -= (1. * i_increase) * dx / 10.;
      i_increase++;
    }
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0) && (N_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0)) || (i_extra > N_EXTRA_NEWT_ITER) ||
        (n_iter >= (N_MAX_NEWT_ITER - 1)))
      keep_iterating = false;
    n_iter++;
  }
  if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x) == 0)) return 1;
  if (fabs(errx) > N_MIN_NEWT_TOL) return 1;
  return 0;
}

// func_vsq2, utoprim_2d_final.c:1082-1157
HD_INLINE void nf2_func(const Noble& c, const double* x, double* dx, double& f, double& df)
{
  const double W = x[0], vsq = x[1];
  const double Wsq = W * W;
  const double p_tmp = nf_pressure_W_vsq(c, W, vsq);
  const double dPdW = nf_dpdW(c, vsq);
  const double dPdvsq = nf_dpdvsq(c, W, vsq);
  const double Bsq = c.Bsq, QdotBsq = c.QdotBsq;
  const double t2 = -0.5 * Bsq + dPdvsq;
  const double t3 = Bsq + W;
  const double t4 = t3 * t3;
  const double t9 = 1 / Wsq;
  const double t11 = c.Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.0 * W) * t9;
  const double t16 = QdotBsq * t9;
  const double t18 = -c.Qdotn - 0.5 * Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
  const double t21 = 1 / t3;
  const double t23 = 1 / W;
  const double t24 = t16 * t23;
  const double t25 = -1.0 + dPdW - t24;
  const double t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
  const double t36 = 1 / t35;
  dx[0] = -(t2 * t11 + t4 * t18) * t21 * t36;
  const double t40 = (vsq + t24) * t3;
  dx[1] = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
  const double r0 = t11, r1 = t18;
  df = -r0 * r0 - r1 * r1;
  f = -0.5 * (df);
}

// general_newton_raphson + validate_x, utoprim_2d_final.c:617-950 with
// USE_LINE_SEARCH -2, NEWCONVERGE 1, CHECK_FOR_STALL 0
HD_INLINE int nf2_gnr(const Noble& c, double* x)
{
  const double gsq_too_big = c.gammafail * c.gammafail;
  double f = 1., df = 1., dx[2], x_old[2], errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep_iterating = true;
  while (keep_iterating) {
    nf2_func(c, x, dx, f, df);
    errx = 0.;
    x_old[0] = x[0];
    x_old[1] = x[1];
    x[0] += dx[0];
    x[1] += dx[1];
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    // validate_x
    x[0] = fabs(x[0]);
    x[0] = (x[0] / c.wglobal > gsq_too_big) ? x_old[0] : x[0];
    x[1] = (x[1] < 0.) ? 0.0 : x[1];
    x[1] = (x[1] > 1.) ? nf_vsq_too_big(c) : x[1];
    if ((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0) && (N_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0)) || (i_extra > N_EXTRA_NEWT_ITER) ||
        (n_iter >= (N_MAX_NEWT_ITER - 1)))
      keep_iterating = false;
    n_iter++;
  }
  if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x[0]) == 0) || (isfinite(x[1]) == 0)) return 1;
  if (fabs(errx) > N_MIN_NEWT_TOL) return 1;
  return 0;
}

// Utoprim_1d_final / Utoprim_2d_final with their Utoprim_new_body
// (utoprim_1d_final.c:26-397, utoprim_2d_final.c:26-397)
template <bool TWO_D>
HD_INLINE int utoprim_final_family(const double* Ug, const Geo<double>& g, double gam, double gammafail, double* prim)
{
  for (int i = B1; i <= B3; i++) prim[i] = Ug[i];
  const double alpha = 1.0 / sqrt(-g.gcon[0]);
  double U[NPR], pr[NPR];
  for (int i = RHO; i <= B3; i++) U[i] = alpha * Ug[i];
  for (int i = 0; i < B1; i++) pr[i] = prim[i];
  for (int i = B1; i <= B3; i++) pr[i] = alpha * prim[i];
  int pfl = PF_NOFAIL, retval = 0;
  do {
    for (int i = B1; i <= B3; i++) pr[i] = U[i];
    Noble c;
    noble_setup(U, g, gam, gammafail, c);
    double utsq = guess_utsq(pr, g);
    if ((utsq < 0.) && (fabs(utsq) < N_MAXNEGUTSQ)) utsq = 0.0;
    if (utsq < 0. || utsq > (gammafail - 1.0) * (gammafail - 1.0)) {
      pfl = PF_CONVUTSQ;
      retval = 1;
      break;
    }
    const double gammasq = 1. + utsq;
    double gamma = sqrt(gammasq);
    double rho0 = c.D / gamma;
    double u = pr[UU];
    double p = (gam - 1.) * u;
    double w = rho0 + u + p;
    double W_last = w * gammasq;
    int i_increase = 0;
    while (((W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq)) <=
            W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq)) &&
           (i_increase < 10)) {
      W_last *= 10.;
      i_increase++;
    }
    c.wglobal = w;
    double W;
    if (TWO_D) {
      // find_root_2D_gen, utoprim_2d_final.c:514-590 (MAX_NEWT_RETRIES 0)
      double x[2];
      x[0] = fabs(W_last);
      const double v0 = fabs(nf_vsq(c, W_last));
      x[1] = (v0 > 1.) ? nf_vsq_too_big(c) : v0;
      retval = nf2_gnr(c, x);
      W = x[0];
    } else {
      double x = W_last;
      retval = nf1_gnr(c, x);
      W = x;
    }
    if ((retval != 0) || (W == N_FAIL_VAL)) {
      pfl = retval * 100 + 1;
      break;
    }
    const double Wtest = W / c.wglobal;
    if (Wtest <= 0. || Wtest > gammafail * gammafail) {
      pfl = PF_CONVW;
      break;
    }
    double vsq = nf_vsq(c, W);
    if ((vsq < 0.) && (fabs(vsq) < NF_MAXNEGVSQ)) vsq = 0.0;
    if ((vsq > nf_vsq_too_big(c)) || (vsq < 0.0)) {
      pfl = PF_CONVUTSQ2;
      break;
    }
    const double gtmp = sqrt(1. - vsq);
    gamma = 1. / gtmp;
    rho0 = c.D * gtmp;
    w = W * (1. - vsq);
    p = (gam - 1.) * (w - rho0) / gam;
    u = w - (rho0 + p);
    if ((rho0 <= 0.) || (u < 0.)) {
      if ((rho0 <= 0.) && (u >= 0.)) pfl = PF_RHONEG;
      if ((rho0 > 0.) && (u < 0.)) pfl = PF_UNEG;
      if ((rho0 <= 0.) && (u < 0.)) pfl = PF_RHOUNEG;
    }
    pr[RHO] = rho0;
    pr[UU] = u;
    double Qtcon[4];
    for (int i = 1; i < 4; i++) Qtcon[i] = c.Qcon[i] + c.ncon[i] * c.Qdotn;
    for (int i = 1; i < 4; i++) pr[U1 + i - 1] = gamma / (W + c.Bsq) * (Qtcon[i] + c.QdotB * c.Bcon[i] / W);
    for (int i = B1; i <= B3; i++) pr[i] = U[i];
  } while (0);
  if (retval == 0)
    for (int i = 0; i < B1; i++) prim[i] = pr[i];
  return pfl;
}

// ------------------------------------------------------------------ 5D2
// dudp_calc_g, utoprim_5d2_final.c:434-565 (eta = rho + gam u + b^2 here)
HD_INLINE void dudp_calc_g5(const double* pr, const State<double>& q, const Geo<double>& g, double gam,
                            double A[5][5])
{
  double dutdui[4], dbtdui[4], dbiduj[4][4], dbsqdui[4], dudduu[4][4], dbdiduj[4][4];
  for (int j = 0; j < 5; j++)
    for (int k = 0; k < 5; k++) A[j][k] = 0.;
  const double bsq = dot4(q.bcon, q.bcov);
  for (int j = 1; j < 4; j++) dutdui[j] = -q.ucov[j] / q.ucov[0];
  {
    const double B[4] = {0., pr[B1], pr[B2], pr[B3]};
    double Bcov[4];
    lower_v(B, g.gcov, Bcov);
    for (int j = 1; j < 4; j++) dbtdui[j] = Bcov[j] + Bcov[0] * dutdui[j];
  }
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) dbiduj[j][k] = 0.;
  for (int j = 1; j < 4; j++)
    for (int k = 1; k < 4; k++)
      dbiduj[j][k] = -q.bcon[j] * dutdui[k] / q.ucon[0] + q.ucon[j] * dbtdui[k] / q.ucon[0];
  for (int j = 1; j < 4; j++) dbiduj[j][j] += q.bcon[0] / q.ucon[0];
  for (int j = 1; j < 4; j++) dbiduj[0][j] = dbtdui[j];
  for (int j = 0; j < 4; j++) dbsqdui[j] = 0.;
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) dbsqdui[j] += 2. * q.bcov[k] * dbiduj[k][j];
  for (int j = 0; j < 4; j++)
    for (int k = 1; k < 4; k++) dudduu[j][k] = gcov_at(g, j, k) + gcov_at(g, j, 0) * dutdui[k];
  for (int j = 0; j < 4; j++)
    for (int k = 1; k < 4; k++) {
      dbdiduj[j][k] = 0.0;
      for (int l = 0; l < 4; l++) dbdiduj[j][k] += gcov_at(g, j, l) * dbiduj[l][k];
    }
  const double eta = pr[RHO] + gam * pr[UU] + bsq;
  A[RHO][RHO] = q.ucon[0];
  for (int j = 0; j < 4; j++) A[UU + j][RHO] = q.ucon[0] * q.ucov[j];
  A[RHO][UU] = 0.0;
  for (int j = 0; j < 4; j++) A[UU + j][UU] = gam * q.ucon[0] * q.ucov[j] + kdelta(0, j) * (gam - 1.0);
  for (int j = 1; j < 4; j++) A[RHO][U1 + j - 1] = pr[RHO] * dutdui[j];
  for (int j = 0; j < 4; j++)
    for (int k = 1; k < 4; k++)
      A[UU + j][U1 + k - 1] = dbsqdui[k] * q.ucon[0] * q.ucov[j] +
                              eta * (dutdui[k] * q.ucov[j] + q.ucon[0] * dudduu[j][k]) +
                              kdelta(j, 0) * 0.5 * dbsqdui[k] - (dbtdui[k] * q.bcov[j] + q.bcon[0] * dbdiduj[j][k]);
  double dgdvi[4], duidvj[4][4];
  const double gamma = gamma_of(pr, g);
  for (int j = 1; j < 4; j++) {
    dgdvi[j] = 0.0;
    for (int k = 1; k < 4; k++) dgdvi[j] += 1.0 / gamma * gcov_at(g, j, k) * pr[U1 + k - 1];
  }
  {
    const double alpha = 1.0 / sqrt(-g.gcon[0]);
    double betacon[4];
    for (int j = 1; j < 4; j++) betacon[j] = g.gcon[j] * alpha * alpha;
    for (int j = 1; j < 4; j++)
      for (int k = 1; k < 4; k++) duidvj[j][k] = kdelta(j, k) - betacon[j] / alpha * dgdvi[k];
  }
  for (int i = 0; i < 5; i++) {
    double t[3];
    for (int j = 1; j < 4; j++) {
      double s = 0.;
      for (int l = 1; l < 4; l++) s += A[RHO + i][U1 + l - 1] * duidvj[l][j];
      t[j - 1] = s;
    }
    for (int j = 0; j < 3; j++) A[i][U1 + j] = t[j];
  }
}

// LU_decompose + LU_substitution, utoprim_5d2_final.c:734-960 (Crout with
// implicit row scaling; no swap that would put a zero on the last
// diagonal; the forward substitution runs its sums downwards)
HD_INLINE void lu5_solve(double A[5][5], double* B)
{
  int permute[5] = {0, 0, 0, 0, 0};
  double row_norm[5];
  const int n = 5;
  bool singular = false;
  for (int i = 0; i < n; i++) {
    double absmax = 0.;
    for (int j = 0; j < n; j++) {
      const double maxtemp = fabs(A[i][j]);
      if (maxtemp > absmax) absmax = maxtemp;
    }
    if (absmax == 0.) {
      singular = true;
      break;
    }
    row_norm[i] = 1. / absmax;
  }
  if (!singular) {
    int max_row = 0;
    for (int j = 0; j < n; j++) {
      for (int i = 0; i < j; i++)
        for (int k = 0; k < i; k++) A[i][j] -= A[i][k] * A[k][j];
      double absmax = 0.0;
      for (int i = j; i < n; i++) {
        for (int k = 0; k < j; k++) A[i][j] -= A[i][k] * A[k][j];
        const double maxtemp = fabs(A[i][j]) * row_norm[i];
        if (maxtemp >= absmax) {
          absmax = maxtemp;
          max_row = i;
        }
      }
      if (max_row != j) {
        if ((j == (n - 2)) && (A[j][j + 1] == 0.)) {
          max_row = j;
        } else {
          for (int k = 0; k < n; k++) {
            const double t = A[j][k];
            A[j][k] = A[max_row][k];
            A[max_row][k] = t;
          }
          row_norm[max_row] = row_norm[j];
        }
      }
      permute[j] = max_row;
      if (A[j][j] == 0.) A[j][j] = 1e-30;
      if (j != (n - 1)) {
        const double maxtemp = 1. / A[j][j];
        for (int i = (j + 1); i < n; i++) A[i][j] *= maxtemp;
      }
    }
  }
  for (int i = 0; i < n; i++) {
    double tmpvar = B[permute[i]];
    B[permute[i]] = B[i];
    for (int j = (i - 1); j >= 0; j--) tmpvar -= A[i][j] * B[j];
    B[i] = tmpvar;
  }
  for (int i = (n - 1); i >= 0; i--) {
    for (int j = (i + 1); j < n; j++) B[i] -= A[i][j] * B[j];
    B[i] /= A[i][i];
  }
}

// func_5d2, utoprim_5d2_final.c:77-300 (NORMMETHOD 1, NEWINVERSION 1)
HD_INLINE void f5d2_func(const double* x, const double* Utarget, const Geo<double>& g, double gam, double* dxm,
                         double& f, double& df)
{
  double pr[NPR], Ucur[NPR], Am[5][5];
  for (int i = 0; i < B1; i++) pr[i] = x[i];
  for (int i = B1; i <= B3; i++) pr[i] = Utarget[i];
  State<double> q;
  state_of(pr, g, q);
  primtoU_nothing(pr, q, gam, Ucur);
  dudp_calc_g5(pr, q, g, gam, Am);
  double norm = 0.0;
  int nterms = 0;
  for (int j = 0; j < 5; j++)
    for (int k = 0; k < 5; k++)
      if (Am[j][k] > DBL_EPS_REF) {
        norm += fabs(Am[j][k]);
        nterms++;
      }
  norm = ((double)(nterms)) / (norm);
  for (int j = 0; j < 5; j++)
    for (int k = 0; k < 5; k++) Am[j][k] *= (norm);
  df = 0.;
  for (int k = 0; k < 5; k++) {
    const double resid = Ucur[k] - Utarget[k];
    dxm[k] = -resid * (norm);
    double residnorm = 0.5 * (fabs(Ucur[k]) + fabs(Utarget[k]));
    residnorm = (residnorm == 0.) ? 1. : 1. / residnorm;
    df -= residnorm * resid * resid;
  }
  f = -0.5 * (df);
  lu5_solve(Am, dxm);
}

// Utoprim_5d2_final with its general_newton_raphson (USE_LINE_SEARCH -2,
// NEWCONVERGE 1, errx from W of calc_errx_5d), utoprim_5d2_final.c:28-75,
// 352-372, 980-1300
HD_INLINE int utoprim_5d2(const double* Ug, const Geo<double>& g, double gam, double* prim)
{
  constexpr double TOL_RESID = 1.e-4;
  double Utarget[NPR], x[NPR];
  for (int k = 0; k < NPR; k++) Utarget[k] = Ug[k];
  for (int k = B1; k <= B3; k++) prim[k] = Utarget[k];
  for (int k = 0; k < NPR; k++) x[k] = prim[k];
  int ret;
  {
    double f = 1., df = 1., dx[5], errx = 1., W = 0., vsq = 0.;
    int n_iter = 0, i_extra = 0, doing_extra = 0;
    bool keep_iterating = true;
    while (keep_iterating) {
      f5d2_func(x, Utarget, g, gam, dx, f, df);
      errx = 0.;
      for (int id = 0; id < 5; id++) x[id] += dx[id];
      const double W_old = W;
      // calc_errx_5d
      vsq = 0.;
      for (int id = 1; id < 4; id++)
        for (int jd = 1; jd < 4; jd++) vsq += gcov_at(g, id, jd) * x[U1 + id - 1] * x[U1 + jd - 1];
      const double gsqtmp = 1. + vsq;
      vsq /= gsqtmp;
      W = gsqtmp * (gam * x[UU] + x[RHO]);
      errx = (W == 0.) ? fabs(W - W_old) : fabs((W - W_old) / W);
      if ((fabs(errx) <= N_NEWT_TOL) && (f <= TOL_RESID) && (doing_extra == 0) && (N_EXTRA_NEWT_ITER > 0))
        doing_extra = 1;
      if (doing_extra == 1) i_extra++;
      if (((fabs(errx) <= N_NEWT_TOL) && (doing_extra == 0)) || (i_extra > N_EXTRA_NEWT_ITER) ||
          (n_iter >= (N_MAX_NEWT_ITER - 1)))
        keep_iterating = false;
      n_iter++;
    }
    bool finite_all = isfinite(f) && isfinite(df);
    for (int id = 0; id < 5; id++) finite_all = finite_all && isfinite(x[id]);
    if (!finite_all) ret = 1;
    else if ((fabs(errx) > N_MIN_NEWT_TOL) || (f > TOL_RESID)) ret = 1;
    else ret = 0;
  }
  if (ret) return PF_CONV;
  // the negative-density codes are set and then overwritten with
  // UTOPRIMNOFAIL (utoprim_5d2_final.c:56-73); gamma_calc cannot fail
  for (int k = 0; k < NPR; k++) prim[k] = x[k];
  return PF_NOFAIL;
}

// UtoU(UEVOLVE -> UNOTHING), phys.c:219-237 (WITHGDET: every e[k] is
// sqrt(-g); the rest mass is added back to UU)
HD_INLINE void evolved_to_geomfree(const double* U, const Geo<double>& g, double* Ug)
{
  for (int k = 0; k < NPR; k++) Ug[k] = U[k] / g.g;
  Ug[UU] += -Ug[RHO];
}

// One method of Utoprimgen_pick (step_ch.c:583-600) other than the 2D:
// Ug geometry-free, pr the guess in and the result out; returns the pflag
// code.  The LDZ method is not part of the chain (step_ch.c:616 leaves it
// out) and returns UTOPRIMFAILCONV here.
HD_INLINE int pick(int which, const double* Ug, const Geo<double>& g, double gam, double gammafail, double* pr)
{
  switch (which) {
    case M_5D1: return utoprim_5d1(Ug, g, gam, pr);
    case M_1D: return utoprim_1d_family<false>(Ug, g, gam, gammafail, pr);
    case M_1DOPT: return utoprim_1d_family<true>(Ug, g, gam, gammafail, pr);
    case M_1DFINAL: return utoprim_final_family<false>(Ug, g, gam, gammafail, pr);
    case M_2DFINAL: return utoprim_final_family<true>(Ug, g, gam, gammafail, pr);
    case M_5D2: return utoprim_5d2(Ug, g, gam, pr);
    default: return PF_CONV;
  }
}

// Utoprimgen_tryagain + Utoprimgen_tryagain_substep, step_ch.c:608-640
// (STEPOVERNEGU 0): while the pflag is nonzero, restore the guess pr0 and
// run the next method.  Uev: the evolved U; pr, pfl: the primary 2D
// inversion's result and code on entry (the chain's second 2D attempt
// repeats them: the 2D inversion is deterministic), the chain's on return.
HD_INLINE int tryagain_chain(const double* Uev, const Geo<double>& g, double gam, double gammafail, const double* pr0,
                             double* pr, int pfl)
{
  if (pfl == 0) return 0;
  double Ug[NPR], pr2d[NPR];
  evolved_to_geomfree(Uev, g, Ug);
  for (int k = 0; k < NPR; k++) pr2d[k] = pr[k];
  const int pfl2d = pfl;
  const int order[7] = {M_5D1, M_2D, M_1D, M_1DOPT, M_1DFINAL, M_2DFINAL, M_5D2};
  for (int m = 0; m < 7; m++) {
    if (pfl == 0) break;
    if (order[m] == M_2D) {
      for (int k = 0; k < NPR; k++) pr[k] = pr2d[k];
      pfl = pfl2d;
      continue;
    }
    for (int k = 0; k < NPR; k++) pr[k] = pr0[k];
    pfl = pick(order[m], Ug, g, gam, gammafail, pr);
  }
  return pfl;
}

}  // namespace ta
}  // namespace harm
