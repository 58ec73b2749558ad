// Per-point GRMHD physics for the B200 step kernels.
//
// Each function restates one reference routine (file:line in the
// pseudotensor/harm_ramt tree) and keeps its floating-point evaluation order
// term by term; the FP64 build is compiled with --fmad=false so that the
// device rounds exactly as the reference's x86-64 FP64 build does.
//
// Geometry is carried per location as the 10 independent components of the
// symmetric g_{mu nu} and g^{mu nu} plus sqrt(-g).  Packed order:
//   00 01 02 03 11 12 13 22 23 33
#pragma once
#include <stdint.h>

namespace harm {

enum { RHO = 0, UU, U1, U2, U3, B1, B2, B3, NPR };
enum { FACE1 = 0, FACE2 = 1, CORN = 2, CENT = 3 };

// pflag codes, global.h:547-559
enum { PF_FIXED = -1, PF_NOFAIL = 0, PF_CONVUTSQ = 2, PF_CONVW = 3, PF_CONVUTSQ2 = 4, PF_RHONEG = 5,
       PF_UNEG = 6, PF_RHOUNEG = 7, PF_GAMMAPERC = 8, PF_UPERC = 9 };
// fatal fail codes, global.h:562-579
enum { FAIL_VCHAR_DISCR = 3, FAIL_COEFF_NEG = 4, FAIL_COEFF_SUP = 5, FAIL_UTCALC_DISCR = 6, FAIL_VSQ_NEG = 9 };
// Utoprim_ffde's space-like drift velocity (phys.ffde.c:281-284): the
// reference aborts the step through MYFUN without a FAIL_* number
constexpr int FAIL_FFDE_SPACELIKE = 20;

// host-and-device inline: the per-zone physics also compiles for the host,
// where the adjoint's building blocks are checked against finite differences
#define HD_INLINE __host__ __device__ __forceinline__

constexpr double DBL_EPS_REF = 2.2204460492503131e-16;  // global.h:710

__host__ __device__ constexpr int sym(int a, int b)
{
  // packed index of the symmetric pair (a,b)
  return (a <= b) ? (a == 0 ? b : (a == 1 ? 3 + b : (a == 2 ? 5 + b : 9)))
                  : (b == 0 ? a : (b == 1 ? 3 + a : (b == 2 ? 5 + a : 9)));
}

template <typename T>
struct Geo {
  T gcov[10];
  T gcon[10];
  T g;
};

template <typename T>
HD_INLINE T rmax(T a, T b) { return (a > b) ? a : b; }  // phys.c:1580
template <typename T>
HD_INLINE T rmin(T a, T b) { return (a > b) ? b : a; }  // phys.c:1587
template <typename T>
HD_INLINE T rsign(T a) { return (a > T(0.0)) ? T(1.0) : ((a < T(0.0)) ? T(-1.0) : T(0.0)); }

template <typename T>
struct State {
  T ucon[4], ucov[4], bcon[4], bcov[4];
};

// v[d], d in 0..3, by selects: a constant d folds to v[d]; a run-time d
// (one code path for both face directions) keeps v in registers
template <typename T>
HD_INLINE T pick4(const T* v, int d) { return (d == 3) ? v[3] : ((d == 2) ? v[2] : ((d == 1) ? v[1] : v[0])); }

// gamma_calc, phys.c:848-877
template <typename T>
HD_INLINE T gamma_of(const T* pr, const Geo<T>& g)
{
  const T* c = g.gcov;
  T qsq = c[4] * pr[U1] * pr[U1] + c[7] * pr[U2] * pr[U2] + c[9] * pr[U3] * pr[U3] +
          T(2.) * (c[5] * pr[U1] * pr[U2] + c[6] * pr[U1] * pr[U3] + c[8] * pr[U2] * pr[U3]);
  return sqrt(T(1.) + qsq);
}

// ucon_calc_rel4vel, phys.c:830-845
template <typename T>
HD_INLINE void ucon_of(const T* pr, const Geo<T>& g, T* ucon)
{
  T alpha = T(1.) / sqrt(-g.gcon[0]);
  T beta1 = g.gcon[1] * alpha * alpha;
  T beta2 = g.gcon[2] * alpha * alpha;
  T beta3 = g.gcon[3] * alpha * alpha;
  T gamma = gamma_of(pr, g);
  ucon[0] = gamma / alpha;
  ucon[1] = pr[U1] - gamma * beta1 / alpha;
  ucon[2] = pr[U2] - gamma * beta2 / alpha;
  ucon[3] = pr[U3] - gamma * beta3 / alpha;
}

// lower, phys.c:633
template <typename T>
HD_INLINE void lower_v(const T* v, const T* c, T* w)
{
  w[0] = c[0] * v[0] + c[1] * v[1] + c[2] * v[2] + c[3] * v[3];
  w[1] = c[1] * v[0] + c[4] * v[1] + c[5] * v[2] + c[6] * v[3];
  w[2] = c[2] * v[0] + c[5] * v[1] + c[7] * v[2] + c[8] * v[3];
  w[3] = c[3] * v[0] + c[6] * v[1] + c[8] * v[2] + c[9] * v[3];
}

template <typename T>
HD_INLINE T dot4(const T* a, const T* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }

// get_state + bcon_calc, phys.c:716-727 and 285-294
template <typename T>
HD_INLINE void state_of(const T* pr, const Geo<T>& g, State<T>& q)
{
  ucon_of(pr, g, q.ucon);
  lower_v(q.ucon, g.gcov, q.ucov);
  q.bcon[0] = pr[B1] * q.ucov[1] + pr[B2] * q.ucov[2] + pr[B3] * q.ucov[3];
#pragma unroll
  for (int j = 1; j <= 3; j++) q.bcon[j] = (pr[B1 - 1 + j] + q.bcon[0] * q.ucon[j]) / q.ucon[0];
  lower_v(q.bcon, g.gcov, q.bcov);
}

// mhd_calc_0, phys.c:381-406 (row `dir` of T^mu_nu)
template <typename T, bool FFDE>
HD_INLINE void mhd_row(const T* pr, int dir, const State<T>& q, T gam, T* mhd)
{
  T r, u, P, w;
  if (!FFDE) {
    r = pr[RHO];
    u = pr[UU];
    P = (gam - T(1.)) * u;
    w = P + r + u;
  } else {
    r = u = P = w = T(0.0);
  }
  T bsq = dot4(q.bcon, q.bcov);
  T eta = w + bsq;
  T ptot = P + bsq * T(0.5);
  const T ud = pick4(q.ucon, dir), bd = pick4(q.bcon, dir);
#pragma unroll
  for (int j = 0; j < 4; j++) mhd[j] = eta * ud * q.ucov[j] + ptot * ((dir == j) ? T(1.) : T(0.)) - bd * q.bcov[j];
}

// primtoflux(UEVOLVE), phys.c:16-56, massflux_calc 59, dualfullfaraday_calc
// (PRIMMAXWELL) 155-185, UtoU(UNOTHING->UEVOLVE) 219-265
template <typename T, bool FFDE>
HD_INLINE void flux_of(const T* pr, const State<T>& q, int dir, const Geo<T>& g, T gam, T* F)
{
  T fin[NPR];
  const T ud = pick4(q.ucon, dir);
  fin[RHO] = pr[RHO] * ud;
  mhd_row<T, FFDE>(pr, dir, q, gam, &fin[UU]);
  if (dir > 0) {
    const T bd = pick4(&pr[B1 - 1], dir);  // B^dir
    fin[B1] = (pr[B1] * ud - bd * q.ucon[1]) / q.ucon[0];
    fin[B2] = (pr[B2] * ud - bd * q.ucon[2]) / q.ucon[0];
    fin[B3] = (pr[B3] * ud - bd * q.ucon[3]) / q.ucon[0];
  } else {
    fin[B1] = pr[B1];
    fin[B2] = pr[B2];
    fin[B3] = pr[B3];
  }
  if (!FFDE) fin[UU] += fin[RHO];
#pragma unroll
  for (int k = 0; k < NPR; k++) F[k] = fin[k] * g.g;
}

// vchar + simplefast, vchar.c:37-135 and 166-234.  The raised unit covectors
// reduce to metric columns, so the dot products are the metric entries the
// reference's zero-padded sums produce.  Returns a fail code.
template <typename T>
HD_INLINE int vchar_of(const T* pr, const State<T>& q, int dir, const Geo<T>& g, T gam, T& vmax, T& vmin)
{
  // NUMEPSILON*100 of the reference's FTYPE (global.h:706-727): DBL_EPSILON
  // for FP64, FLT_EPSILON for the FP32 faces of the mixed form
  const T eps100 = (sizeof(T) == 8) ? T(DBL_EPS_REF * 100.0) : T(1.19209290e-07 * 100.0);
  T bsq = dot4(q.bcon, q.bcov);
  T rho = pr[RHO], u = pr[UU];
  T WW = rho + gam * u, cs2, EF, va2;
  if (WW > T(0.0)) cs2 = gam * (gam - T(1.)) * u / WW;
  else WW = cs2 = T(0.0);
  EF = bsq + WW;
  if (EF > T(0.0)) va2 = bsq / EF;
  else EF = va2 = T(0.0);
  T cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < T(0.0)) {
    if (cms2 / (cs2 + va2) > -eps100) cms2 = T(0.0);
    else return FAIL_COEFF_NEG;
  }
  if (cms2 > T(1.)) {
    if (cms2 < T(1.0) + eps100) cms2 = T(1.0);
    else return FAIL_COEFF_SUP;
  }
  // Acon = g^{mu dir}, Bcon = g^{mu t}
  T Acon[4], Bcon[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const T col[4] = {g.gcon[sym(m, 0)], g.gcon[sym(m, 1)], g.gcon[sym(m, 2)], g.gcon[sym(m, 3)]};
    Acon[m] = pick4(col, dir);
    Bcon[m] = g.gcon[sym(m, 0)];
  }
  // dot(Acon,Acov) etc. with unit covectors: zero terms added exactly as the
  // reference does (x*0 contributes a signed zero that cannot change a sum)
  T Asq = Acon[0] * T(dir == 0) + Acon[1] * T(dir == 1) + Acon[2] * T(dir == 2) + Acon[3] * T(dir == 3);
  T Bsq = Bcon[0] * T(1.) + Bcon[1] * T(0.) + Bcon[2] * T(0.) + Bcon[3] * T(0.);
  T Au = T(dir == 0) * q.ucon[0] + T(dir == 1) * q.ucon[1] + T(dir == 2) * q.ucon[2] + T(dir == 3) * q.ucon[3];
  T Bu = T(1.) * q.ucon[0] + T(0.) * q.ucon[1] + T(0.) * q.ucon[2] + T(0.) * q.ucon[3];
  T AB = Acon[0] * T(1.) + Acon[1] * T(0.) + Acon[2] * T(0.) + Acon[3] * T(0.);
  T Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  T A = Bu2 - (Bsq + Bu2) * cms2;
  T B = T(2.) * (AuBu - (AB + AuBu) * cms2);
  T C = Au2 - (Asq + Au2) * cms2;
  T discr = B * B - T(4.) * A * C;
  // the reference's absolute -1e-10 round-off allowance (vchar.c:203); FP32
  // faces (mixed form) allow round-off relative to the terms, 100 FLT_EPSILON
  const T dtol = (sizeof(T) == 8) ? T(1E-10)
                                  : fmax(T(1E-10), T(1.19209290e-07 * 100.0) * (B * B + fabs(T(4.) * A * C)));
  if ((discr < T(0.0)) && (discr > -dtol)) discr = T(0.0);
  else if (discr < -dtol) return FAIL_VCHAR_DISCR;
  discr = sqrt(discr);
  T vm = -(-B + discr) / (T(2.) * A);
  T vp = -(-B - discr) / (T(2.) * A);
  if (vp < vm) {
    vmax = vm;
    vmin = vp;
  } else {
    vmax = vp;
    vmin = vm;
  }
  return 0;
}

// limit_gamma, fixup.c:1298-1354.  Returns a fail code.
template <typename T>
HD_INLINE int limit_gamma(T gammamax, T* pr, const Geo<T>& g)
{
  if (gammamax <= T(1.0)) return 0;
  T gamma = gamma_of(pr, g);
  if (gamma > gammamax && gamma != T(1.0)) {
    T pref = (gammamax * gammamax - T(1.)) / (gamma * gamma - T(1.));
    if (pref < T(0.0)) return FAIL_UTCALC_DISCR;
    T f = sqrt(pref);
    pr[U1] *= f;
    pr[U2] *= f;
    pr[U3] *= f;
  }
  return 0;
}

// MC slope, interp.c:106-118 with MINMOD, interp.h:13-14
template <typename T>
HD_INLINE T minmod(T a, T b) { return (a * b <= T(0)) ? T(0.0) : ((fabs(a) < fabs(b)) ? a : b); }
template <typename T>
HD_INLINE T mc_slope(T yl, T yc, T yr)
{
  T Dqm = T(2.0) * (yc - yl);
  T Dqp = T(2.0) * (yr - yc);
  T Dqc = T(0.5) * (yr - yl);
  return minmod(Dqc, minmod(Dqm, Dqp));
}

// para4 with the MC sub-limiter, interp.c:444-538, in its three parts.  A
// zone's two raw interface values and the slopes they use are functions of
// the values they sit between, the same whichever zone's para4 evaluates
// them (the reference's operand order kept), so neighbouring zones may
// share them; the limiting is the zone's own.
// the MC-limited slope at y0 between ym and yp (the loop body)
template <typename T>
HD_INLINE T para_dq(T ym, T y0, T yp)
{
  T Dqm = T(2.0) * (y0 - ym);
  T Dqp = T(2.0) * (yp - y0);
  T Dqc = T(0.5) * (yp - ym);
  T aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
  T s = Dqm * Dqp;
  return (s <= T(0.)) ? T(0.) : rmin(aDqc, rmin(aDqm, aDqp)) * rsign(Dqc);
}
// the raw interface value between a lower zone (value ylo, slope dlo) and
// an upper one (yhi, dhi)
template <typename T>
HD_INLINE T para_face(T ylo, T yhi, T dlo, T dhi)
{
  return T(0.5) * (yhi + ylo) - (dhi - dlo) / T(8.0);
}
// the zone value y's limited left and right states from its raw interface
// values l (lower side, toward ym) and r (upper side, toward yp)
template <typename T>
HD_INLINE void para_limit(T ym, T y, T yp, T l, T r, T& lout, T& rout)
{
  l = rmax(rmin(y, ym), l);
  l = rmin(rmax(y, ym), l);
  r = rmax(rmin(y, yp), r);
  r = rmin(rmax(y, yp), r);
  T qa = (r - y) * (y - l);
  T qd = (r - l);
  T qe = T(8.0) * (y - T(0.5) * (l + r));
  if (qa <= T(0.)) {
    l = y;
    r = y;
  } else {
    if (qd * (qd - qe) < T(0.0)) l = T(3.0) * y - T(2.0) * r;
    if (qd * (qd + qe) < T(0.0)) r = T(3.0) * y - T(2.0) * l;
  }
  lout = l;
  rout = r;
}
template <typename T>
HD_INLINE void para4(T y0, T y1, T y2, T y3, T y4, T& lout, T& rout)
{
  const T d1 = para_dq(y0, y1, y2), d2 = para_dq(y1, y2, y3), d3 = para_dq(y2, y3, y4);
  para_limit(y1, y2, y3, para_face(y1, y2, d1, d2), para_face(y2, y3, d2, d3), lout, rout);
}

// Deterministic Newton cycle-break factor in [0,1): splitmix64 finaliser
// (Steele, Lea & Flood 2014) of the iterate's bits and the iteration count.
// Replaces rand()/RAND_MAX at utoprim_2d.c:669 (a serial global RNG stream).
HD_INLINE uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double cycle_break_uniform(double x0, double x1, int n_iter)
{
  uint64_t a = (uint64_t)__double_as_longlong(x0), b = (uint64_t)__double_as_longlong(x1);
  uint64_t h = mix64(a ^ mix64(b ^ (uint64_t)(uint32_t)n_iter));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------------------
// 2D Noble et al. con-to-prim, utoprim_2d.c (always FP64)
struct U2PCtx {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, wglobal, gam;
};

// utsq_calc, utoprim_2d.c:318-338
HD_INLINE double utsq_calc(const U2PCtx& c, double W)
{
  double Wsq = W * W, W4 = Wsq * Wsq;
  return (c.Bsq * c.QdotBsq + W * (2. * c.QdotBsq + c.Qtsq * W)) /
         (W4 + 2. * c.Bsq * Wsq * W + Wsq * (c.Bsq * c.Bsq - c.Qtsq) - c.QdotBsq * (2. * W + c.Bsq));
}

// func_vsq Newton step, utoprim_2d.c:748-798
HD_INLINE void func_vsq(const U2PCtx& c, double W, double vsq, double& dx0, double& dx1)
{
  const double Bsq = c.Bsq, QdotBsq = c.QdotBsq, Qtsq = c.Qtsq, Qdotn = c.Qdotn, D = c.D, gam = c.gam;
  double Wsq = W * W;
  double gtmp = 1. - vsq;
  double p_tmp = (gam - 1.) * (W * gtmp - D * sqrt(gtmp)) / gam;
  double dPdW = (gam - 1.) * (1. - vsq) / gam;
  double dPdvsq = (gam - 1.) * (0.5 * D / sqrt(1. - vsq) - W) / gam;
  double BW = Bsq + W;
  double t2 = (Qtsq - vsq * (BW * BW) + (QdotBsq * (Bsq + 2 * W)) / Wsq);
  double t3 = (Qdotn - (Bsq * (1 + vsq)) / 2. + QdotBsq / (2. * Wsq) - W + p_tmp);
  double QW3 = QdotBsq / (Wsq * W);
  dx0 = (-Bsq / 2. + dPdvsq) * t2 + (BW * BW) * t3;
  dx1 = -((-1 + dPdW - QW3) * t2) - 2 * (vsq + QW3) * BW * t3;
  double detJ = BW * ((-1 + dPdW - QW3) * BW + ((Bsq - 2 * dPdvsq) * (QdotBsq + vsq * (Wsq * W))) / (Wsq * W));
  dx0 /= -(detJ);
  dx1 /= -(detJ);
}

// general_newton_raphson + validate_x(vartype 3), utoprim_2d.c:606-740, 556-600
// Returns 0/1 as the reference does, or NEWTON_DEFERRED when `maxit` (< 200)
// iterations ran without convergence.  The loop's whole state is then saved
// to st[0], st[ss], ... st[4 ss] (x0, x1, errx, errx_old, iteration count)
// when st is given, and a later call with `resume` set continues from it up
// to the full 200: the iteration sequence is deterministic, so the split
// solve reaches the reference's result with no iteration repeated.
constexpr int NEWTON_DEFERRED = -7;
constexpr int NEWTON_STATE = 5;
__device__ __forceinline__ int newton_vsq(const U2PCtx& c, double& x0, double& x1, double gammafail, int& niter_out,
                                          int maxit, double* st, long long ss, bool resume)
{
  constexpr int MAX_NEWT_ITER = 200;
  constexpr double NEWT_TOL = 1.0e-15, MIN_NEWT_TOL = 1.0e-10, W_TOO_BIG = 1.e9;
  const double vsq_too_big = (1.0 - 1.0 / (gammafail - 1.0));
  double errx = 1., errx_old = 2., errx_oldest;
  int n_iter = 0;
  if (resume) {
    x0 = st[0];
    x1 = st[ss];
    errx = st[2 * ss];
    errx_old = st[3 * ss];
    n_iter = (int)st[4 * ss];
  }
  while ((errx > NEWT_TOL) && (n_iter < maxit)) {
    double dx0, dx1;
    func_vsq(c, x0, x1, dx0, dx1);
    if (((n_iter + 1) % 10) == 0) {
      double r = cycle_break_uniform(x0, x1, n_iter);
      dx0 *= r;
      dx1 *= r;
    }
    errx_oldest = errx_old;
    errx_old = errx;
    errx = 0.;
    double xo0 = x0;
    x0 += dx0 * 1.0;
    errx += (x0 == 0.) ? fabs(dx0) : fabs(dx0 / x0);
    x1 += dx1 * 1.0;
    errx += (x1 == 0.) ? fabs(dx1) : fabs(dx1 / x1);
    errx /= 1. * 2;
    x0 = fabs(x0);
    x0 = (x0 / c.wglobal > W_TOO_BIG) ? xo0 : x0;
    x1 = (x1 < 0.) ? 0.0 : x1;
    x1 = (x1 > 1.) ? vsq_too_big : x1;
    if (((errx_old == errx) || (errx_oldest == errx)) && (errx < MIN_NEWT_TOL)) errx = -errx;
    n_iter++;
  }
  niter_out = n_iter;
  if (maxit < MAX_NEWT_ITER && n_iter >= maxit && errx > NEWT_TOL) {
    if (st) {
      st[0] = x0;
      st[ss] = x1;
      st[2 * ss] = errx;
      st[3 * ss] = errx_old;
      st[4 * ss] = (double)n_iter;
    }
    return NEWTON_DEFERRED;
  }
  if (n_iter >= MAX_NEWT_ITER) return (errx > MIN_NEWT_TOL) ? 1 : 0;
  return 0;
}

// ucon_calc_3vel, phys.c:885-957: u^mu from v^i = u^i/u^t (packed gcov);
// nonzero when the velocity is not time-like
HD_INLINE int ucon_3vel(const double* v, const double* c, double* ucon)
{
  const double discr = +c[0] + c[4] * v[1] * v[1] + c[7] * v[2] * v[2] + c[9] * v[3] * v[3] +
                       2. * (c[1] * v[1] + c[2] * v[2] + c[3] * v[3] + c[5] * v[1] * v[2] + c[6] * v[1] * v[3] +
                             c[8] * v[2] * v[3]);
  if (discr > 0.) return 1;
  ucon[0] = 1. / sqrt(-discr);
#pragma unroll
  for (int j = 1; j < 4; j++) ucon[j] = v[j] * ucon[0];
  return 0;
}

// Utoprimgen(UEVOLVE) for EOMFFDE, step_ch.c:544-546: UtoU without the
// rest-mass term (phys.c:228-233) -> Utoprim_ffde, phys.ffde.c:141-372
// (CHECKBSQMINUSESQ 1, AVOIDUTINF 2): B^i/alpha and B_i/alpha (U2BBsq,
// 1261-1284), E^i/alpha from B_j x T^t_k (TtoEconOalpha, 1287-1318), the
// B^2 - E^2 > 0 cap on the drift Lorentz factor, v^i (EBcovtovcon,
// 551-560), u^i through ucon_calc_3vel (vcon2pr's active branch,
// transforms.c:372-377, stores u^i).  pr[RHO], pr[UU] keep the guess.
// Returns 0 or FAIL_FFDE_SPACELIKE.  utoprim_ffde_geomfree takes U in the
// geometry-free form (T^t_mu, B^i), as filterffde (phys.ffde.c:1957-1980)
// passes it; utoprim_ffde the evolved form (times sqrt(-g)).
HD_INLINE int utoprim_ffde_geomfree(const double* U, const Geo<double>& g, double* pr, double gammamax)
{
  const double alphasq = 1. / (-g.gcon[0]);
  double Bcon[4] = {0.0, U[B1], U[B2], U[B3]}, Bcov[4];
  lower_v(Bcon, g.gcov, Bcov);
  double Bsq = 0.0;
#pragma unroll
  for (int j = 1; j < 4; j++) Bsq += Bcov[j] * Bcon[j];
  double o = 1.0 / (Bsq * g.g);
  double Econ[4], Ecov[4];
  Econ[0] = 0;
  Econ[1] = (Bcov[2] * U[U3] - Bcov[3] * U[U2]) * (o);
  Econ[2] = (Bcov[3] * U[U1] - Bcov[1] * U[U3]) * (o);
  Econ[3] = (Bcov[1] * U[U2] - Bcov[2] * U[U1]) * (o);
  double realBsq = Bsq;
  lower_v(Econ, g.gcov, Ecov);
  double Esq = 0.0;
#pragma unroll
  for (int j = 1; j < 4; j++) Esq += Econ[j] * Ecov[j];
  const double BsqmEsq = Bsq - Esq;
  const double gammasq = Bsq / BsqmEsq;
  if ((gammasq > gammamax * gammamax) || (gammasq < 1.0)) {
    const double Gsq = 1.0 - 1.0 / (gammamax * gammamax);
    realBsq = (sqrt(Esq * Bsq / Gsq));
  }
  o = 1.0 / (realBsq * g.g);
  double vcon[4];
  vcon[0] = 0.;
  vcon[1] = alphasq * (-g.gcon[1] + (Ecov[2] * Bcov[3] - Ecov[3] * Bcov[2]) * o);
  vcon[2] = alphasq * (-g.gcon[2] + (Ecov[3] * Bcov[1] - Ecov[1] * Bcov[3]) * o);
  vcon[3] = alphasq * (-g.gcon[3] + (Ecov[1] * Bcov[2] - Ecov[2] * Bcov[1]) * o);
  double ucon[4];
  if (ucon_3vel(vcon, g.gcov, ucon)) return FAIL_FFDE_SPACELIKE;
  pr[U1] = ucon[1];
  pr[U2] = ucon[2];
  pr[U3] = ucon[3];
  pr[B1] = U[B1];
  pr[B2] = U[B2];
  pr[B3] = U[B3];
  return 0;
}

HD_INLINE int utoprim_ffde(const double* Uin, const Geo<double>& g, double* pr, double gammamax)
{
  double U[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) U[k] = Uin[k] / g.g;
  return utoprim_ffde_geomfree(U, g, pr, gammamax);
}

// lower_g / raise_g of utoprim_2d.c:365-392: sums started from 0.
HD_INLINE void lower_g(const double* v, const double* c, double* w)
{
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += c[sym(i, j)] * v[j];
    w[i] = s;
  }
}

// Utoprimgen(UEVOLVE) -> UtoU -> Utoprim_2d -> Utoprim_new_body:
// step_ch.c:468-552, phys.c:219-265, utoprim_2d.c:25-310.  U is the evolved
// conserved vector (with sqrt(-g)); pr holds the guess on entry.  Returns
// the pflag code; *niter gets the Newton iteration count.  nst, nss, resume:
// the Newton state of a deferred solve (newton_vsq), or null.
__device__ __forceinline__ int utoprim_2d(const double* U, const Geo<double>& g, double* pr, double gam, double gammafail,
                                          int* niter, int maxit = 200, double* nst = nullptr, long long nss = 0,
                                          bool resume = false)
{
  constexpr double W_TOO_BIG = 1.e9, FAIL_VAL = 1.e30;
  double Ug[NPR], Ut[NPR], pt[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) Ug[k] = U[k] / g.g;
  Ug[UU] += -Ug[RHO];
  const double alpha = 1.0 / sqrt(-g.gcon[0]);
  Ut[RHO] = Ug[RHO] * alpha;
#pragma unroll
  for (int k = UU; k <= U3; k++) Ut[k] = -alpha * Ug[k];
#pragma unroll
  for (int k = B1; k <= B3; k++) Ut[k] = alpha * Ug[k];
#pragma unroll
  for (int k = 0; k < B1; k++) pt[k] = pr[k];
  // body
  *niter = 0;
  int pfl = 0;
  {
    const double utsq_too_big = ((gammafail - 1.0) * (gammafail - 1.0));
    U2PCtx c;
    c.gam = gam;
    double Bcon[4] = {0., Ut[B1], Ut[B2], Ut[B3]}, Bcov[4], Qcov[4] = {Ut[UU], Ut[U1], Ut[U2], Ut[U3]}, Qcon[4];
    lower_g(Bcon, g.gcov, Bcov);
    lower_g(Qcov, g.gcon, Qcon);
    c.Bsq = 0.;
#pragma unroll
    for (int i = 1; i < 4; i++) c.Bsq += Bcon[i] * Bcov[i];
    double QdotB = 0.;
#pragma unroll
    for (int i = 0; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
    c.QdotBsq = QdotB * QdotB;
    const double lapse = sqrt(-1. / g.gcon[0]);
    double ncov[4] = {-lapse, 0., 0., 0.}, ncon[4];
    lower_g(ncov, g.gcon, ncon);
    c.Qdotn = Qcon[0] * ncov[0];
    double Qsq = 0.;
#pragma unroll
    for (int i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
    c.Qtsq = Qsq + c.Qdotn * c.Qdotn;
    c.D = Ut[RHO];
    double utsq = 0.;
#pragma unroll
    for (int i = 1; i < 4; i++)
#pragma unroll
      for (int j = 1; j < 4; j++) utsq += g.gcov[sym(i, j)] * pt[U1 + i - 1] * pt[U1 + j - 1];
    if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
    if (utsq < 0. || utsq > utsq_too_big) {
      pfl = PF_CONVUTSQ;
    } else {
      double rho0 = pt[RHO], u = pt[UU];
      double p = (gam - 1.) * u;
      double w = rho0 + u + p;
      double W = w * (1. + utsq);
      c.wglobal = w;
      double x0 = fabs(W), ut = fabs(utsq_calc(c, W));
      double x1 = (ut > 0.) ? (ut / (ut + 1.)) : 0.0;
      int ret = newton_vsq(c, x0, x1, gammafail, *niter, maxit, nst, nss, resume);
      if (ret == NEWTON_DEFERRED) return NEWTON_DEFERRED;
      if (ret != 0) {
        pfl = ret * 100 + 1;
      } else if ((W = x0) == FAIL_VAL) {
        pfl = 1;
      } else if ((W / c.wglobal <= 0.) || (W / c.wglobal > W_TOO_BIG)) {
        pfl = PF_CONVW;
      } else {
        utsq = utsq_calc(c, W);
        if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
        if (utsq < 0. || utsq > utsq_too_big) {
          pfl = PF_CONVUTSQ2;
        } else {
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
          pt[RHO] = rho0;
          pt[UU] = u;
#pragma unroll
          for (int i = 1; i < 4; i++) {
            double Qt = Qcon[i] + ncon[i] * c.Qdotn;
            pt[U1 + i - 1] = -gamma * Qt / (W + c.Bsq) - gamma * QdotB * Bcon[i] / (W * (W + c.Bsq));
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < B1; k++) pr[k] = pt[k];
  // B: the body stores U's field (alpha*B), which Utoprim_2d divides back
#pragma unroll
  for (int k = B1; k <= B3; k++) pr[k] = Ut[k] / alpha;
  return pfl;
}

}  // namespace harm
