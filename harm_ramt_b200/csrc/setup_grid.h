// Grid geometry of the host-side problem set-ups (setup_torus.cpp,
// setup_dipole.cu): the reference's coord.c / metric.c / set_grid.c for the
// two coordinate systems the problems use, restated with the reference's
// evaluation order so that the tables agree with its own bit for bit.
//   torus:  MKS defcoord 0 on Kerr-Schild (KSCOORDS)
//   dipole: defcoord 6 (log r, uniform theta) on flat space in spherical
//           polar coordinates (SPCMINKMETRIC)
// Set-up code, run once on the host; the step never calls it.
#pragma once
#include <math.h>
#include <string.h>

namespace harm_setup {

constexpr int NG = 3;
constexpr int FACE1 = 0, FACE2 = 1, CORN = 2, CENT = 3;
enum { RHO = 0, UU, U1, U2, U3, B1, B2, B3 };
enum { METRIC_KS = 0, METRIC_SPCMINK = 1 };

struct Coords {
  int defcoord = 0;          // 0: MKS (hslope), 6: log r and uniform theta
  int metric = METRIC_KS;    // the MCOORD of the problem
  double a = 0, R0 = 0, Rin = 0, Rout = 0, hslope = 0, startx1 = 0, startx2 = 0, dx1 = 0, dx2 = 0;
};

// coord(), coord.c:920-938
inline void coord_of(const Coords& c, int i, int j, int loc, double* X)
{
  if (loc == FACE1) {
    X[1] = c.startx1 + (i + 0) * c.dx1;
    X[2] = c.startx2 + ((j + 0) + 0.5) * c.dx2;
  } else if (loc == FACE2) {
    X[1] = c.startx1 + ((i + 0) + 0.5) * c.dx1;
    X[2] = c.startx2 + (j + 0) * c.dx2;
  } else if (loc == CENT) {
    X[1] = c.startx1 + ((i + 0) + 0.5) * c.dx1;
    X[2] = c.startx2 + ((j + 0) + 0.5) * c.dx2;
  } else {
    X[1] = c.startx1 + (i + 0) * c.dx1;
    X[2] = c.startx2 + (j + 0) * c.dx2;
  }
  X[0] = X[3] = 0.0;
}

// bl_coord for defcoord 0 and 6 with COORDSINGFIX (SINGSMALL 1e-20),
// coord.c:334-453
inline void bl_of(const Coords& c, const double* X, double* r, double* th)
{
  *r = c.R0 + exp(X[1]);
  if (c.defcoord == 6) *th = M_PI * X[2];
  else *th = M_PI * X[2] + ((1. - c.hslope) / 2.) * sin(2. * M_PI * X[2]);
  if (fabs(*th) < 1E-20) {
    if (*th >= 0) *th = 1E-20;
    if (*th < 0) *th = -1E-20;
  }
}

// dxdxp_analytic for defcoord 0 and 6 (both diagonal), coord.c:480-491, 534-536
inline void dxdxp_of(const Coords& c, const double* X, double r, double d[4])
{
  d[0] = 1.0;
  d[1] = r - c.R0;
  d[2] = (c.defcoord == 6) ? M_PI : M_PI + (1. - c.hslope) * M_PI * cos(2. * M_PI * X[2]);
  d[3] = 1.0;
}

// set_gcov_ksmetric (metric.c:540-597) or set_gcov_spcminkmetric
// (metric.c:511-535), then gcov2gcovprim (metric.c:1057-1083) with the
// diagonal Jacobian: g'_{jk} = sum_lm g_{lm} d_{lj} d_{mk}
inline void gcov_prim(const Coords& c, const double* X, double g[4][4])
{
  double r, th;
  bl_of(c, X, &r, &th);
  double m[4][4];
  if (c.metric == METRIC_SPCMINK) {
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) m[j][k] = 0.0;
    m[0][0] = -1.0;
    m[1][1] = 1.0;
    m[2][2] = r * r;
    m[3][3] = (r * sin(th)) * (r * sin(th));
  } else {
    const double a = c.a;
    const double cth = cos(th), sth = sin(th), s2 = sth * sth;
    const double rho2 = r * r + a * a * cth * cth;
    m[0][0] = (-1. + 2. * r / rho2);
    m[0][1] = (2. * r / rho2);
    m[0][2] = (0);
    m[0][3] = (-2. * a * r * s2 / rho2);
    m[1][0] = m[0][1];
    m[1][1] = (1. + 2. * r / rho2);
    m[1][2] = (0);
    m[1][3] = (-a * s2 * (1. + 2. * r / rho2));
    m[2][0] = (0);
    m[2][1] = (0);
    m[2][2] = (rho2);
    m[2][3] = (0);
    m[3][0] = m[0][3];
    m[3][1] = m[1][3];
    m[3][2] = (0);
    m[3][3] = (s2 * (rho2 + a * a * s2 * (1. + 2. * r / rho2)));
  }
  double d[4];
  dxdxp_of(c, X, r, d);
  double dm[4][4] = {{0}};
  for (int k = 0; k < 4; k++) dm[k][k] = d[k];
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) {
      double t = 0.;
      for (int l = 0; l < 4; l++)
        for (int q = 0; q < 4; q++) t += m[l][q] * dm[l][j] * dm[q][k];
      g[j][k] = t;
    }
}

// Gauss-Jordan elimination with full pivoting (the published Numerical
// Recipes gaussj that matrix_inverse, metric.c:1146-1162, calls on the
// metric): a[4][4] is replaced by its inverse.  Returns 1 if singular.
inline int gauss_jordan_inverse(double a[4][4])
{
  constexpr int n = 4;
  int indxc[n], indxr[n], ipiv[n] = {0, 0, 0, 0};
  int irow = 0, icol = 0;
  for (int i = 0; i < n; i++) {
    double big = 0.0;
    for (int j = 0; j < n; j++)
      if (ipiv[j] != 1)
        for (int k = 0; k < n; k++) {
          if (ipiv[k] == 0) {
            if (fabs(a[j][k]) >= big) {
              big = fabs(a[j][k]);
              irow = j;
              icol = k;
            }
          } else if (ipiv[k] > 1) {
            return 1;
          }
        }
    ++ipiv[icol];
    if (irow != icol)
      for (int l = 0; l < n; l++) {
        const double t = a[irow][l];
        a[irow][l] = a[icol][l];
        a[icol][l] = t;
      }
    indxr[i] = irow;
    indxc[i] = icol;
    if (a[icol][icol] == 0.0) return 1;
    const double pivinv = 1.0 / a[icol][icol];
    a[icol][icol] = 1.0;
    for (int l = 0; l < n; l++) a[icol][l] *= pivinv;
    for (int ll = 0; ll < n; ll++)
      if (ll != icol) {
        const double dum = a[ll][icol];
        a[ll][icol] = 0.0;
        for (int l = 0; l < n; l++) a[ll][l] -= a[icol][l] * dum;
      }
  }
  for (int l = n - 1; l >= 0; l--)
    if (indxr[l] != indxc[l])
      for (int k = 0; k < n; k++) {
        const double t = a[k][indxr[l]];
        a[k][indxr[l]] = a[k][indxc[l]];
        a[k][indxc[l]] = t;
      }
  return 0;
}

// gcon_func (metric.c:74-130): set_gcon_ksmetric (metric.c:666-722) then
// gcon2gconprim (metric.c:1085-1106) for Kerr-Schild -- the inverse
// Jacobian of a diagonal matrix is its reciprocal diagonal, which the
// reference's Gauss-Jordan produces exactly (pivot 1/d_kk); for the flat
// spherical metric the prime gcov inverted numerically (matrix_inverse).
inline int gcon_prim(const Coords& c, const double* X, double g[4][4])
{
  if (c.metric == METRIC_SPCMINK) {
    gcov_prim(c, X, g);
    return gauss_jordan_inverse(g);
  }
  double r, th;
  bl_of(c, X, &r, &th);
  const double a = c.a;
  const double cth = cos(th), sth = sin(th), s2 = sth * sth;
  const double rho2 = r * r + a * a * cth * cth;
  double ks[4][4];
  ks[0][0] = (-(1. + 2. * r / rho2));
  ks[0][1] = (2. * r / rho2);
  ks[0][2] = (0);
  ks[0][3] = (0);
  ks[1][0] = ks[0][1];
  ks[1][1] = ((r * (r - 2.) + a * a) / rho2);
  ks[1][2] = (0);
  ks[1][3] = (a / rho2);
  ks[2][0] = ks[0][2];
  ks[2][1] = ks[1][2];
  ks[2][2] = (1. / rho2);
  ks[2][3] = (0);
  ks[3][0] = ks[0][3];
  ks[3][1] = ks[1][3];
  ks[3][2] = ks[2][3];
  ks[3][3] = (1. / (rho2 * s2));
  double d[4];
  dxdxp_of(c, X, r, d);
  double id[4][4] = {{0}};
  for (int k = 0; k < 4; k++) id[k][k] = 1.0 / d[k];
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) {
      double t = 0.;
      for (int l = 0; l < 4; l++)
        for (int m = 0; m < 4; m++) t += id[j][l] * id[k][m] * ks[l][m];
      g[j][k] = t;
    }
  return 0;
}

// gdet_func, metric.c:1109-1140: LU decomposition with implicit partial
// pivoting (the Numerical Recipes ludcmp of ludcmp.c), det = d * prod(diag)
inline double gdet_of(const double gin[4][4])
{
  double a[5][5], vv[5], d = 1.0;
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) a[j + 1][k + 1] = gin[j][k];
  const int n = 4;
  int imax = 0;
  for (int i = 1; i <= n; i++) {
    double big = 0.0, temp;
    for (int j = 1; j <= n; j++)
      if ((temp = fabs(a[i][j])) > big) big = temp;
    if (big == 0.0) return NAN;
    vv[i] = 1.0 / big;
  }
  for (int j = 1; j <= n; j++) {
    for (int i = 1; i < j; i++) {
      double sum = a[i][j];
      for (int k = 1; k < i; k++) sum -= a[i][k] * a[k][j];
      a[i][j] = sum;
    }
    double big = 0.0, dum;
    for (int i = j; i <= n; i++) {
      double sum = a[i][j];
      for (int k = 1; k < j; k++) sum -= a[i][k] * a[k][j];
      a[i][j] = sum;
      if ((dum = vv[i] * fabs(sum)) >= big) {
        big = dum;
        imax = i;
      }
    }
    if (j != imax) {
      for (int k = 1; k <= n; k++) {
        dum = a[imax][k];
        a[imax][k] = a[j][k];
        a[j][k] = dum;
      }
      d = -d;
      vv[imax] = vv[j];
    }
    if (a[j][j] == 0.0) a[j][j] = 1.0e-30;
    if (j != n) {
      dum = 1.0 / (a[j][j]);
      for (int i = j + 1; i <= n; i++) a[i][j] *= dum;
    }
  }
  for (int j = 1; j <= n; j++) d *= a[j][j];
  return (d >= 0) ? NAN : sqrt(-d);
}

// conn_func_numerical1 with GAMMIEDERIVATIVE and CONNDELTA 1e-5,
// metric.c:1188-1262: centred differences of g'_{mu nu}, lowered Christoffel
// symbols, then raised with g'^{mu nu} at CENT.  conn[k][l][j] = Gamma^k_{lj}.
inline void conn_of(const Coords& c, const double* X, const double gcon[4][4], double conn[4][4][4])
{
  const double DELTA = 1E-5;
  double dg[4][4][4], tmp[4][4][4];
  for (int k = 0; k < 4; k++) {
    double Xh[4], Xl[4], gh[4][4], gl[4][4];
    for (int l = 0; l < 4; l++) Xh[l] = Xl[l] = X[l];
    Xh[k] += DELTA;
    Xl[k] -= DELTA;
    gcov_prim(c, Xh, gh);
    gcov_prim(c, Xl, gl);
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) dg[i][j][k] = (gh[i][j] - gl[i][j]) / (Xh[k] - Xl[k]);
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) tmp[i][j][k] = 0.5 * (dg[j][i][k] + dg[k][i][j] - dg[k][j][i]);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) {
        double s = 0.;
        for (int l = 0; l < 4; l++) s += gcon[i][l] * tmp[l][j][k];
        conn[i][j][k] = s;
      }
}

// set_grid() (set_grid.c:6-89) over the whole grid, ghost zones included:
// gcov, gcon, gdet at the four locations, the connection at CENT and the
// per-zone floors of set_density_floors (rescaletype 0, fixup.c:996-1110)
// with fixup1zone's lower limits (fixup.c:295-307).  Returns 1 if a metric
// inverse fails.
inline int grid_tables(const Coords& c, int n1, int n2, double rhomin, double uumin, double rhominlimit,
                       double uuminlimit, double* gcov, double* gcon, double* gdet, double* conn, double* floors)
{
  const int n2m = n2 + 2 * NG;
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j < n2 + NG; j++) {
      const long long zr = (long long)(i + NG) * n2m + (j + NG);
      for (int loc = 3; loc >= 0; loc--) {
        double X[4], gv[4][4], gn[4][4];
        coord_of(c, i, j, loc, X);
        gcov_prim(c, X, gv);
        if (gcon_prim(c, X, gn)) return 1;
        memcpy(gcov + (zr * 4 + loc) * 16, gv, sizeof(gv));
        memcpy(gcon + (zr * 4 + loc) * 16, gn, sizeof(gn));
        gdet[zr * 4 + loc] = gdet_of(gv);
        if (loc == CENT) {
          double cn[4][4][4];
          conn_of(c, X, gn, cn);
          memcpy(conn + zr * 64, cn, sizeof(cn));
          double r, th;
          bl_of(c, X, &r, &th);
          double fr = rhomin * pow(r, -1.5), fu = uumin * pow(r, -2.5);
          if (fr < rhominlimit) fr = rhominlimit;
          if (fu < uuminlimit) fu = uuminlimit;
          floors[zr * 2 + 0] = fr;
          floors[zr * 2 + 1] = fu;
        }
      }
    }
  return 0;
}

// ------------------------------------------------------------------ state
struct G {
  const double* gcov;  // 16
  const double* gcon;  // 16
  double g;
};

inline double gamma_of(const double* pr, const G& g)
{
  const double* c = g.gcov;
  double qsq = c[5] * pr[U1] * pr[U1] + c[10] * pr[U2] * pr[U2] + c[15] * pr[U3] * pr[U3] +
               2. * (c[6] * pr[U1] * pr[U2] + c[7] * pr[U1] * pr[U3] + c[11] * pr[U2] * pr[U3]);
  return sqrt(1. + qsq);
}

inline void ucon_rel4(const double* pr, const G& g, double* ucon)
{
  double alpha = 1. / sqrt(-g.gcon[0]);
  double b1 = g.gcon[1] * alpha * alpha, b2 = g.gcon[2] * alpha * alpha, b3 = g.gcon[3] * alpha * alpha;
  double gamma = gamma_of(pr, g);
  ucon[0] = gamma / alpha;
  ucon[1] = pr[U1] - gamma * b1 / alpha;
  ucon[2] = pr[U2] - gamma * b2 / alpha;
  ucon[3] = pr[U3] - gamma * b3 / alpha;
}

inline void lower4(const double* v, const double* c, double* w)
{
  w[0] = c[0] * v[0] + c[1] * v[1] + c[2] * v[2] + c[3] * v[3];
  w[1] = c[1] * v[0] + c[5] * v[1] + c[6] * v[2] + c[7] * v[3];
  w[2] = c[2] * v[0] + c[6] * v[1] + c[10] * v[2] + c[11] * v[3];
  w[3] = c[3] * v[0] + c[7] * v[1] + c[11] * v[2] + c[15] * v[3];
}

inline double bsq_of(const double* pr, const G& g)
{
  double ucon[4], ucov[4], bcon[4], bcov[4];
  ucon_rel4(pr, g, ucon);
  lower4(ucon, g.gcov, ucov);
  bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
  for (int j = 1; j <= 3; j++) bcon[j] = (pr[B1 - 1 + j] + bcon[0] * ucon[j]) / ucon[0];
  lower4(bcon, g.gcov, bcov);
  return bcon[0] * bcov[0] + bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3];
}

// ucon2pr(VELREL4), transforms.c:322-346
inline void ucon_to_rel4(const double* ucon, const G& g, double* pr)
{
  double alphasq = 1. / (-g.gcon[0]);
  double gammaoalpha = ucon[0];
  for (int j = 1; j <= 3; j++) pr[U1 + j - 1] = ucon[j] + alphasq * g.gcon[j] * gammaoalpha;
}

// limit_gamma, fixup.c:1298-1354.  Returns 1 on a negative discriminant.
inline int limit_gamma(double gammamax, double* pr, const G& g)
{
  if (gammamax <= 1.0) return 0;
  double gamma = gamma_of(pr, g);
  if (gamma > gammamax && gamma != 1.0) {
    double pref = (gammamax * gammamax - 1.) / (gamma * gamma - 1.);
    if (pref < 0.0) return 1;
    double f = sqrt(pref);
    pr[U1] *= f;
    pr[U2] *= f;
    pr[U3] *= f;
  }
  return 0;
}

}  // namespace harm_setup
