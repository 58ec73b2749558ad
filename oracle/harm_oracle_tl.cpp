/*
 * Tangent-linear (forward-mode) form of the oracle's step (test
 * infrastructure only: the reference gradient the adjoint kernels are
 * checked against).
 *
 * harm_oracle.c is compiled a second time with its floating-point type
 * replaced by a dual number (value, tangent): every operation carries the
 * derivative along one input direction through the same arithmetic, in the
 * same order, taking the same branch at every limiter, floor, repair and
 * wavespeed choice as the value does (the oracle's only library functions
 * are sqrt and fabs).  The values are therefore the oracle's own, bit for
 * bit, and the tangents are the exact derivative of the branch taken -- the
 * quantity the adjoint computes in reverse.  The Newton inversion is
 * differentiated through its iterations (at convergence the same as the
 * implicit-function derivative to round-off), the cycle-break factor and
 * every discrete decision carry no tangent.
 *
 * Exports (prefix tl_): create on the oracle's geometry, the boundary fill
 * and one step of a state with its tangent, and the horizon accounting with
 * its tangent.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

namespace tl {

struct Dual {
  double v, d;  // value first: the oracle's bit-level reads of a double see the value
  Dual() = default;
  Dual(double x) : v(x), d(0.0) {}
  Dual(int x) : v((double)x), d(0.0) {}
  Dual(long x) : v((double)x), d(0.0) {}
  Dual(unsigned long x) : v((double)x), d(0.0) {}
  Dual(unsigned long long x) : v((double)x), d(0.0) {}
  Dual(double x, double dx) : v(x), d(dx) {}
};

inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator+(Dual a) { return a; }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b)
{
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
inline Dual& operator/=(Dual& a, Dual b) { return a = a / b; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }
inline Dual sqrt(Dual a)
{
  const double s = ::sqrt(a.v);
  return Dual(s, a.d / (2.0 * s));
}
inline Dual fabs(Dual a) { return (a.v < 0.0 || (a.v == 0.0 && signbit(a.v))) ? -a : a; }

}  // namespace tl

using tl::Dual;

#define double Dual
#include "harm_oracle.c"
#undef double

namespace {

struct TL {
  ho_state* s;
  int n1m, n2m;
  Dual *gcov, *gcon, *gdet, *conn, *floors, *p;
};

Dual* lift(const double* x, size_t n)
{
  Dual* y = (Dual*)calloc(n, sizeof(Dual));
  for (size_t k = 0; k < n; k++) y[k] = Dual(x[k]);
  return y;
}

void pack(TL* t, const double* p, const double* dp)
{
  const size_t n = (size_t)t->n1m * t->n2m * NPR;
  for (size_t k = 0; k < n; k++) t->p[k] = Dual(p[k], dp ? dp[k] : 0.0);
}

void unpack(const TL* t, double* p, double* dp)
{
  const size_t n = (size_t)t->n1m * t->n2m * NPR;
  for (size_t k = 0; k < n; k++) {
    p[k] = t->p[k].v;
    if (dp) dp[k] = t->p[k].d;
  }
}

}  // namespace

/* the oracle's plain configuration, field by field (harm_oracle.h's ho_config
   with double in place of the dual type) */
struct tl_config {
  int n1, n2, lim, fluxmethod, eom;
  double cour, gam, dx1, dx2, safe, defcon, gammamax, gammafail, bsqorholimit, bsqoulimit, tf;
  int bc;
  double omegastar;
  int fluxadjust;
  double gammadamp;
};

extern "C" {

void* tl_create(const tl_config* c, const double* gcov, const double* gcon, const double* gdet, const double* conn,
                const double* floors)
{
  TL* t = (TL*)calloc(1, sizeof(TL));
  t->n1m = c->n1 + 2 * NG;
  t->n2m = c->n2 + 2 * NG;
  const size_t nz = (size_t)t->n1m * t->n2m;
  t->gcov = lift(gcov, nz * 64);
  t->gcon = lift(gcon, nz * 64);
  t->gdet = lift(gdet, nz * 4);
  t->conn = lift(conn, nz * 64);
  t->floors = lift(floors, nz * 2);
  t->p = (Dual*)calloc(nz * NPR, sizeof(Dual));
  ho_config hc;
  hc.n1 = c->n1;
  hc.n2 = c->n2;
  hc.lim = c->lim;
  hc.fluxmethod = c->fluxmethod;
  hc.eom = c->eom;
  hc.cour = c->cour;
  hc.gam = c->gam;
  hc.dx1 = c->dx1;
  hc.dx2 = c->dx2;
  hc.safe = c->safe;
  hc.defcon = c->defcon;
  hc.gammamax = c->gammamax;
  hc.gammafail = c->gammafail;
  hc.bsqorholimit = c->bsqorholimit;
  hc.bsqoulimit = c->bsqoulimit;
  hc.tf = c->tf;
  hc.bc = c->bc;
  hc.omegastar = c->omegastar;
  hc.fluxadjust = c->fluxadjust;
  hc.gammadamp = c->gammadamp;
  t->s = ho_create(&hc, t->gcov, t->gcon, t->gdet, t->conn, t->floors);
  return t;
}

void tl_destroy(void* h)
{
  TL* t = (TL*)h;
  if (!t) return;
  ho_destroy(t->s);
  free(t->gcov);
  free(t->gcon);
  free(t->gdet);
  free(t->conn);
  free(t->floors);
  free(t->p);
  free(t);
}

/* bound_prim of a state and its tangent, in place */
void tl_bound(void* h, double* p, double* dp)
{
  TL* t = (TL*)h;
  pack(t, p, dp);
  ho_bound(t->s, t->p);
  unpack(t, p, dp);
}

/* one step of the state and its tangent with the given dt (held fixed: no
   tangent); returns the oracle's fail code */
int tl_step(void* h, double* p, double* dp, int* pflag, double t0, double dt)
{
  TL* t = (TL*)h;
  pack(t, p, dp);
  Dual tt(t0), dd(dt);
  const int rc = ho_step(t->s, t->p, pflag, &tt, &dd);
  unpack(t, p, dp);
  return rc;
}

/* the horizon accounting of the last step (ho_get_horizon) with tangents */
void tl_horizon(void* h, double* out6, double* dout6)
{
  TL* t = (TL*)h;
  Dual o[6];
  ho_get_horizon(t->s, o);
  for (int k = 0; k < 6; k++) {
    out6[k] = o[k].v;
    dout6[k] = o[k].d;
  }
}

}  // extern "C"
