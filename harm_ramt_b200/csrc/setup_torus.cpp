// Host-side plugin surface for standalone runs: the modified Kerr-Schild
// grid and the Fishbone-Moncrief torus that the reference builds in
// coord.c / metric.c / set_grid.c / init.fishmon.c / initbase.c.
//
// This is set-up code (run once, on the host), not the step: it produces the
// geometry tables and the initial primitive state in the reference layout
// that harm_upload_geometry() / harm_set_prims() take.  The arithmetic
// follows the reference's evaluation order so that the geometry agrees with
// the reference bit for bit.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/harm_b200.h"
#include "../../include/harm_setup.h"
#include "setup_grid.h"

namespace {

using namespace harm_setup;

// the reference's seeded generator ranc() (ranc.c:31-54) over libc rand()
struct Ranc {
  int aa[64], S[64], n = 0;
  void seed(int iseed)
  {
    static const int P[64] = {46337, 46327, 46309, 46307, 46301, 46279, 46273, 46271, 46261, 46237, 46229, 46219, 46199,
                              46187, 46183, 46181, 46171, 46153, 46147, 46141, 46133, 46103, 46099, 46093, 46091, 46073,
                              46061, 46051, 46049, 46027, 46021, 45989, 45979, 45971, 45959, 45953, 45949, 45943, 45893,
                              45887, 45869, 45863, 45853, 45841, 45833, 45827, 45823, 45821, 45817, 45779, 45767, 45763,
                              45757, 45751, 45737, 45707, 45697, 45691, 45677, 45673, 45667, 45659, 45641, 45631};
    srand(iseed);
    n = 0;
    for (int i = 0; i < 64; i++) {
      aa[i] = 0;
      S[i] = 0;
      while ((aa[i] = (0x7fff & rand())) < (2 << 8) || aa[i] > P[i] - (2 << 8))
        ;
      while ((S[i] = (0x7fff & rand())) < 1 || aa[i] > P[i] - 1)
        ;
    }
    memcpy(Pp, P, sizeof(P));
  }
  int Pp[64];
  double next()
  {
    n = S[n] & (64 - 1);
    S[n] = (S[n] * aa[n]) % Pp[n];
    return (double)S[n] / (double)Pp[n];
  }
};

}  // namespace

extern "C" {

void harm_torus_default_params(harm_torus_params* p)
{
  memset(p, 0, sizeof(*p));
  p->n1 = 128;
  p->n2 = 128;
  p->a = 0.9375;
  p->hslope = 0.3;
  p->rout = 40.0;
  p->rin_over_rhor = 0.98;
  p->gam = 4. / 3.;
  p->torus_rin = 6.0;
  p->torus_rmax = 12.0;
  p->kappa = 1.e-3;
  p->beta = 1.e2;
  p->randfact = 4.e-2;
  p->seed = 7;
  p->rhomin = 1.e-4;
  p->uumin = 1.e-6;
  p->rhominlimit = 1.e-20;
  p->uuminlimit = 1.e-20;
  p->gammamax = 25.0;
}

int harm_torus_geometry(const harm_torus_params* P, double* gcov, double* gcon, double* gdet, double* conn, double* floors,
                        double* grid_out)
{
  if (!P || !gcov || !gcon || !gdet || !conn || !floors) return HARM_EINVAL;
  const int n1 = P->n1, n2 = P->n2;
  Coords c;
  c.a = P->a;
  c.R0 = 0.0;
  const double rhor = 1. + 1 * sqrt(1. - c.a * c.a);  // rhor_calc(0), phys.c:1075
  c.Rin = P->rin_over_rhor * rhor;
  c.Rout = P->rout;
  c.hslope = P->hslope;
  // set_points defcoord 0, coord.c:722-727
  c.startx1 = log(c.Rin - c.R0);
  c.startx2 = 0.;
  c.dx1 = log((c.Rout - c.R0) / (c.Rin - c.R0)) / n1;
  c.dx2 = 1. / n2;
  if (grid_tables(c, n1, n2, P->rhomin, P->uumin, P->rhominlimit, P->uuminlimit, gcov, gcon, gdet, conn, floors))
    return HARM_EINVAL;
  if (grid_out) {
    grid_out[0] = c.startx1;
    grid_out[1] = c.startx2;
    grid_out[2] = c.dx1;
    grid_out[3] = c.dx2;
    grid_out[4] = c.Rin;
    grid_out[5] = rhor;
  }
  return HARM_OK;
}

// init() of initbase.c:297-562 with init.fishmon.c's torus, up to (but not
// including) the final fixup/bound: the caller applies harm_torus_finish()
// or uploads and lets the device bound it.
int harm_torus_dump_coords(const harm_torus_params* P, harm_dump_header* hdr, double* coords)
{
  if (!P || !hdr || !coords) return HARM_EINVAL;
  const int n1 = P->n1, n2 = P->n2, n2m = n2 + 2 * NG;
  Coords c;
  c.a = P->a;
  c.R0 = 0.0;
  const double rhor = 1. + 1 * sqrt(1. - c.a * c.a);
  c.Rin = P->rin_over_rhor * rhor;
  c.Rout = P->rout;
  c.hslope = P->hslope;
  c.startx1 = log(c.Rin - c.R0);
  c.startx2 = 0.;
  c.dx1 = log((c.Rout - c.R0) / (c.Rin - c.R0)) / n1;
  c.dx2 = 1. / n2;
  hdr->startx1 = c.startx1;
  hdr->startx2 = c.startx2;
  hdr->a = c.a;
  hdr->R0 = c.R0;
  hdr->Rin = c.Rin;
  hdr->Rout = c.Rout;
  hdr->hslope = c.hslope;
  hdr->defcoord = 0;
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j < n2 + NG; j++) {
      double X[4], r, th;
      coord_of(c, i, j, CENT, X);
      bl_of(c, X, &r, &th);
      double* o = coords + ((long long)(i + NG) * n2m + (j + NG)) * 4;
      o[0] = X[1];
      o[1] = X[2];
      o[2] = r;
      o[3] = th;
    }
  return HARM_OK;
}

}  // extern "C"

namespace {

// MKS defcoord 0 coordinates of the torus grid
Coords torus_coords(const harm_torus_params* P)
{
  Coords c;
  c.a = P->a;
  c.R0 = 0.0;
  const double rhor = 1. + 1 * sqrt(1. - c.a * c.a);
  c.Rin = P->rin_over_rhor * rhor;
  c.Rout = P->rout;
  c.hslope = P->hslope;
  c.startx1 = log(c.Rin - c.R0);
  c.startx2 = 0.;
  c.dx1 = log((c.Rout - c.R0) / (c.Rin - c.R0)) / P->n1;
  c.dx2 = 1. / P->n2;
  return c;
}

// init() for the torus; A (may be NULL) receives the corner vector
// potential, norm (may be NULL) the two field normalisation factors
int torus_init_impl(const harm_torus_params* P, const double* gcov, const double* gcon, const double* gdet,
                    double* prims, double* A_out, double* norm_out)
{
  if (!P || !gcov || !gcon || !gdet || !prims) return HARM_EINVAL;
  const int n1 = P->n1, n2 = P->n2, n2m = n2 + 2 * NG, n1m = n1 + 2 * NG;
  const Coords c = torus_coords(P);
  const double a = c.a, gam = P->gam;
  auto Z = [&](int i, int j) { return (long long)(i + NG) * n2m + (j + NG); };
  auto geo = [&](int i, int j) {
    G g;
    const long long z = Z(i, j);
    g.gcov = gcov + (z * 4 + CENT) * 16;
    g.gcon = gcon + (z * 4 + CENT) * 16;
    g.g = gdet[z * 4 + CENT];
    return g;
  };
  auto PR = [&](int i, int j) { return prims + Z(i, j) * 8; };
  memset(prims, 0, sizeof(double) * 8 * (size_t)n1m * n2m);

  Ranc rng;
  rng.seed(P->seed);
  rng.next();  // ranc(7) in init_global returns (and consumes) a deviate too
  // lfish_calc, init.fishmon.c:380-405
  const double rmax = P->torus_rmax, rin = P->torus_rin;
  const double r_ = rmax;
  const double l =
      (((pow(a, 2) - 2. * a * sqrt(r_) + pow(r_, 2)) *
        ((-2. * a * r_ * (pow(a, 2) - 2. * a * sqrt(r_) + pow(r_, 2))) / sqrt(2. * a * sqrt(r_) + (-3. + r_) * r_) +
         ((a + (-2. + r_) * sqrt(r_)) * (pow(r_, 3) + pow(a, 2) * (2. + r_))) / sqrt(1 + (2. * a) / pow(r_, 1.5) - 3. / r_))) /
       (pow(r_, 3) * sqrt(2. * a * sqrt(r_) + (-3. + r_) * r_) * (pow(a, 2) + (-2. + r_) * r_)));
  const double kappa = P->kappa;
  // init_dsandvels over the full grid (i outer), init.fishmon.c:115-226
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j < n2 + NG; j++) {
      double X[4], r, th;
      coord_of(c, i, j, CENT, X);
      bl_of(c, X, &r, &th);
      const double sth = sin(th), cth = cos(th);
      const double DD = r * r - 2. * r + a * a;
      const double AA = (r * r + a * a) * (r * r + a * a) - DD * a * a * sth * sth;
      const double SS = r * r + a * a * cth * cth;
      const double thin = M_PI / 2.;
      const double sthin = sin(thin), cthin = cos(thin);
      const double DDin = rin * rin - 2. * rin + a * a;
      const double AAin = (rin * rin + a * a) * (rin * rin + a * a) - DDin * a * a * sthin * sthin;
      const double SSin = rin * rin + a * a * cthin * cthin;
      double lnh;
      if (r >= rin) {
        lnh = 0.5 * log((1. + sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * sth * AA * sth))) / (SS * DD / AA)) -
              0.5 * sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * AA * sth * sth)) - 2. * a * r * l / AA -
              (0.5 * log((1. + sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin))) /
                         (SSin * DDin / AAin)) -
               0.5 * sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin)) - 2. * a * rin * l / AAin);
      } else {
        lnh = 1.;
      }
      double* pr = PR(i, j);
      const G g = geo(i, j);
      if (lnh < 0. || r < rin) {
        // set_atmosphere(-1), fixup.c:1121-1190, then the PRIMECOORDS round
        // trip of bl2met2metp2v (transforms.c:9-47)
        pr[RHO] = P->rhomin * pow(r, -1.5);
        pr[UU] = P->uumin * pow(r, -2.5);
        pr[U1] = pr[U2] = pr[U3] = 0.0;
        pr[B1] = pr[B2] = pr[B3] = 0;
        double ucon[4];
        ucon_rel4(pr, g, ucon);
        ucon_to_rel4(ucon, g, pr);
      } else {
        const double hm1 = exp(lnh) - 1.;
        const double rho = pow(hm1 * (gam - 1.) / (kappa * gam), 1. / (gam - 1.));
        const double u = kappa * pow(rho, gam) / (gam - 1.);
        const double expm2chi = SS * SS * DD / (AA * AA * sth * sth);
        const double up1 = sqrt((-1. + sqrt(1. + 4. * l * l * expm2chi)) / 2.);
        const double up = 2. * a * r * sqrt(1. + up1 * up1) / sqrt(AA * SS * DD) + sqrt(SS / AA) * up1 / sth;
        pr[RHO] = rho;
        pr[UU] = u * (1. + P->randfact * (rng.next() - 0.5));
        pr[U1] = 0.;
        pr[U2] = 0.;
        pr[U3] = 1.0 * up;
        // VEL4 in Boyer-Lindquist -> u^mu (ucon_calc_4vel with the BL metric,
        // metric.c:601-655, phys.c:962-1012) -> Kerr-Schild (bltoks,
        // transforms.c:109-166) -> prime coords (mettometp) -> rel. 4-velocity
        double ucon[4];
        {
          const double s2 = sth * sth, a2 = a * a, r2 = r * r;
          const double DDb = 1. - 2. / r + a2 / r2;
          const double mu = 1. + a2 * cth * cth / r2;
          double bl[4][4] = {{0}};
          bl[0][0] = (-(1. - 2. / (r * mu)));
          bl[0][3] = (-2. * a * s2 / (r * mu));
          bl[1][1] = (mu / DDb);
          bl[2][2] = (r2 * mu);
          bl[3][0] = bl[0][3];
          bl[3][3] = (r2 * sth * sth * (1. + a2 / r2 + 2. * a2 * s2 / (r2 * r * mu)));
          ucon[1] = pr[U1];
          ucon[2] = pr[U2];
          ucon[3] = pr[U3];
          const double AAq = bl[0][0];
          const double BBq = 2. * (bl[0][1] * ucon[1] + bl[0][2] * ucon[2] + bl[0][3] * ucon[3]);
          const double CCq = 1. + bl[1][1] * ucon[1] * ucon[1] + bl[2][2] * ucon[2] * ucon[2] + bl[3][3] * ucon[3] * ucon[3] +
                             2. * (bl[1][2] * ucon[1] * ucon[2] + bl[1][3] * ucon[1] * ucon[3] + bl[2][3] * ucon[2] * ucon[3]);
          const double discr = BBq * BBq - 4. * AAq * CCq;
          if (discr < 0.) return HARM_EINVAL;
          ucon[0] = (-BBq - sqrt(discr)) / (2. * AAq);
        }
        {
          double tr[4][4] = {{0}};
          tr[0][0] = (1);
          tr[0][1] = (2. * r / (r * r - 2. * r + a * a));
          tr[1][1] = (1);
          tr[2][2] = (1);
          tr[3][1] = (a / (r * r - 2. * r + a * a));
          tr[3][3] = (1);
          double t[4] = {0., 0., 0., 0.};
          for (int jj = 0; jj < 4; jj++)
            for (int kk = 0; kk < 4; kk++) t[jj] += tr[jj][kk] * ucon[kk];
          for (int jj = 0; jj < 4; jj++) ucon[jj] = t[jj];
        }
        {
          double d[4];
          dxdxp_of(c, X, r, d);
          double id[4][4] = {{0}};
          for (int k = 0; k < 4; k++) id[k][k] = 1.0 / d[k];
          double t[4] = {0., 0., 0., 0.};
          for (int jj = 0; jj < 4; jj++)
            for (int kk = 0; kk < 4; kk++) t[jj] += id[jj][kk] * ucon[kk];
          for (int jj = 0; jj < 4; jj++) ucon[jj] = t[jj];
        }
        ucon_to_rel4(ucon, g, pr);
      }
    }
  // normalize_densities, init.fishmon.c:278-306
  double rhomax = 0, umax = 0;
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      double X[4], r, th;
      coord_of(c, i, j, CENT, X);
      bl_of(c, X, &r, &th);
      const double* pr = PR(i, j);
      if (pr[RHO] > rhomax) rhomax = pr[RHO];
      if (pr[UU] > umax && r > rin) umax = pr[UU];
    }
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      PR(i, j)[RHO] /= rhomax;
      PR(i, j)[UU] /= rhomax;
    }
  umax /= rhomax;
  rhomax = 1.;
  // init_atmosphere on the active zones, init.fishmon.c:90-112: where the
  // torus is below the atmosphere, take the atmosphere (the reference's
  // uninitialised B components of its temporary are taken as zero here)
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      double X[4], r, th;
      coord_of(c, i, j, CENT, X);
      bl_of(c, X, &r, &th);
      double* pr = PR(i, j);
      const G g = geo(i, j);
      const double arho = P->rhomin * pow(r, -1.5), au = P->uumin * pow(r, -2.5);
      if (pr[RHO] < arho) {
        pr[RHO] = arho;
        pr[UU] = au;
        pr[U1] = pr[U2] = pr[U3] = 0.0;
        pr[B1] = pr[B2] = pr[B3] = 0.0;
      }
      double ucon[4];
      ucon_rel4(pr, g, ucon);
      ucon_to_rel4(ucon, g, pr);
    }
  // fixup(): fixup1zone on the active zones (floors, gamma limit)
  const double gmax = P->gammamax;
  auto fixup_all = [&]() {
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n2; j++) {
        double X[4], r, th;
        coord_of(c, i, j, CENT, X);
        bl_of(c, X, &r, &th);
        double* pr = PR(i, j);
        double fr = P->rhomin * pow(r, -1.5), fu = P->uumin * pow(r, -2.5);
        if (fr < P->rhominlimit) fr = P->rhominlimit;
        if (fu < P->uuminlimit) fu = P->uuminlimit;
        if (fr > pr[RHO]) pr[RHO] = fr;
        if (fu > pr[UU]) pr[UU] = fu;
        limit_gamma(gmax, pr, geo(i, j));
      }
  };
  fixup_all();
  // the vector potential only needs bounded densities: rho is a plain copy
  // in bound_prim (outflow in x1, mirror in x2)
  for (int j = 0; j < n2; j++)
    for (int i = -1; i >= -NG; i--) {
      PR(i, j)[RHO] = PR(0, j)[RHO];
      PR(n1 - 1 - i, j)[RHO] = PR(n1 - 1, j)[RHO];
    }
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j <= -1; j++) {
      PR(i, j)[RHO] = PR(i, -j - 1)[RHO];
      PR(i, n2 - 1 - j)[RHO] = PR(i, n2 + j)[RHO];
    }
  // init_vpot at corners (DISKFIELD), init.fishmon.c:236-268, and
  // vpot2field, initbase.c:565-618, on the active zones
  std::vector<double> A((size_t)(n1 + 1) * (n2 + 1), 0.0);
  for (int i = 0; i <= n1; i++)
    for (int j = 0; j <= n2; j++) {
      double rho_av = 0.25 * (PR(i, j)[RHO] + PR(i - 1, j)[RHO] + PR(i, j - 1)[RHO] + PR(i - 1, j - 1)[RHO]);
      double q = rho_av / rhomax - 0.2;
      double Av = 0;
      if (q > 0.) Av += q;
      A[(size_t)i * (n2 + 1) + j] = Av;
    }
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      const G g = geo(i, j);
      auto AA_ = [&](int ii, int jj) { return A[(size_t)ii * (n2 + 1) + jj]; };
      double* pr = PR(i, j);
      pr[B1] = (-AA_(i, j) + AA_(i, j + 1) - AA_(i + 1, j) + AA_(i + 1, j + 1)) / (2. * c.dx2 * g.g);
      pr[B2] = -(-AA_(i, j) - AA_(i, j + 1) + AA_(i + 1, j) + AA_(i + 1, j + 1)) / (2. * c.dx1 * g.g);
    }
  // normalize_field twice, init.fishmon.c:310-375 (initbase.c:459 and 490)
  for (int pass = 0; pass < 2; pass++) {
    double bsq_max = 0.;
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n2; j++) {
        double b = bsq_of(PR(i, j), geo(i, j));
        if (b > bsq_max) bsq_max = b;
      }
    const double beta_act = (gam - 1.) * umax / (0.5 * bsq_max);
    const double norm = sqrt(beta_act / P->beta);
    if (norm_out) norm_out[pass] = norm;
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n2; j++) {
        PR(i, j)[B1] *= norm;
        PR(i, j)[B2] *= norm;
        PR(i, j)[B3] *= norm;
      }
  }
  fixup_all();
  if (A_out) std::copy(A.begin(), A.end(), A_out);
  return HARM_OK;
}

}  // namespace

extern "C" {

int harm_torus_init(const harm_torus_params* P, const double* gcov, const double* gcon, const double* gdet, double* prims)
{
  return torus_init_impl(P, gcov, gcon, gdet, prims, nullptr, nullptr);
}

int harm_torus_init_vpot(const harm_torus_params* P, const double* gcov, const double* gcon, const double* gdet,
                         double* prims, double* A, double* norm)
{
  if (!A || !norm) return HARM_EINVAL;
  return torus_init_impl(P, gcov, gcon, gdet, prims, A, norm);
}

int harm_torus_vpot_to_field(const harm_torus_params* P, const double* gdet, const double* A, const double* norm,
                             double* prims)
{
  if (!P || !gdet || !A || !norm || !prims) return HARM_EINVAL;
  const int n1 = P->n1, n2 = P->n2, n2m = n2 + 2 * NG;
  const Coords c = torus_coords(P);
  auto AA = [&](int i, int j) { return A[(size_t)i * (n2 + 1) + j]; };
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      const long long z = (long long)(i + NG) * n2m + (j + NG);
      const double g = gdet[z * 4 + CENT];
      double* pr = prims + z * 8;
      // vpot2field (initbase.c:565-618), then the two normalisations
      pr[B1] = (-AA(i, j) + AA(i, j + 1) - AA(i + 1, j) + AA(i + 1, j + 1)) / (2. * c.dx2 * g);
      pr[B2] = -(-AA(i, j) - AA(i, j + 1) + AA(i + 1, j) + AA(i + 1, j + 1)) / (2. * c.dx1 * g);
      for (int pass = 0; pass < 2; pass++) {
        pr[B1] *= norm[pass];
        pr[B2] *= norm[pass];
      }
    }
  return HARM_OK;
}

int harm_torus_vpot_adjoint(const harm_torus_params* P, const double* gdet, const double* grad_prims,
                            const double* norm, double* grad_A)
{
  if (!P || !gdet || !grad_prims || !norm || !grad_A) return HARM_EINVAL;
  const int n1 = P->n1, n2 = P->n2, n2m = n2 + 2 * NG;
  const Coords c = torus_coords(P);
  const double s = norm[0] * norm[1];
  for (size_t k = 0; k < (size_t)(n1 + 1) * (n2 + 1); k++) grad_A[k] = 0.;
  auto GA = [&](int i, int j) -> double& { return grad_A[(size_t)i * (n2 + 1) + j]; };
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      const long long z = (long long)(i + NG) * n2m + (j + NG);
      const double g = gdet[z * 4 + CENT];
      const double c1 = grad_prims[z * 8 + B1] * s / (2. * c.dx2 * g);
      const double c2 = grad_prims[z * 8 + B2] * s / (2. * c.dx1 * g);
      GA(i, j) += -c1 + c2;
      GA(i, j + 1) += c1 + c2;
      GA(i + 1, j) += -c1 - c2;
      GA(i + 1, j + 1) += c1 - c2;
    }
  return HARM_OK;
}

}  // extern "C"
