// Host-side plugin surface for the force-free aligned rotator: the grid and
// the initial state that the reference builds with init.ns.c (no disk,
// dipole field), bounds.ns.c, coord.c defcoord 6 and metric.c's flat
// spherical metric (SPCMINKMETRIC), through initbase.c's init() for EOMFFDE.
//
// Set-up code, run once on the host.  It is compiled as CUDA only to share
// the step's host-and-device physics (state_of, flux_of and the force-free
// inversion of harm_device.cuh), which filterffde applies to every zone; the
// arithmetic keeps the reference's evaluation order.
#include <math.h>
#include <string.h>

#include <vector>

#include "../../include/harm_b200.h"
#include "../../include/harm_setup.h"
#include "harm_device.cuh"
#include "setup_grid.h"

namespace {

using harm_setup::Coords;
using harm_setup::G;

// defcoord 6 coordinates of the dipole grid (init_grid of the problem with
// R0 = 0, set_points coord.c:763-768)
Coords dipole_coords(const harm_dipole_params* P)
{
  Coords c;
  c.defcoord = 6;
  c.metric = harm_setup::METRIC_SPCMINK;
  c.a = 0.0;
  c.R0 = 0.0;
  c.Rin = P->rin;
  c.Rout = P->rout;
  c.startx1 = log(c.Rin - c.R0);
  c.startx2 = 0.;
  c.dx1 = log((c.Rout - c.R0) / (c.Rin - c.R0)) / P->n1;
  c.dx2 = 1. / P->n2;
  return c;
}

// the packed symmetric metric of the step's physics from a full 4 x 4 table
harm::Geo<double> packed(const G& g)
{
  harm::Geo<double> q;
  for (int j = 0; j < 4; j++)
    for (int k = j; k < 4; k++) {
      q.gcov[harm::sym(j, k)] = g.gcov[j * 4 + k];
      q.gcon[harm::sym(j, k)] = g.gcon[j * 4 + k];
    }
  q.g = g.g;
  return q;
}

// filterffde, phys.ffde.c:1957-1980: the state's conserved quantities in
// the geometry-free form (primtoU with UNOTHING: T^t_mu with rho = u = p = 0,
// B^i), the force-free inversion, then the densities zeroed.  The
// inversion's return value is not looked at, as in the reference.
void filter_ffde(double* pr, const G& g, double gam, double gammamax)
{
  const harm::Geo<double> geo = packed(g);
  harm::State<double> q;
  harm::state_of(pr, geo, q);
  harm::Geo<double> unit = geo;
  unit.g = 1.0;  // flux_of's factor sqrt(-g): the UNOTHING form has none
  double U[harm::NPR], out[harm::NPR];
  harm::flux_of<double, true>(pr, q, 0, unit, gam, U);
  for (int k = 0; k < harm::NPR; k++) out[k] = pr[k];
  (void)harm::utoprim_ffde_geomfree(U, geo, out, gammamax);
  for (int k = 0; k < harm::NPR; k++) pr[k] = out[k];
  pr[harm::RHO] = pr[harm::UU] = 0.0;
}

}  // namespace

extern "C" {

void harm_dipole_default_params(harm_dipole_params* p)
{
  memset(p, 0, sizeof(*p));
  p->n1 = 512;
  p->n2 = 256;
  p->rin = 1.0;
  p->rout = 100.0;
  p->gam = 4. / 3.;
  p->bpole = 1.0;
  p->omegastar = 0.2;
  p->rhomin = 1.e-10;
  p->uumin = 1.e-11;
  p->rhominlimit = 1.e-20;
  p->uuminlimit = 1.e-20;
  p->gammamax = 25.0;
}

int harm_dipole_geometry(const harm_dipole_params* P, double* gcov, double* gcon, double* gdet, double* conn,
                         double* floors, double* grid_out)
{
  if (!P || !gcov || !gcon || !gdet || !conn || !floors || P->n1 < 1 || P->n2 < 1) return HARM_EINVAL;
  const Coords c = dipole_coords(P);
  if (harm_setup::grid_tables(c, P->n1, P->n2, P->rhomin, P->uumin, P->rhominlimit, P->uuminlimit, gcov, gcon, gdet,
                              conn, floors))
    return HARM_EINVAL;
  if (grid_out) {
    grid_out[0] = c.startx1;
    grid_out[1] = c.startx2;
    grid_out[2] = c.dx1;
    grid_out[3] = c.dx2;
    grid_out[4] = c.Rin;
    grid_out[5] = c.Rout;
  }
  return HARM_OK;
}

int harm_dipole_init(const harm_dipole_params* P, const double* gcov, const double* gcon, const double* gdet,
                     double* prims)
{
  using namespace harm_setup;
  if (!P || !gcov || !gcon || !gdet || !prims || P->n1 < 1 || P->n2 < 1) return HARM_EINVAL;
  const int n1 = P->n1, n2 = P->n2, n1m = n1 + 2 * NG, n2m = n2 + 2 * NG;
  const Coords c = dipole_coords(P);
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
  // init_nodisk over the whole grid (init.ns.c:422-440): set_atmosphere(-1)
  // for EOMFFDE -- no densities, zero relative 4-velocity, no field -- then
  // bl2met2metp2v's PRIMECOORDS round trip through u^mu (transforms.c:9-47)
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j < n2 + NG; j++) {
      double* pr = PR(i, j);
      for (int k = 0; k < 8; k++) pr[k] = 0.0;
      double ucon[4];
      ucon_rel4(pr, geo(i, j), ucon);
      ucon_to_rel4(ucon, geo(i, j), pr);
    }
  // normalize_densities and the atmosphere are no-ops without a disk, and
  // the first fixup and bound are GRMHD-only (initbase.c:380-405).
  // init_vpot at every corner of the grid, ghosts included (DIPOLEFIELD,
  // init.ns.c:496-530)
  auto AI = [&](int i, int j) { return (size_t)(i + NG) * n2m + (j + NG); };
  std::vector<double> A((size_t)n1m * n2m, 0.0);
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j < n2 + NG; j++) {
      double X[4], r, th;
      coord_of(c, i, j, CORN, X);
      bl_of(c, X, &r, &th);
      double Av = 0;
      Av += 0.5 * P->bpole * c.Rin * c.Rin * c.Rin * sin(th) * sin(th) / r;
      A[AI(i, j)] = Av;
    }
  // vpot2field, initbase.c:565-618: flux-CT field of every zone whose four
  // corners exist, then the last column and row copied from their
  // neighbours and the two corner zones of the first column
  for (int i = -NG; i <= n1 + NG - 2; i++)
    for (int j = -NG; j <= n2 + NG - 2; j++) {
      const G g = geo(i, j);
      double* pr = PR(i, j);
      pr[B1] = (-A[AI(i, j)] + A[AI(i, j + 1)] - A[AI(i + 1, j)] + A[AI(i + 1, j + 1)]) / (2. * c.dx2 * g.g);
      pr[B2] = -(-A[AI(i, j)] - A[AI(i, j + 1)] + A[AI(i + 1, j)] + A[AI(i + 1, j + 1)]) / (2. * c.dx1 * g.g);
    }
  for (int i = -NG; i < n1 + NG; i++)
    for (int j = -NG; j < n2 + NG; j++) {
      if (i == n1 - 1 + NG) {
        PR(i, j)[B1] = PR(i - 1, j)[B1];
        PR(i, j)[B2] = PR(i - 1, j)[B2];
      } else if (j == n2 - 1 + NG) {
        PR(i, j)[B1] = PR(i, j - 1)[B1];
        PR(i, j)[B2] = PR(i, j - 1)[B2];
      }
    }
  PR(-NG, -NG)[B1] = PR(-NG + 1, -NG)[B1];
  PR(-NG, -NG)[B2] = PR(-NG + 1, -NG)[B2];
  PR(-NG, n2 - 1 + NG)[B1] = PR(-NG + 1, n2 - 1 + NG)[B1];
  PR(-NG, n2 - 1 + NG)[B2] = PR(-NG + 1, n2 - 1 + NG)[B2];
  // normalize_field and init_postfield do nothing for this problem; each is
  // followed by filterffde over the whole grid (initbase.c:486-515)
  for (int pass = 0; pass < 2; pass++)
    for (int i = -NG; i < n1 + NG; i++)
      for (int j = -NG; j < n2 + NG; j++) filter_ffde(PR(i, j), geo(i, j), P->gam, P->gammamax);
  // fixup (FIXUPAFTERINIT): for EOMFFDE fixup1zone only limits the Lorentz
  // factor (fixup.c:293, 337-341), on the active zones
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) limit_gamma(P->gammamax, PR(i, j), geo(i, j));
  return HARM_OK;
}

}  // extern "C"
