// Adjoint (reverse-mode) kernels of one RK2 step of the FP64 GRMHD path on
// the torus boundaries, dt held at the forward run's values.
//
// One substep of the forward step is: update (U(pi) + c dt (flux divergence
// with flux-CT + geometric source of pb), con-to-prim, floors, Lorentz
// limit) -> bound + POLEDEATH -> check-solution / fixup_utoprim -> bound +
// POLEDEATH.  Its adjoint runs the pieces backwards (host sequence in
// harm_capi.cu, adjoint_substep): k_adj_poledeath + k_adj_ghosts (second
// bound), k_adj_fixup, k_adj_poledeath + k_adj_ghosts (first bound),
// k_adj_update (floors, limit, inverse function theorem on the con-to-prim
// Jacobian), k_adj_upi (U(pi)), k_adj_source (geometric source), k_adj_corner (flux-CT
// EMFs), then per direction k_adj_faces (face fluxes -> interface-state
// adjoints) and k_adj_recon (reconstructions, scattered onto pb with
// atomics).  All adjoint arrays are planes in the step's layout, ghost zones
// included.
#include <cuda_runtime.h>

#include "harm_adjoint.cuh"
#include "harm_kernels.cuh"

namespace harm {

namespace {

__device__ __forceinline__ void load_prims(const double* __restrict__ pv, long long pl, long long z, double* p)
{
#pragma unroll
  for (int k = 0; k < NPR; k++) p[k] = pv[k * pl + z];
}

__device__ __forceinline__ bool active(const StepArgs& a, int i, int j)
{
  return i >= 0 && i < a.gr.n1 && j >= 0 && j < a.gr.n2;
}

}  // namespace

// edot seed: d/dp of w dt (b^2 u^r u_t - b^r b_t) sqrt(-g) dx2 2pi at the
// zones (0, j) of the step's final state (diag_flux's EM terms, as horizon_terms
// forms); dt is the step's (a.sc->dt)
__global__ void k_adj_seed_edot(StepArgs a, const double* __restrict__ pv, double* lam, double wfac)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const double w = wfac * a.sc->dt;
  if (j >= a.gr.n2 || w == 0.) return;
  const long long pl = a.gr.plane, z = a.gr.at(0, j);
  double p[NPR];
  load_prims(pv, pl, z, p);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  State<double> q;
  state_of(p, g, q);
  const double sg = g.g * a.pp.dx2 * (2.0 * 3.14159265358979323846);
  const double bsq = dot4(q.bcon, q.bcov);
  StateAdj qb;
  qb.zero();
  const double bsqb = w * q.ucon[1] * q.ucov[0] * sg;
  qb.ucon[1] += w * bsq * q.ucov[0] * sg;
  qb.ucov[0] += w * bsq * q.ucon[1] * sg;
  qb.bcon[1] += -w * q.bcov[0] * sg;
  qb.bcov[0] += -w * q.bcon[1] * sg;
  for (int k = 0; k < 4; k++) {
    qb.bcon[k] += bsqb * q.bcov[k];
    qb.bcov[k] += bsqb * q.bcon[k];
  }
  double pb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  adj_state(p, g, q, qb, pb);
#pragma unroll
  for (int k = 0; k < NPR; k++) lam[k * pl + z] += pb[k];
}

// POLEDEATH zeroes u~2 and B2 of the first and last active rows after the
// ghosts were filled: those outputs do not depend on their inputs
__global__ void k_adj_poledeath(StepArgs a, double* lam)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.gr.n1) return;
  const int j = (blockIdx.y == 0) ? 0 : a.gr.n2 - 1;
  const long long z = a.gr.at(i, j);
  lam[U2 * a.gr.plane + z] = 0.;
  lam[B2 * a.gr.plane + z] = 0.;
}

// Ghost zones (torus): each is a function of one active zone (x1 outflow
// copy with inflow check and Lorentz limit, polar mirror copy, u~2 and B2
// zeroed on POLEDEATH rows).  Its adjoint goes to that zone (atomic adds);
// the ghost's own entry is cleared.  src: the active values the bound read.
__global__ void k_adj_ghosts(StepArgs a, double* lam, const double* __restrict__ src)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - NG;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - NG;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i >= n1 + NG || j >= n2 + NG) return;
  const bool xin = (i >= 0 && i < n1), yin = (j >= 0 && j < n2);
  if (xin && yin) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  double lg[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) {
    lg[k] = lam[k * pl + z];
    lam[k * pl + z] = 0.;
  }
  const int jm = yin ? j : ((j < 0) ? (-j - 1) : (2 * n2 - 1 - j));
  const bool zeroed = (!yin) || (j == 0 || j == n2 - 1);  // POLEDEATH of the torus
  if (zeroed) {
    lg[U2] = 0.;
    lg[B2] = 0.;
  }
  const int si = xin ? i : ((i < 0) ? 0 : n1 - 1);
  const long long zs = a.gr.at(si, jm);
  if (!xin) {
    // x1 map evaluated with the ghost (i, jm)'s geometry, on the source's u~
    double s[NPR];
    load_prims(src, pl, zs, s);
    Geo<double> g;
    load_geo(a, CENT, a.gr.at(i, jm), g);
    double ucon[4];
    ucon_of(s, g, ucon);
    const bool dofix = ((i <= -1) && (ucon[1] > 0.)) || ((i >= n1) && (ucon[1] < 0.));
    Tan<3> u[3];
    for (int m = 0; m < 3; m++) {
      u[m] = Tan<3>(s[U1 + m]);
      u[m].d[m] = 1.;
    }
    if (x1_velocity_map(u, g, a.pp.gammamax, dofix)) return;
    double lu[3] = {0., 0., 0.};
    for (int m = 0; m < 3; m++)
      for (int c = 0; c < 3; c++) lu[c] += lg[U1 + m] * u[m].d[c];
    lg[U1] = lu[0];
    lg[U2] = lu[1];
    lg[U3] = lu[2];
  }
#pragma unroll
  for (int k = 0; k < NPR; k++)
    if (lg[k] != 0.) atomicAdd(&lam[k * pl + zs], lg[k]);
}

// fixup_utoprim's repairs (fixup.c:527-928 as k_fixup_compute forms them):
// a repaired zone's rho..u3 are an average of neighbours of the snapshot
// (the recorded set), then Lorentz-limited at min(its own gamma, GAMMAMAX).
// lam_in: adjoint after the repair; lam_snap (zeroed by the caller): adjoint
// of the snapshot, ghosts included.
__global__ void k_adj_fixup(StepArgs a, const double* __restrict__ lam_in, double* lam_snap,
                            const double* __restrict__ snap, const int* __restrict__ flag,
                            const unsigned char* __restrict__ fixset)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (!active(a, i, j)) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  double lo[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) lo[k] = lam_in[k * pl + z];
  if (flag[z] != PF_FIXED) {
#pragma unroll
    for (int k = 0; k < NPR; k++)
      if (lo[k] != 0.) atomicAdd(&lam_snap[k * pl + z], lo[k]);
    return;
  }
  // the neighbour set: offsets and weights
  int ni[8], nj[8], nn = 0;
  double w[8];
  const int set = fixset[z];
  auto put = [&](int di, int dj, double ww) {
    ni[nn] = di;
    nj[nn] = dj;
    w[nn] = ww;
    nn++;
  };
  if (set == 0) {
    put(0, 1, 0.25); put(0, -1, 0.25); put(-1, 0, 0.25); put(1, 0, 0.25);
  } else if (set == 1) {
    put(1, 1, 0.25); put(1, -1, 0.25); put(-1, 1, 0.25); put(-1, -1, 0.25);
  } else if (set == 2) {
    put(0, 1, 0.5); put(0, -1, 0.5);
  } else if (set == 3) {
    put(1, 0, 0.5); put(-1, 0, 0.5);
  } else if (set == 4) {
    put(1, 1, 0.5); put(-1, -1, 0.5);
  } else if (set == 5) {
    put(1, -1, 0.5); put(-1, 1, 0.5);
  } else if (set < 14) {
    const int oi[8] = {1, 1, 1, 0, -1, -1, -1, 0};
    const int oj[8] = {1, 0, -1, -1, -1, 0, 1, 1};
    put(oi[set - 6], oj[set - 6], 1.0);
  } else {
    put(0, 1, 0.125); put(0, -1, 0.125); put(-1, 0, 0.125); put(1, 0, 0.125);
    put(1, 1, 0.125); put(1, -1, 0.125); put(-1, 1, 0.125); put(-1, -1, 0.125);
  }
  // forward recompute of the averaged state
  double own[NPR], pr[NPR];
  load_prims(snap, pl, z, own);
  for (int k = 0; k < NPR; k++) pr[k] = own[k];
  for (int k = 0; k <= U3; k++) {
    double s = 0.;
    for (int m = 0; m < nn; m++) s += w[m] * snap[k * pl + a.gr.at(i + ni[m], j + nj[m])];
    pr[k] = s;
  }
  Geo<double> g;
  load_geo(a, CENT, z, g);
  const double gown = gamma_of(own, g);
  const bool capped = gown > a.pp.gammamax;
  const double gm = capped ? a.pp.gammamax : gown;
  double lp[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  adj_limit_gamma(gm, pr, g, lo, lp);
  // the limit's dependence on gm (the zone's own gamma when below GAMMAMAX)
  if (!capped && gm > 1.0) {
    const double gamma = gamma_of(pr, g);
    if (gamma > gm && gamma != 1.0) {
      const double f = sqrt((gm * gm - 1.) / (gamma * gamma - 1.));
      double fb = 0.;
      for (int k = U1; k <= U3; k++) fb += lo[k] * pr[k];
      const double gmb = fb * gm / ((gamma * gamma - 1.) * f);
      double lown[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
      adj_gamma(own, g, gmb, lown);
      for (int k = U1; k <= U3; k++)
        if (lown[k] != 0.) atomicAdd(&lam_snap[k * pl + z], lown[k]);
    }
  }
  for (int k = 0; k <= U3; k++)
    if (lp[k] != 0.)
      for (int m = 0; m < nn; m++) atomicAdd(&lam_snap[k * pl + a.gr.at(i + ni[m], j + nj[m])], w[m] * lp[k]);
  for (int k = B1; k <= B3; k++)
    if (lp[k] != 0.) atomicAdd(&lam_snap[k * pl + z], lp[k]);
}

// The zone update's con-to-prim: lam (adjoint of the update's output) ->
// ubar (Ubar, the adjoint of the updated conserved vector) and lam_dU (=
// c dt Ubar, for the fluxes and the source; c = cfac, dt the step's
// a.sc->dt).
// pinv: the inverted primitives before floors; flaginv: the inversion's
// pflag.  The geometric source's adjoint is k_adj_source's: built into this
// kernel (after the con-to-prim Jacobian), sm_100a code of nvcc 12.9 gave
// source adjoints that differ from the same function's host build and from
// finite differences, at any ptxas optimisation level.
__global__ void k_adj_update(StepArgs a, const double* __restrict__ lam, const double* __restrict__ pinv,
                             const int* __restrict__ flaginv, double cfac, double* ubar, double* lam_dU)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (!active(a, i, j)) return;
  const double cdt = cfac * a.sc->dt;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  const double gam = a.pp.gam;
  double lp[NPR], Ub[NPR];
  load_prims(lam, pl, z, lp);
  if (flaginv[z] != 0) {
    // a failed inversion: only B = U_B / sqrt(-g) is kept from it
    for (int k = 0; k < NPR; k++) Ub[k] = 0.;
    for (int k = B1; k <= B3; k++) Ub[k] = lp[k] / g.g;
  } else {
    double p1[NPR];
    load_prims(pinv, pl, z, p1);
    const double frho = a.geo[(long long)GEO_FLOOR * pl + z], fu = a.geo[(long long)(GEO_FLOOR + 1) * pl + z];
    const bool crho = frho > p1[RHO], cu = fu > p1[UU];
    double pfl[NPR];
    for (int k = 0; k < NPR; k++) pfl[k] = p1[k];
    if (crho) pfl[RHO] = frho;
    if (cu) pfl[UU] = fu;
    double l1[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
    adj_limit_gamma(a.pp.gammamax, pfl, g, lp, l1);
    if (crho) l1[RHO] = 0.;
    if (cu) l1[UU] = 0.;
    if (ift_solve(p1, g, gam, l1, Ub))
      for (int k = 0; k < NPR; k++) Ub[k] = 0.;
  }
  for (int k = 0; k < NPR; k++) {
    ubar[k * pl + z] = Ub[k];
    lam_dU[k * pl + z] = cdt * Ub[k];
  }
}

// Uf = U(pi) + c dt (dUr + dUg): the U(pi) part, lam_pi += (dU/dp at pi)^T
// ubar (a kernel of its own: with the implicit-function step in the same
// kernel both ran at two blocks per SM)
__global__ void k_adj_upi(StepArgs a, const double* __restrict__ ubar, const double* __restrict__ pi, double* lam_pi)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (!active(a, i, j)) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  double Ub[NPR], p[NPR];
  load_prims(ubar, pl, z, Ub);
  load_prims(pi, pl, z, p);
  State<double> q;
  state_of(p, g, q);
  StateAdj qb;
  qb.zero();
  double lpi[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  adj_flux(p, q, 0, g, a.pp.gam, Ub, qb, lpi);
  adj_state(p, g, q, qb, lpi);
  for (int k = 0; k < NPR; k++) lam_pi[k * pl + z] += lpi[k];
}

// The geometric source dUg[UU+l] = g sum_jj sum_k T^jj_k Gamma^k_{l jj} at
// pb, whose adjoint in U is lam_dU (the update's c dt Ubar): lam_b (the pb
// adjoint) is set to the source's part, the faces add theirs after.
__global__ void k_adj_source(StepArgs a, const double* __restrict__ pb, const double* __restrict__ lam_dU,
                             double* lam_b)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (!active(a, i, j)) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  double p[NPR], conn40[40], dUgb[4];
  load_prims(pb, pl, z, p);
  for (int c = 0; c < 40; c++) conn40[c] = a.geo[(long long)(GEO_CONN + c) * pl + z];
  for (int l = 0; l < 4; l++) dUgb[l] = lam_dU[(UU + l) * pl + z];
  double lb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  adj_source(p, g, a.pp.gam, conn40, dUgb, lb);
  for (int k = 0; k < NPR; k++) lam_b[k * pl + z] = lb[k];
}

// flux-CT corner EMFs, from the B1/B2 rows of lam_dU of the four zones that
// share the corner (c = (i, j) for i in [0, N1], j in [0, N2])
__global__ void k_adj_corner(StepArgs a, const double* __restrict__ lam_dU, double* lam_e)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > a.gr.n1 || j > a.gr.n2) return;
  const long long pl = a.gr.plane;
  const double idx1 = 1.0 / a.pp.dx1, idx2 = 1.0 / a.pp.dx2;
  double e = 0.;
  auto add = [&](int zi, int zj, double c1, double c2) {
    if (!active(a, zi, zj)) return;
    const long long zz = a.gr.at(zi, zj);
    e += lam_dU[B1 * pl + zz] * c1 * idx2 + lam_dU[B2 * pl + zz] * c2 * idx1;
  };
  add(i, j, -0.5, 0.5);
  add(i - 1, j, -0.5, -0.5);
  add(i, j - 1, 0.5, 0.5);
  add(i - 1, j - 1, 0.5, -0.5);
  lam_e[a.gr.at(i, j)] = e;
}

// One face direction: the face-flux adjoint (from lam_dU of the two zones,
// the EMF adjoints of its corners, and a seed seed_fac dt on the x1 mass flux
// at i = 0), fix_flux's zeroed components, then the face itself: sl, sr (8
// planes each, indexed by the face) get the adjoints of its left and right
// interface states, zero where the face carries none.  k_adj_recon takes
// them through the reconstructions.
template <int dir>
__global__ void k_adj_faces(StepArgs a, const double* __restrict__ pb, const double* __restrict__ lam_dU,
                            const double* __restrict__ lam_e, double* sl, double* sr, double seed_fac)
{
  const double seed_mdot = seed_fac * a.sc->dt;
  const int i = blockIdx.x * blockDim.x + threadIdx.x - (dir == 2 ? 1 : 0);
  const int j = blockIdx.y * blockDim.y + threadIdx.y - (dir == 1 ? 1 : 0);
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i > n1 || j > n2) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const double idx1 = 1.0 / a.pp.dx1, idx2 = 1.0 / a.pp.dx2;
  const int di = (dir == 1), dj = (dir == 2);
  double Fb[NPR];
  auto ldu = [&](int zi, int zj, int k) -> double {
    return active(a, zi, zj) ? lam_dU[k * pl + a.gr.at(zi, zj)] : 0.;
  };
  auto le = [&](int ci, int cj) -> double {
    return (ci >= 0 && ci <= n1 && cj >= 0 && cj <= n2) ? lam_e[a.gr.at(ci, cj)] : 0.;
  };
  auto gc = [&](int ci, int cj) -> double { return gdet_at(a, CORN, a.gr.at(ci, cj)); };
  const double id = (dir == 1) ? idx1 : idx2;
  for (int k = 0; k < NPR; k++) Fb[k] = id * (ldu(i, j, k) - ldu(i - di, j - dj, k));
  if (dir == 1) {
    Fb[B1] = 0.;
    double f = 0.;
    const double gf = gdet_at(a, FACE1, z);
    if (!(j == n2 && i < n1)) f += le(i, j) * 0.25 * ((i <= n1 && j >= 0 && j <= n2) ? gc(i, j) : 0.) / gf;
    if (!(j == -1 && i < n1) && j + 1 >= 0 && j + 1 <= n2) f += le(i, j + 1) * 0.25 * gc(i, j + 1) / gf;
    if (j == n2 - 1 && i < n1) f += -le(i, n2) * 0.25 * gc(i, n2) / gdet_at(a, FACE1, a.gr.at(i, n2));
    if (j == 0 && i < n1) f += -le(i, 0) * 0.25 * gc(i, 0) / gdet_at(a, FACE1, a.gr.at(i, -1));
    Fb[B2] = f;
    if (i == 0 && j >= 0 && j < n2) Fb[RHO] += seed_mdot;
  } else {
    Fb[B2] = 0.;
    const double gf = gdet_at(a, FACE2, z);
    double f = 0.;
    if (i >= 0 && j >= 0) f += -le(i, j) * 0.25 * gc(i, j) / gf;
    if (i + 1 <= n1 && j >= 0) f += -le(i + 1, j) * 0.25 * gc(i + 1, j) / gf;
    Fb[B1] = f;
    const bool polar = (j == 0 || j == n2) && (i < n1);
    const bool equator = (j == (n2 - 1) / 2) && (i >= 0) && (i < n1);
    if (polar || equator)
      for (int k = 0; k < NPR; k++)
        if (k != U2) Fb[k] = 0.;
  }
  bool any = false;
  for (int k = 0; k < NPR; k++) any |= (Fb[k] != 0.);
  double plb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.}, prb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  auto store = [&]() {
    for (int k = 0; k < NPR; k++) {
      sl[k * pl + z] = plb[k];
      sr[k * pl + z] = prb[k];
    }
  };
  if (!any) {
    store();
    return;
  }
  // the two interface states: right state of zone (i-di, j-dj), left of (i, j)
  const int para = (a.pp.lim == 4);
  const long long s = (dir == 1) ? 1LL : (long long)a.gr.pitch;
  const long long zl = z - s;
  double pls[NPR], prs[NPR];
  for (int k = 0; k < NPR; k++) {
    double yl[5], yr[5];
    for (int m = 0; m < 5; m++) {
      const long long o = (long long)(m - 2) * s;
      const bool in = para || (m >= 1 && m <= 3);
      yl[m] = in ? pb[k * pl + zl + o] : 0.;
      yr[m] = in ? pb[k * pl + z + o] : 0.;
    }
    double lo, ro;
    if (para) {
      para4(yl[0], yl[1], yl[2], yl[3], yl[4], lo, ro);
      pls[k] = ro;
      para4(yr[0], yr[1], yr[2], yr[3], yr[4], lo, ro);
      prs[k] = lo;
    } else {
      double dq = mc_slope(yl[1], yl[2], yl[3]);
      pls[k] = yl[2] + 0.5 * dq;
      dq = mc_slope(yr[1], yr[2], yr[3]);
      prs[k] = yr[2] - 0.5 * dq;
    }
  }
  Geo<double> g;
  load_geo(a, dir == 1 ? FACE1 : FACE2, z, g);
  if (dir == 1 && (i == 0 || i == n1) && j >= -1 && j < n2 && Fb[RHO] != 0.) {
    // fix_flux's mass-flux sign clamp at the x1 ends (torus: both OUTFLOW)
    double Fo[NPR];
    if (!face_flux_primal(pls, prs, g, dir, a.pp.gam, a.pp.gammamax, a.pp.fluxmethod, Fo)) {
      if ((i == 0 && Fo[RHO] > 0) || (i == n1 && Fo[RHO] < 0)) Fb[RHO] = 0.;
    }
  }
  if (adj_face_flux(pls, prs, g, dir, a.pp.gam, a.pp.gammamax, a.pp.fluxmethod, Fb, plb, prb))
    for (int k = 0; k < NPR; k++) plb[k] = prb[k] = 0.;
  store();
}

// The reconstructions of one direction backwards: zone (i, j), i in
// [-1, N1], j in [-1, N2], has its left state on face (i, j) (that face's
// right state, adjoint sr) and its right state on the next face (that
// face's left state, adjoint sl); its MC/PARA4 rows (both states from one
// evaluation) scatter them onto lam_b at the stencil zones.
// A field component whose whole stencil lies below B_NOISE sqrt(rho) of
// the zone (b^2/rho < 1e-20: round-off left where no field has arrived)
// takes the rows of a tie (each state = the zone's value).  There the
// limiter's branch is set by round-off, the exact derivative holds only for
// perturbations below that level, and its transpose over many steps grows
// without bound; any resolvable perturbation sees the tie's rows.
constexpr double B_NOISE = 1e-10;

template <int dir>
__global__ void k_adj_recon(StepArgs a, const double* __restrict__ pb, const double* __restrict__ sl,
                            const double* __restrict__ sr, double* lam_b)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i > n1 || j > n2) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const long long s = (dir == 1) ? 1LL : (long long)a.gr.pitch;
  // faces of this direction: x1 i in [0, N1], j in [-1, N2]; x2 j in [0, N2], i in [-1, N1]
  const int f0 = (dir == 1) ? i : j, nf = (dir == 1) ? n1 : n2;
  const bool has_l = (f0 >= 0 && f0 <= nf), has_r = (f0 + 1 >= 0 && f0 + 1 <= nf);
  const int para = (a.pp.lim == 4);
  const double bnoise = B_NOISE * sqrt(fmax(pb[RHO * pl + z], 0.));
  for (int k = 0; k < NPR; k++) {
    const double ll = has_l ? sr[k * pl + z] : 0., lr = has_r ? sl[k * pl + z + s] : 0.;
    if (ll == 0. && lr == 0.) continue;
    double y[5], ymax = 0.;
    for (int m = 0; m < 5; m++) {
      const bool in = para || (m >= 1 && m <= 3);
      y[m] = in ? pb[k * pl + z + (long long)(m - 2) * s] : 0.;
      ymax = fmax(ymax, fabs(y[m]));
    }
    double cl[5], cr[5];
    if (k >= B1 && ymax < bnoise) {
      for (int m = 0; m < 5; m++) cl[m] = cr[m] = (m == 2) ? 1. : 0.;
    } else {
      recon_rows(para, y, cl, cr);
    }
    for (int m = 0; m < 5; m++) {
      const double v = cl[m] * ll + cr[m] * lr;
      if (v != 0.) atomicAdd(&lam_b[k * pl + z + (long long)(m - 2) * s], v);
    }
  }
}

// dt held at recorded values: dt of step k before it runs
__global__ void k_set_dt(StepArgs a, const double* __restrict__ dts, int k) { a.sc->dt = dts[k]; }
__global__ void k_get_dt(StepArgs a, double* dts, int k) { dts[k] = a.sc->dt; }

// clears the ghost zones of an adjoint (the objective weights active zones)
__global__ void k_mask_ghosts(StepArgs a, double* lam)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - NG;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - NG;
  if (i >= a.gr.n1 + NG || j >= a.gr.n2 + NG || active(a, i, j)) return;
  for (int k = 0; k < NPR; k++) lam[k * a.gr.plane + a.gr.at(i, j)] = 0.;
}

// y += x over n values
__global__ void k_axpy(double* y, const double* __restrict__ x, long long n)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] += x[t];
}

// <lam, p> over active zones: out[block] = the block's partial sum (fixed
// order inside the block; the host adds the partials in block order)
__global__ void k_dot_active(StepArgs a, const double* __restrict__ lam, const double* __restrict__ pv, double* out)
{
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  double s = 0.;
  if (active(a, i, j)) {
    const long long z = a.gr.at(i, j);
    for (int k = 0; k < NPR; k++) s += lam[k * a.gr.plane + z] * pv[k * a.gr.plane + z];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if ((t & 31) == 0) sh[t >> 5] = s;
  __syncthreads();
  if (t == 0) {
    double b = 0.;
    for (int w = 0; w < (int)((blockDim.x * blockDim.y + 31) / 32); w++) b += sh[w];
    out[blockIdx.y * gridDim.x + blockIdx.x] = b;
  }
}

// the direction is a template parameter: every dir-indexed state component
// is then a constant index and stays in registers
template __global__ void k_adj_faces<1>(StepArgs, const double*, const double*, const double*, double*, double*,
                                        double);
template __global__ void k_adj_faces<2>(StepArgs, const double*, const double*, const double*, double*, double*,
                                        double);
template __global__ void k_adj_recon<1>(StepArgs, const double*, const double*, const double*, double*);
template __global__ void k_adj_recon<2>(StepArgs, const double*, const double*, const double*, double*);

}  // namespace harm
