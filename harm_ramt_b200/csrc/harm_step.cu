// HARM finite-volume step on sm_100a: the kernels of one RK2 substep.
//
// Substep pipeline (reference step_ch.c:79-136 for one timeorder):
//   k_flux         fluxcalc x1 and x2 faces + fix_flux + per-block dt minima
//                  (with the flux switch, the first substep also forms the
//                  b^2 flags and flux choices)
//   k_emf          flux_ct corner EMFs (Toth, CORNGDETVERSION 1)
//   k_update       advance_standard zone loop: U(pi), geometric source(pb),
//                  flux divergence with the CT-rewritten B fluxes, RK combine,
//                  2D Newton con-to-prim, fixup1zone
//   k_update_tail  inversions still unconverged after 16 Newton iterations
//   k_bound_gc     bound_prim + bound_pflag (ghost zones) and the check-
//                  solution gamma table
//   k_checksol,
//   k_checksol_rounds  fixup_checksolution (parallel fixed-point sweep, exact)
//   k_fixup_compute    fixup_utoprim from a snapshot
//   k_bound_fix    the repairs applied, the second bound and POLEDEATH; after
//                  the last substep its last block also ends the step
//                  (horizon sums, new dt)
// The adjoint's recording path, the force-free step and the currents use
// k_bound, k_poledeath, k_gammacheck, k_fixup_apply, k_bsqflags, k_step_end.
#include <cuda_runtime.h>
#include "harm_step_impl.cuh"
#include "harm_tryagain.cuh"

namespace harm {

// ---------------------------------------------------------------- flags
// get_bsqflags, fixup.c:1197-1295 over the DQZLOOP range [-1,N1]x[-1,N2]
// (with fluxadjust also the flux choice of each zone)
__global__ void k_bsqflags(StepArgs a, const double* __restrict__ pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
  if (i > a.gr.n1 || j > a.gr.n2) return;
  const long long z = a.gr.at(i, j);
  if (a.pp.eom && !a.pp.fluxadjust) {  // the b^2 checks are GRMHD-only (fixup.c:1214-1233)
    a.bsqf[z] = 0;
    return;
  }
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = __ldg(pv + k * a.gr.plane + z);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  unsigned char b = 0;
  if (!a.pp.eom) {
    State<double> q;
    state_of(pr, g, q);
    b = bsq_flag(a, pr, q);
  }
  a.bsqf[z] = b;
  if (a.pp.fluxadjust) {
    // FLAGREALFLUX (fixup.c:1236-1245, 1284-1290): the Lorentz-factor flag
    // joins the b^2 flags; where any is 2 the hydro fluxes step down from
    // fluxmethod (HLL -> LAXF, not below LAXF)
    const double gamma = gamma_of(pr, g);
    const int f1 = (gamma > 2.0 * a.pp.gammadamp) ? 2 : ((gamma > a.pp.gammadamp) ? 1 : 0);
    const int rf = ((b & 3) == 2 || f1 == 2 || (b >> 2) == 2) ? a.pp.fluxmethod - 1 : a.pp.fluxmethod;
    a.fluxf[z] = (unsigned char)(rf < 0 ? 0 : rf);
  }
}

// The deferred inversions of k_update, continued from the Newton state
// k_update saved (repair scratch planes 0-4) up to the full iteration limit.
// A deferred zone's pf slot was not written, so pi still holds its guess.
// TA: the UTOPRIMTRYAGAIN retry chain follows a failed 2D inversion (those
// zones carry no saved state and are solved afresh).
template <bool TA>
__global__ void __launch_bounds__(64) k_update_tail(StepArgs a, const double* __restrict__ pi, double* __restrict__ pf)
{
  const int nd = a.sc->ndeferred;
  const long long pl = a.gr.plane;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nd; w += gridDim.x * blockDim.x) {
    const long long z = a.worklist[w];
    const int i = (int)(z % a.gr.pitch) - NG, j = (int)(z / a.gr.pitch) - NG;
    Geo<double> g;
    load_geo(a, CENT, z, g);
    double U[NPR], pfz[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) {
      U[k] = a.ubuf[k * pl + z];
      pfz[k] = pi[k * pl + z];
    }
    int niter;
    double* nst = a.fixbuf + z;
    const bool resume = nst[(NEWTON_STATE - 1) * pl] >= 0.0;
    int pfl = utoprim_2d(U, g, pfz, a.pp.gam, a.pp.gammafail, &niter, 200, nst, pl, resume);
    if (TA && pfl != 0) {
      double pr0[NPR];
#pragma unroll
      for (int k = 0; k < NPR; k++) pr0[k] = pi[k * pl + z];
      pfl = ta::tryagain_chain(U, g, a.pp.gam, a.pp.gammafail, pr0, pfz, pfl);
    }
    finish_zone(a, g, z, i, j, pfz, pfl, pf, __ldg(a.geo + (long long)GEO_FLOOR * pl + z),
                __ldg(a.geo + (long long)(GEO_FLOOR + 1) * pl + z));
    atomicAdd(&a.sc->newton_iters, (unsigned long long)niter);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.sc->ndeferred_total += nd;
}

// One con-to-prim method (Utoprimgen_pick ids, step_ch.h:39-53), or the
// whole Utoprimgen with the retry chain (which = -1), at nz listed zones:
// zones (i, j) pairs, U (evolved form) and pr (guess in, result out) 8 per
// zone, pfl out.
__global__ void k_invert_zones(StepArgs a, int which, int nz, const int* __restrict__ zones, const double* __restrict__ U,
                               double* pr, int* pfl)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nz) return;
  const long long z = a.gr.at(zones[2 * k], zones[2 * k + 1]);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  double u[NPR], p[NPR], p0[NPR];
  for (int m = 0; m < NPR; m++) {
    u[m] = U[NPR * k + m];
    p[m] = p0[m] = pr[NPR * k + m];
  }
  int code;
  if (which == ta::M_2D || which < 0) {
    int niter;
    code = utoprim_2d(u, g, p, a.pp.gam, a.pp.gammafail, &niter);
    if (which < 0) code = ta::tryagain_chain(u, g, a.pp.gam, a.pp.gammafail, p0, p, code);
  } else {
    double Ug[NPR];
    ta::evolved_to_geomfree(u, g, Ug);
    code = ta::pick(which, Ug, g, a.pp.gam, a.pp.gammafail, p);
  }
  for (int m = 0; m < NPR; m++) pr[NPR * k + m] = p[m];
  pfl[k] = code;
}

// ---------------------------------------------------------------- bounds
// inflow_check_rel4vel for dir 1 at CENT, fixup.c:1733-1830: the outer x1
// end is OUTFLOW for both problems, the inner one only for the torus
__device__ __forceinline__ int inflow_check_x1(const StepArgs& a, int i, double* pr, const Geo<double>& g)
{
  double ucon[4];
  ucon_of(pr, g, ucon);
  const bool inner_outflow = (a.pp.bc == 0);
  const bool dofix = ((i <= -1) && inner_outflow && (ucon[1] > 0.)) || ((i >= a.gr.n1) && (ucon[1] < 0.));
  if (!dofix) return 0;
  double gamma = gamma_of(pr, g);
  pr[U1] /= gamma;
  pr[U2] /= gamma;
  pr[U3] /= gamma;
  const double alpha = 1. / sqrt(-g.gcon[0]);
  const double betacon = g.gcon[1] * alpha * alpha;
  pr[U1] = betacon / alpha;
  double vsq = 0.;
#pragma unroll
  for (int jj = 1; jj < 4; jj++)
#pragma unroll
    for (int kk = 1; kk < 4; kk++) vsq += g.gcov[sym(jj, kk)] * pr[U1 + jj - 1] * pr[U1 + kk - 1];
  if (vsq < 0.0) {
    if (vsq > -DBL_EPS_REF * 100.0) vsq = 0.0;
    else return FAIL_VSQ_NEG;
  }
  if (vsq >= 1.0) vsq = 1.0 - 1.0 / (a.pp.gammamax * a.pp.gammamax);
  gamma = 1. / sqrt(1. - vsq);
  pr[U1] *= gamma;
  pr[U2] *= gamma;
  pr[U3] *= gamma;
  return 0;
}

// A value of an active zone as the second bound_prim of a substep reads it
// when the repairs of fixup_utoprim are applied in the same kernel (APPLY):
// a repaired zone's rho..u~3 come from the repair buffer (the zone's own
// thread writes them to pv in that kernel), everything else from pv.
// Repaired = a failed inversion or a check-solution decision (the zones
// k_fixup_compute wrote), or PF_FIXED once the zone's thread has marked it.
template <bool APPLY>
__device__ __forceinline__ double srcv(const StepArgs& a, const double* pv, long long zs, int k)
{
  const long long pl = a.gr.plane;
  if (APPLY && k <= U3) {
    if (a.pflag[zs] != 0 || a.chk[zs] != 0) return a.fixbuf[k * pl + zs];
  }
  return pv[k * pl + zs];
}

// x1 ghost zone (i, j) of the rotating star, bounds.ns.c:96-203 (NSSURFACE)
// and 207-271 (OUTFLOW), EXTRAP 1: densities scaled by sqrt(-g); inside, the
// velocity of the surface rotating at omegastar (vcon2pr -> ucon_calc_3vel;
// left as it was if that fails) and the field of the step's p; outside,
// linear extrapolation factors in x1
template <bool APPLY>
__device__ __forceinline__ void x1_ghost_star(const StepArgs& a, const double* pv, int i, int j, double* pr)
{
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const int ri = (i < 0) ? 0 : a.gr.n1 - 1;
  const long long zr = a.gr.at(ri, j);
  const double gr_ = gdet_at(a, CENT, zr), gi = gdet_at(a, CENT, z);
#pragma unroll
  for (int k = RHO; k <= UU; k++) pr[k] = srcv<APPLY>(a, pv, zr, k) * gr_ / gi;
  if (i < 0) {
    Geo<double> g;
    load_geo(a, CENT, z, g);
    const double vcon[4] = {0., 0., 0., a.pp.omegastar};
    double ucon[4];
    if (!ucon_3vel(vcon, g.gcov, ucon)) {
      pr[U1] = ucon[1];
      pr[U2] = ucon[2];
      pr[U3] = ucon[3];
    } else {
#pragma unroll
      for (int k = U1; k <= U3; k++) pr[k] = pv[k * pl + z];
    }
#pragma unroll
    for (int k = B1; k <= B3; k++) pr[k] = a.pstep[k * pl + z];
  } else {
    const double dx1 = a.pp.dx1;
    pr[U1] = srcv<APPLY>(a, pv, zr, U1) * (1. - 2 * (i - ri) * dx1);
#pragma unroll
    for (int k = U2; k <= U3; k++) pr[k] = srcv<APPLY>(a, pv, zr, k) * (1. - (i - ri) * dx1);
    pr[B1] = pv[B1 * pl + zr] * gr_ / gi;
#pragma unroll
    for (int k = B2; k <= B3; k++) pr[k] = pv[k * pl + zr] * (1. - (i - ri) * dx1);
  }
}

// outflow copy + inflow check + gamma limit of an x1 ghost zone (i, j),
// bounds.fishmon.c:28-60 and 192-230 (EXTRAP 0), or the star's
template <bool APPLY>
__device__ __forceinline__ void x1_ghost(const StepArgs& a, const double* pv, int i, int j, double* pr, int phase)
{
  if (a.pp.bc == 1) {
    x1_ghost_star<APPLY>(a, pv, i, j, pr);
  } else {
    const int is = (i < 0) ? 0 : a.gr.n1 - 1;
    const long long zs = a.gr.at(is, j);
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = srcv<APPLY>(a, pv, zs, k);
  }
  Geo<double> g;
  load_geo(a, CENT, a.gr.at(i, j), g);
  int rc = inflow_check_x1(a, i, pr, g);
  if (!rc) rc = limit_gamma(a.pp.gammamax, pr, g);
  if (rc) report_fail(a.sc, phase, rc, bound_order(a.gr.n1, a.gr.n2, i, j));
}

// bound_prim (bounds.fishmon.c:14-330 or bounds.ns.c:10-355) and
// bound_pflag (boundsint.c:4-60) for every ghost zone; reads only active
// zones, writes only ghost zones.  Polar ghosts of the x1 ghost columns take
// the x1 ghost value of their mirror row, as the reference's x1-then-x2 order
// produces.  The torus's POLEDEATH rows are zeroed here for ghost zones and
// by k_poledeath for the first and last active rows.
template <bool APPLY>
__device__ __forceinline__ void bound_ghost(const StepArgs& a, double* pv, int i, int j, int with_pflag)
{
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  const bool xin = (i >= 0 && i < n1), yin = (j >= 0 && j < n2);
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  double pr[NPR];
  const bool poledeath = (a.pp.bc == 0);
  const int phase = a.phase0 + (with_pflag ? PH_BOUND1 : PH_BOUND2);
  if (yin) {
    x1_ghost<APPLY>(a, pv, i, j, pr, phase);
    if (poledeath && (j == 0 || j == n2 - 1)) {
      pr[U2] *= 0.;
      pr[B2] *= 0.;
    }
  } else {
    const int jm = (j < 0) ? (-j - 1) : (2 * n2 - 1 - j);
    if (xin) {
      const long long zs = a.gr.at(i, jm);
#pragma unroll
      for (int k = 0; k < NPR; k++) pr[k] = srcv<APPLY>(a, pv, zs, k);
    } else {
      x1_ghost<APPLY>(a, pv, i, jm, pr, phase);
    }
    if (poledeath) {
      pr[U2] *= 0.;
      pr[B2] *= 0.;
    }
  }
#pragma unroll
  for (int k = 0; k < NPR; k++) pv[k * pl + z] = pr[k];
  if (with_pflag) {
    const int is = (i < 0) ? 0 : ((i >= n1) ? n1 - 1 : i);
    const int js = (j < 0) ? (-j - 1) : ((j >= n2) ? (2 * n2 - 1 - j) : j);
    a.pflag[z] = a.pflag[a.gr.at(is, js)];
  }
}

__global__ void k_bound(StepArgs a, double* pv, int with_pflag)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - NG;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - NG;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i >= n1 + NG || j >= n2 + NG) return;
  if (i >= 0 && i < n1 && j >= 0 && j < n2) return;
  bound_ghost<false>(a, pv, i, j, with_pflag);
}

// The end of a GRMHD substep in one kernel: fixup_utoprim's repairs applied
// (the zones k_fixup_compute repaired take their rho..u~3 from the repair
// buffer and are flagged PF_FIXED, fixup.c:527-928), the second bound_prim
// (bounds.fishmon.c:14-330; the ghost zones read a repaired zone's values
// from the repair buffer, so they see the repaired state whichever thread
// runs first) and its POLEDEATH zeroing of u~2 and B2 on the first and last
// active rows (bounds.fishmon.c:296-327).  The zeroing comes after the
// ghosts have read those rows in the reference: a zone there that was not
// repaired holds u~2 = B2 = 0 already (the first bound zeroed them and
// nothing changed them since), so the ghosts read the same value before or
// after it is rewritten; a repaired one is read from the repair buffer.
//
// With step_end set (after the last substep) the grid starts with `hrows`
// extra rows of blocks (launched first, so that their latency overlaps the
// zones' work): their threads form the horizon terms of rows j from the
// final state of zone (0, j) -- the value its own thread writes in this
// kernel: the repair buffer's or pv's, times 0 for u~2 and B2 on the
// POLEDEATH rows (x * 0 of a value already zeroed is the same zero) -- into
// ubuf, and the last block to finish runs step_end_finish (the blocks count
// themselves in sc->blocks_done).
__device__ __forceinline__ void bound_fix_zone(const StepArgs& a, double* pv, int i, int j)
{
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i >= n1 + NG || j >= n2 + NG) return;
  if (i >= 0 && i < n1 && j >= 0 && j < n2) {
    const long long pl = a.gr.plane, z = a.gr.at(i, j);
    const int f = a.pflag[z];
    const int c = a.chk[z];
    if (f != 0 || c != 0) {
#pragma unroll
      for (int k = 0; k <= U3; k++) pv[k * pl + z] = a.fixbuf[k * pl + z];
      a.pflag[z] = PF_FIXED;
      atomicAdd(&a.sc->fixups, 1);
    }
    if (a.pp.bc == 0 && (j == 0 || j == n2 - 1)) {
      pv[U2 * pl + z] *= 0.;
      pv[B2 * pl + z] *= 0.;
    }
    return;
  }
  bound_ghost<true>(a, pv, i, j, 0);
}

template <typename FT>
__global__ void k_bound_fix(StepArgs a, double* pv, int step_end, int hrows)
{
  if ((int)blockIdx.y >= hrows) {
    bound_fix_zone(a, pv, blockIdx.x * blockDim.x + threadIdx.x - NG,
                   (blockIdx.y - hrows) * blockDim.y + threadIdx.y - NG);
  } else {
    const int nt = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int j = (blockIdx.y * gridDim.x + blockIdx.x) * nt + tid;
    if (j < a.gr.n2) {
      const long long pl = a.gr.plane, z = a.gr.at(0, j);
      double pr[NPR], t4[4];
#pragma unroll
      for (int k = 0; k < NPR; k++) pr[k] = srcv<true>(a, pv, z, k);
      if (a.pp.bc == 0 && (j == 0 || j == a.gr.n2 - 1)) {
        pr[U2] *= 0.;
        pr[B2] *= 0.;
      }
      horizon_terms<FT>(a, pr, j, t4);
#pragma unroll
      for (int k = 0; k < 4; k++) a.ubuf[k * pl + j] = t4[k];
    }
  }
  if (!step_end) return;
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    __threadfence();
    const unsigned nb = gridDim.x * gridDim.y;
    last = (atomicAdd(&a.sc->blocks_done, 1u) == nb - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  step_end_finish<true>(a, a.ubuf, a.gr.plane);
  if (threadIdx.x == 0 && threadIdx.y == 0) a.sc->blocks_done = 0;
}

void launch_bound_fix(int mixed, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, double* pv, int step_end)
{
  const int hrows = step_end ? (a.gr.n2 + g.x * b.x * b.y - 1) / (g.x * b.x * b.y) : 0;
  g.y += hrows;
  if (mixed) k_bound_fix<float><<<g, b, 0, s>>>(a, pv, step_end, hrows);
  else k_bound_fix<double><<<g, b, 0, s>>>(a, pv, step_end, hrows);
}

// POLEDEATH on the first and last active x2 rows (bounds.fishmon.c:296-327)
__global__ void k_poledeath(StepArgs a, double* pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.gr.n1) return;
  const int j = (blockIdx.y == 0) ? 0 : a.gr.n2 - 1;
  const long long z = a.gr.at(i, j);
  pv[U2 * a.gr.plane + z] *= 0.;
  pv[B2 * a.gr.plane + z] *= 0.;
}

// ---------------------------------------------------------------- check solution
// fixup_checksolution, fixup.c:388-488.  gammacheck first (DQZLOOP range).
// With poledeath set, each thread of the first or last active row first
// applies the POLEDEATH zeroing of k_poledeath to its own zone (the bound
// before this kernel has read those rows already; this kernel reads only
// its own zone).
// The first bound of a GRMHD substep with the gamma table of the check-
// solution vote in one kernel: ghost zones are filled (bound_prim +
// bound_pflag) and those of the one-zone ring set their gamma from the value
// just formed; active zones of the DQZLOOP range set theirs from pv, with
// the POLEDEATH zeroing of u~2 and B2 on the first and last rows applied to
// the copy only -- the ghosts read those rows before the zeroing, as the
// reference's bound does, so k_checksol writes it to pv (it reads only u of
// its neighbours).
__device__ __forceinline__ void gammacheck_set(const StepArgs& a, long long z, const double* pr)
{
  if (a.bsqf[z] == 0 || a.pflag[z] != 0) return;
  Geo<double> g;
  load_geo(a, CENT, z, g);
  a.gammacheck[z] = gamma_of(pr, g);
}

__global__ void k_bound_gc(StepArgs a, double* pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - NG;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - NG;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) a.sc->nchk = 0;
  if (i >= n1 + NG || j >= n2 + NG) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const bool ring = i >= -1 && i <= n1 && j >= -1 && j <= n2;
  if (i >= 0 && i < n1 && j >= 0 && j < n2) {
    double pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = pv[k * pl + z];
    if (a.pp.bc == 0 && (j == 0 || j == n2 - 1)) {
      pr[U2] *= 0.;
      pr[B2] *= 0.;
    }
    gammacheck_set(a, z, pr);
    return;
  }
  bound_ghost<false>(a, pv, i, j, 1);
  if (ring) {
    double pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = pv[k * pl + z];
    gammacheck_set(a, z, pr);
  }
}

__global__ void k_gammacheck(StepArgs a, double* __restrict__ pv, int poledeath)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) a.sc->nchk = 0;
  if (i > a.gr.n1 || j > a.gr.n2) return;
  const long long z = a.gr.at(i, j);
  if (poledeath && i >= 0 && i < a.gr.n1 && (j == 0 || j == a.gr.n2 - 1)) {
    pv[U2 * a.gr.plane + z] *= 0.;
    pv[B2 * a.gr.plane + z] *= 0.;
  }
  if (a.bsqf[z] == 0 || a.pflag[z] != 0) return;
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = pv[k * a.gr.plane + z];
  Geo<double> g;
  load_geo(a, CENT, z, g);
  a.gammacheck[z] = gamma_of(pr, g);
}

// The check-solution vote of candidate zone (i, j) (fixup.c:402-482).  The
// reference sweeps zones in ZLOOP order (i outer, j inner) and a zone it
// flags is seen as failed by the zones after it: with `prev` given, an
// earlier active neighbour whose decision there is nonzero counts as failed;
// without, as the pflag says alone.  The neighbour list and the vote keep the
// reference's form (its list names (+1, +1) twice and not (-1, +1); every
// vote is gated on the first neighbour's ratio).
__device__ __forceinline__ unsigned char checksol_vote(const StepArgs& a, const double* __restrict__ pv, int i, int j,
                                                       long long z, const unsigned char* prev)
{
  const long long pl = a.gr.plane;
  const int di[8] = {0, 0, 1, -1, 1, 1, 1, -1};
  const int dj[8] = {1, -1, 0, 0, 1, -1, 1, -1};
  const double g0 = a.gammacheck[z], u0 = pv[UU * pl + z];
  double pd[8], pd2[8];
#pragma unroll
  for (int l = 0; l < 8; l++) {
    const int ii = i + di[l], jj = j + dj[l];
    const long long zz = a.gr.at(ii, jj);
    bool ok = (a.pflag[zz] == 0);
    const bool earlier = (ii < i) || (ii == i && jj < j);
    if (ok && prev && earlier && ii >= 0 && ii < a.gr.n1 && jj >= 0 && jj < a.gr.n2 && prev[zz] != 0) ok = false;
    pd[l] = ok ? (a.gammacheck[zz] / g0) : -1;
    pd2[l] = ok ? (pv[UU * pl + zz] / u0) : -1;
  }
  int v0 = 0, v1 = 0, nv = 0;
#pragma unroll
  for (int l = 0; l < 8; l++) {
    if (pd[0] >= 0.0) {
      if ((fabs(pd[l]) > 2.0) || (fabs(pd[l]) < 1.0 / 2.0)) v0++;
      if ((fabs(pd2[l]) > 10.0) || (fabs(pd2[l]) < 1.0 / 10.0)) v1++;
      nv++;
    }
  }
  unsigned char d = 0;
  if (v0 > nv * 0.5) d = PF_GAMMAPERC;
  if (v1 > nv * 0.5) d = PF_UPERC;
  return d;
}

__device__ __forceinline__ bool checksol_candidate(const StepArgs& a, int i, int j)
{
  if (i < 0 || i >= a.gr.n1 || j < 0 || j >= a.gr.n2) return false;
  const long long z = a.gr.at(i, j);
  return a.bsqf[z] != 0 && a.pflag[z] == 0;
}

// Round 0 of the sweep: every candidate voted as if no earlier zone were
// flagged, into decision plane 0.  A vote can only lose counts when an
// earlier neighbour is flagged (a failed neighbour's ratio of -1 counts no
// vote), so the sweep's flagged set is a subset of round 0's, and only a
// zone flagged here that has an earlier candidate neighbour (of its list:
// (i, j-1), (i-1, j), (i-1, j-1)) can end differently: those go to the
// worklist (the deferred-inversion list, idle by now) for k_checksol_rounds.
// With poledeath set (after k_bound_gc) the thread of a zone on the first or
// last row applies the POLEDEATH zeroing of u~2 and B2 to pv first.
__global__ void k_checksol(StepArgs a, double* __restrict__ pv, int poledeath)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.gr.n1 || j >= a.gr.n2) return;
  const long long z = a.gr.at(i, j);
  if (poledeath && (j == 0 || j == a.gr.n2 - 1)) {
    pv[U2 * a.gr.plane + z] *= 0.;
    pv[B2 * a.gr.plane + z] *= 0.;
  }
  if (a.bsqf[z] == 0 || a.pflag[z] != 0) {
    a.chk[z] = 0;
    return;
  }
  const unsigned char d = checksol_vote(a, pv, i, j, z, nullptr);
  a.chk[z] = d;
  if (d != 0 && (checksol_candidate(a, i, j - 1) || checksol_candidate(a, i - 1, j) ||
                 checksol_candidate(a, i - 1, j - 1)))
    a.worklist[atomicAdd(&a.sc->nchk, 1)] = (int)z;
}

// The rest of the sweep, one block: the worklist zones re-vote from the
// previous round's decisions of their earlier neighbours (plane 0), new
// decisions staged in plane 1 (indexed by worklist slot) and copied back,
// until a round changes nothing.  The earlier-than relation is acyclic, so
// these rounds reach the sweep's unique fixed point within (longest chain of
// worklist zones + 1) rounds; after CHK_MAX_ROUNDS without it (never seen)
// thread 0 runs the reference's sweep itself over every zone.
constexpr int CHK_MAX_ROUNDS = 64;
__global__ void __launch_bounds__(1024) k_checksol_rounds(StepArgs a, const double* __restrict__ pv)
{
  const int nw = a.sc->nchk;
  if (nw == 0) return;
  if (threadIdx.x == 0) a.sc->chk_multi++;
  unsigned char* d0 = a.chk;
  unsigned char* dn = a.chk + a.gr.plane;
  __shared__ int changed;
  bool settled = false;
  for (int r = 1; r <= CHK_MAX_ROUNDS; r++) {
    if (threadIdx.x == 0) changed = 0;
    __syncthreads();
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
      const long long z = a.worklist[w];
      const int i = (int)(z % a.gr.pitch) - NG, j = (int)(z / a.gr.pitch) - NG;
      const unsigned char d = checksol_vote(a, pv, i, j, z, d0);
      dn[w] = d;
      if (d != d0[z]) changed = 1;
    }
    __syncthreads();
    if (!changed) {
      settled = true;
      break;
    }
    for (int w = threadIdx.x; w < nw; w += blockDim.x) d0[a.worklist[w]] = dn[w];
    __syncthreads();
  }
  if (settled || threadIdx.x != 0) return;
  for (int i = 0; i < a.gr.n1; i++)
    for (int j = 0; j < a.gr.n2; j++) {
      const long long z = a.gr.at(i, j);
      d0[z] = 0;
      if (a.bsqf[z] == 0 || a.pflag[z] != 0) continue;
      d0[z] = checksol_vote(a, pv, i, j, z, d0);
    }
}

// ---------------------------------------------------------------- fixup_utoprim
// fixup.c:527-928 (UTOPRIMAVG, NOGOODAVERAGE): repaired values from the
// unmodified neighbours (the reference's prc snapshot), written to fixbuf.
__global__ void k_fixup_compute(StepArgs a, const double* __restrict__ pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.gr.n1 || j >= a.gr.n2) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const unsigned char* chk = a.chk;
  int f = a.pflag[z];
  if (f == 0) f = chk[z];
  if (f == 0) return;
  // neighbour goodness with the check-solution decisions applied
  auto good = [&](int ii, int jj) -> bool {
    const long long zz = a.gr.at(ii, jj);
    if (a.pflag[zz] != 0) return false;
    if (ii >= 0 && ii < a.gr.n1 && jj >= 0 && jj < a.gr.n2 && chk[zz] != 0) return false;
    return true;
  };
  auto P = [&](int ii, int jj, int k) -> double { return pv[k * pl + a.gr.at(ii, jj)]; };
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = pv[k * pl + z];
  Geo<double> g;
  load_geo(a, CENT, z, g);
  double gamma = gamma_of(pr, g);
  if (gamma > a.pp.gammamax) gamma = a.pp.gammamax;
  // neighbour set (recorded for the adjoint): 0 the four faces, 1 the four
  // corners, 2 x2 pair, 3 x1 pair, 4 and 5 the diagonal pairs, 6 + m the
  // first good single neighbour m, 14 the all-neighbour fallback
  int set;
  if (good(i, j + 1) && good(i, j - 1) && good(i + 1, j) && good(i - 1, j)) {
    set = 0;
    for (int k = 0; k <= U3; k++) pr[k] = 0.25 * (P(i, j + 1, k) + P(i, j - 1, k) + P(i - 1, j, k) + P(i + 1, j, k));
  } else if (good(i + 1, j + 1) && good(i + 1, j - 1) && good(i - 1, j + 1) && good(i - 1, j - 1)) {
    set = 1;
    for (int k = 0; k <= U3; k++) pr[k] = 0.25 * (P(i + 1, j + 1, k) + P(i + 1, j - 1, k) + P(i - 1, j + 1, k) + P(i - 1, j - 1, k));
  } else if (good(i, j + 1) && good(i, j - 1)) {
    set = 2;
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i, j + 1, k) + P(i, j - 1, k));
  } else if (good(i + 1, j) && good(i - 1, j)) {
    set = 3;
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i + 1, j, k) + P(i - 1, j, k));
  } else if (good(i + 1, j + 1) && good(i - 1, j - 1)) {
    set = 4;
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i + 1, j + 1, k) + P(i - 1, j - 1, k));
  } else if (good(i + 1, j - 1) && good(i - 1, j + 1)) {
    set = 5;
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i + 1, j - 1, k) + P(i - 1, j + 1, k));
  } else {
    const int oi[8] = {1, 1, 1, 0, -1, -1, -1, 0};
    const int oj[8] = {1, 0, -1, -1, -1, 0, 1, 1};
    int m = 0;
    for (; m < 8; m++)
      if (good(i + oi[m], j + oj[m])) break;
    if (m < 8) {
      set = 6 + m;
      for (int k = 0; k <= U3; k++) pr[k] = P(i + oi[m], j + oj[m], k);
    } else {
      set = 14;
      for (int k = 0; k <= U3; k++)
        pr[k] = 0.5 * (0.25 * (P(i, j + 1, k) + P(i, j - 1, k) + P(i - 1, j, k) + P(i + 1, j, k)) +
                       0.25 * (P(i + 1, j + 1, k) + P(i + 1, j - 1, k) + P(i - 1, j + 1, k) + P(i - 1, j - 1, k)));
    }
  }
  if (a.rec_fixset) a.rec_fixset[z] = (unsigned char)set;
  int rc = limit_gamma(gamma, pr, g);
  if (rc) report_fail(a.sc, a.phase0 + PH_FIXUP, rc, zone_order(i, j));
#pragma unroll
  for (int k = 0; k <= U3; k++) a.fixbuf[k * pl + z] = pr[k];
}

__global__ void k_fixup_apply(StepArgs a, double* pv, int grmhd)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.gr.n1 || j >= a.gr.n2) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  int f = a.pflag[z];
  const int c = a.chk[z];
  if (f == 0 && c != 0) f = c;
  if (f == 0) return;
  if (grmhd) {
#pragma unroll
    for (int k = 0; k <= U3; k++) pv[k * pl + z] = a.fixbuf[k * pl + z];
    a.pflag[z] = PF_FIXED;
    atomicAdd(&a.sc->fixups, 1);
  } else {
    a.pflag[z] = f;
  }
}

// ---------------------------------------------------------------- currents
// current_doprecalc(0..3, p) with WHICHCURRENTCALC 1 (phys.c:1124-1218): at
// every zone centre (ghosts included) the F^{i t} components go to the next
// level of a three-level ring (the reference shifts slot 0 -> 4 -> 3), F^{i r}
// and F^{i h} to their slots, and the six F^{mu nu} to fcon.
__global__ void k_faraday(StepArgs a, const double* __restrict__ pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - NG;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - NG;
  if (i >= a.gr.n1 + NG || j >= a.gr.n2 + NG) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = __ldg(pv + k * pl + z);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  State<double> q;
  state_of(pr, g, q);
  const double* b = q.bcov;
  const double* u = q.ucov;
  double* c = a.cur + z;
  const int lv = (a.sc->cur_ring + 1) % 3;
  c[(CUR_RING + 3 * lv + 0) * pl] = -1.0 / g.g * (-b[3] * u[2] + b[2] * u[3]);
  c[(CUR_RING + 3 * lv + 1) * pl] = -1.0 / g.g * (b[3] * u[1] - b[1] * u[3]);
  c[(CUR_RING + 3 * lv + 2) * pl] = -1.0 / g.g * (-b[2] * u[1] + b[1] * u[2]);
  c[(CUR_S1 + 0) * pl] = -1.0 / g.g * (b[3] * u[2] - b[2] * u[3]);
  c[(CUR_S1 + 1) * pl] = -1.0 / g.g * (-b[3] * u[0] + b[0] * u[3]);
  c[(CUR_S1 + 2) * pl] = -1.0 / g.g * (b[2] * u[0] - b[0] * u[2]);
  c[(CUR_S2 + 0) * pl] = -1.0 / g.g * (-b[3] * u[1] + b[1] * u[3]);
  c[(CUR_S2 + 1) * pl] = -1.0 / g.g * (b[3] * u[0] - b[0] * u[3]);
  c[(CUR_S2 + 2) * pl] = -1.0 / g.g * (-b[1] * u[0] + b[0] * u[1]);
  c[(CUR_FCON + 0) * pl] = -1.0 / g.g * (b[3] * u[2] - b[2] * u[3]);
  c[(CUR_FCON + 1) * pl] = -1.0 / g.g * (-b[3] * u[1] + b[1] * u[3]);
  c[(CUR_FCON + 2) * pl] = -1.0 / g.g * (b[2] * u[1] - b[1] * u[2]);
  c[(CUR_FCON + 3) * pl] = -1.0 / g.g * (b[3] * u[0] - b[0] * u[3]);
  c[(CUR_FCON + 4) * pl] = -1.0 / g.g * (-b[2] * u[0] + b[0] * u[2]);
  c[(CUR_FCON + 5) * pl] = -1.0 / g.g * (b[1] * u[0] - b[0] * u[1]);
}

// current_calc_1, phys.c:1335-1455, over i in [-2, N1+2), j in [-2, N2+2):
// J^mu = (1/g) d_nu (g F^{mu nu}) with centred space differences and, from the
// third call on, the one-sided second-order time derivative through the three
// ring levels (dt of this step and of the previous call).  J^h's x1 difference
// takes g at i-1 from the zone itself, as the reference's geomr does.
__global__ void k_current(StepArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - (NG - 1);
  const int j = blockIdx.y * blockDim.y + threadIdx.y - (NG - 1);
  if (i >= a.gr.n1 + NG - 1 || j >= a.gr.n2 + NG - 1) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const long long zrp = a.gr.at(i + 1, j), zrm = a.gr.at(i - 1, j), zhp = a.gr.at(i, j + 1), zhm = a.gr.at(i, j - 1);
  const DevScalars* sc = a.sc;
  const int ln = (sc->cur_ring + 1) % 3, l0 = sc->cur_ring, l3 = (sc->cur_ring + 2) % 3;
  const double dtl = sc->clastdt, dtr = sc->dt;
  const double idx1 = 1.0 / (2.0 * a.pp.dx1), idx2 = 1.0 / (2.0 * a.pp.dx2);
  const double gt = gdet_at(a, CENT, z), grp = gdet_at(a, CENT, zrp), grm = gdet_at(a, CENT, zrm);
  const double ghp = gdet_at(a, CENT, zhp), ghm = gdet_at(a, CENT, zhm);
  const double* c = a.cur;
#define S1(zz, k) c[(CUR_S1 + (k)) * pl + (zz)]
#define S2(zz, k) c[(CUR_S2 + (k)) * pl + (zz)]
  double* J = a.cur + CUR_JCON * pl + z;
  J[0] = 1. / gt * (grp * S1(zrp, 0) - grm * S1(zrm, 0)) * idx1 + 1. / gt * (ghp * S2(zhp, 0) - ghm * S2(zhm, 0)) * idx2;
  double d[3] = {0., 0., 0.};
  const bool timed = sc->ccalls >= 2;
  if (timed) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double fl = c[(CUR_RING + 3 * l3 + k) * pl + z], f0 = c[(CUR_RING + 3 * l0 + k) * pl + z];
      const double fr = c[(CUR_RING + 3 * ln + k) * pl + z];
      const double AA = (dtr * (fl - f0) + dtl * (fr - f0)) / (dtl * dtr * (dtl + dtr));
      const double BB = (-dtr * dtr * (fl - f0) + dtl * dtl * (fr - f0)) / (dtl * dtr * (dtl + dtr));
      d[k] = 2.0 * AA * dtr + BB;
    }
  }
  // the reference adds the integer 0 where there is no time derivative
  J[pl] = (timed ? d[0] : 0.) + 1. / gt * (ghp * S2(zhp, 1) - ghm * S2(zhm, 1)) * idx2;
  J[2 * pl] = (timed ? d[1] : 0.) + 1. / gt * (grp * S1(zrp, 1) - gt * S1(zrm, 1)) * idx1;
  J[3 * pl] = (timed ? d[2] : 0.) + 1. / gt * (grp * S1(zrp, 2) - grm * S1(zrm, 2)) * idx1 +
              1. / gt * (ghp * S2(zhp, 2) - ghm * S2(zhm, 2)) * idx2;
#undef S1
#undef S2
}

// the statics of current_calc_1 (calls, lastdt) and the ring's newest level
__global__ void k_currents_commit(StepArgs a)
{
  DevScalars* s = a.sc;
  s->cur_ring = (s->cur_ring + 1) % 3;
  s->ccalls += 1;
  s->clastdt = s->dt;
}

// ---------------------------------------------------------------- dumps
// The dynamic columns of dump_content, dump.c:87-191, for the active zone
// (i, j) at row j*N1 + i (DUMPLOOP order, global.h:1047): p (8), divb
// (SETFDIVBFLUXCT, global.h:1152-1180), u^mu, u_mu, b^mu, b_mu, vmin/vmax in
// x1 and x2 (vchar), sqrt(-g), J^mu, J_mu, F^{mu nu} (6), F_{mu nu} (6
// through lowerf, phys.c:655-689): DUMP_DYNCOLS values.  A vchar failure
// (the reference's FAILSTATEMENT) is counted in *nfail.
constexpr int DUMP_DYNCOLS = 50;
__global__ void k_dump_columns(StepArgs a, const double* __restrict__ pv, double* __restrict__ out, int* nfail)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i >= n1 || j >= n2) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  double* o = out + ((long long)j * n1 + i) * DUMP_DYNCOLS;
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = pv[k * pl + z];
  Geo<double> g;
  load_geo(a, CENT, z, g);
  State<double> q;
  state_of(pr, g, q);
  double vmax1, vmin1, vmax2, vmin2;
  int rc = vchar_of(pr, q, 1, g, a.pp.gam, vmax1, vmin1);
  if (!rc) rc = vchar_of(pr, q, 2, g, a.pp.gam, vmax2, vmin2);
  if (rc) {
    atomicAdd(nfail, 1);
    vmax1 = vmin1 = vmax2 = vmin2 = 0.;
  }
  // divb (FLUXCT form); 0 on the first active row and at j = N2
  double divb = 0.;
  if (j != 0 && j != n2) {
    const long long z10 = a.gr.at(i - 1, j), z01 = a.gr.at(i, j - 1), z11 = a.gr.at(i - 1, j - 1);
    const double g00 = gdet_at(a, CENT, z), g10 = gdet_at(a, CENT, z10), g01 = gdet_at(a, CENT, z01);
    const double g11 = gdet_at(a, CENT, z11);
    const double b1_00 = pv[B1 * pl + z] * g00, b1_01 = pv[B1 * pl + z01] * g01, b1_10 = pv[B1 * pl + z10] * g10;
    const double b1_11 = pv[B1 * pl + z11] * g11;
    const double b2_00 = pv[B2 * pl + z] * g00, b2_10 = pv[B2 * pl + z10] * g10, b2_01 = pv[B2 * pl + z01] * g01;
    const double b2_11 = pv[B2 * pl + z11] * g11;
    const double dx1 = a.pp.dx1, dx2 = a.pp.dx2;
    const double mx = (dx1 > dx2) ? dx1 : dx2;
    const double num = 0.5 * (b1_00 + b1_01 - b1_10 - b1_11) / dx1 + 0.5 * (b2_00 + b2_10 - b2_01 - b2_11) / dx2;
    const double den = gdet_at(a, CORN, z) * 0.125 *
                       fabs(fabs(b1_00 + b1_01 + b1_10 + b1_11 + b2_00 + b2_10 + b2_01 + b2_11) + 1.e-20);
    divb = fabs(mx * num / den);
  }
  int c = 0;
#pragma unroll
  for (int k = 0; k < NPR; k++) o[c++] = pr[k];
  o[c++] = divb;
#pragma unroll
  for (int k = 0; k < 4; k++) o[c++] = q.ucon[k];
#pragma unroll
  for (int k = 0; k < 4; k++) o[c++] = q.ucov[k];
#pragma unroll
  for (int k = 0; k < 4; k++) o[c++] = q.bcon[k];
#pragma unroll
  for (int k = 0; k < 4; k++) o[c++] = q.bcov[k];
  o[c++] = vmin1;
  o[c++] = vmax1;
  o[c++] = vmin2;
  o[c++] = vmax2;
  o[c++] = g.g;
  double jc[4], jv[4], fc[6];
#pragma unroll
  for (int k = 0; k < 4; k++) jc[k] = a.cur[(CUR_JCON + k) * pl + z];
#pragma unroll
  for (int k = 0; k < 6; k++) fc[k] = a.cur[(CUR_FCON + k) * pl + z];
  lower_v(jc, g.gcov, jv);
#pragma unroll
  for (int k = 0; k < 4; k++) o[c++] = jc[k];
#pragma unroll
  for (int k = 0; k < 4; k++) o[c++] = jv[k];
#pragma unroll
  for (int k = 0; k < 6; k++) o[c++] = fc[k];
  // lowerf: F_{jk} = sum_{jp,kp} F^{jp kp} g_{j jp} g_{k kp}, summed in the
  // reference's loop order from 0, for the six upper-triangle pairs
  double F[4][4];
  F[0][0] = F[1][1] = F[2][2] = F[3][3] = 0;
  F[0][1] = fc[0];
  F[0][2] = fc[1];
  F[0][3] = fc[2];
  F[1][2] = fc[3];
  F[1][3] = fc[4];
  F[2][3] = fc[5];
  F[1][0] = -fc[0];
  F[2][0] = -fc[1];
  F[3][0] = -fc[2];
  F[2][1] = -fc[3];
  F[3][1] = -fc[4];
  F[3][2] = -fc[5];
  const int pj[6] = {0, 0, 0, 1, 1, 2}, pk[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
  for (int m = 0; m < 6; m++) {
    double s = 0;
#pragma unroll
    for (int jp = 0; jp < 4; jp++)
#pragma unroll
      for (int kp = 0; kp < 4; kp++) s += F[jp][kp] * g.gcov[sym(pj[m], jp)] * g.gcov[sym(pk[m], kp)];
    o[c++] = s;
  }
}

// ---------------------------------------------------------------- layouts
// Reference layout (defs.h: zone (ii, jj) at ii*n2m + jj, components
// fastest) <-> the step's planes.  Threads run along the planes' fast index
// i, so every plane store is coalesced and every zone's 8 reference-layout
// values are one contiguous 64 B read (or write).
__global__ void k_ref_to_planes(StepArgs a, const double* __restrict__ ref, const int* __restrict__ refflag,
                                double* __restrict__ pv)
{
  const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int n1m = a.gr.n1 + 2 * NG, n2m = a.gr.n2 + 2 * NG;
  if (ii >= n1m || jj >= n2m) return;
  const long long zr = (long long)ii * n2m + jj, zd = (long long)jj * a.gr.pitch + ii;
  const double2* src = reinterpret_cast<const double2*>(ref + zr * NPR);
#pragma unroll
  for (int k = 0; k < NPR / 2; k++) {
    const double2 v = __ldg(src + k);
    pv[(2 * k) * a.gr.plane + zd] = v.x;
    pv[(2 * k + 1) * a.gr.plane + zd] = v.y;
  }
  if (refflag) a.pflag[zd] = __ldg(refflag + zr * 5);
}

__global__ void k_planes_to_ref(StepArgs a, const double* __restrict__ pv, double* __restrict__ ref, int* __restrict__ refflag)
{
  const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int n1m = a.gr.n1 + 2 * NG, n2m = a.gr.n2 + 2 * NG;
  if (ii >= n1m || jj >= n2m) return;
  const long long zr = (long long)ii * n2m + jj, zd = (long long)jj * a.gr.pitch + ii;
  double2* dst = reinterpret_cast<double2*>(ref + zr * NPR);
#pragma unroll
  for (int k = 0; k < NPR / 2; k++) dst[k] = make_double2(pv[(2 * k) * a.gr.plane + zd], pv[(2 * k + 1) * a.gr.plane + zd]);
  if (refflag) {
    const unsigned char b = a.bsqf[zd];
    int* f = refflag + zr * 5;
    f[0] = a.pflag[zd];
    f[1] = 0;
    f[2] = b & 3;
    f[3] = (b >> 2) & 3;
    // FLAGREALFLUX where get_bsqflags sets it (the DQZLOOP range)
    const int i = ii - NG, j = jj - NG;
    f[4] = (a.fluxf && i >= -1 && i <= a.gr.n1 && j >= -1 && j <= a.gr.n2) ? (int)a.fluxf[zd] : 0;
  }
}

// launchers of the templated kernels: the FP64 instantiations here, the
// mixed-precision ones in harm_step_mixed.cu

void launch_flux(int para, int mixed, int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a,
                 const CUtensorMap& prim_map)
{
  if (mixed) launch_flux_mixed(para, ffde, g, b, s, a, prim_map);
  else if (ffde) {
    if (para) flux_rows_launch<double, true, true>(g, b, s, a, prim_map);
    else flux_rows_launch<double, false, true>(g, b, s, a, prim_map);
  } else if (para) flux_rows_launch<double, true, false>(g, b, s, a, prim_map);
  else flux_rows_launch<double, false, false>(g, b, s, a, prim_map);
}

void launch_emf(int mixed, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const double* pv)
{
  if (mixed) launch_emf_mixed(g, b, s, a, pv);
  else k_emf<double><<<g, b, 0, s>>>(a, pv);
}

void launch_update(int mixed, int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map,
                   const double* pi, const double* pb, double* pf, double c2)
{
  if (mixed) launch_update_mixed(ffde, g, b, s, a, map, pi, pb, pf, c2);
  else if (ffde) update_launch<double, true>(g, b, s, a, map, pi, pb, pf, c2);
  else update_launch<double, false>(g, b, s, a, map, pi, pb, pf, c2);
  if (!ffde) {
    if (a.pp.tryagain) k_update_tail<true><<<148, 64, 0, s>>>(a, pi, pf);
    else k_update_tail<false><<<148, 64, 0, s>>>(a, pi, pf);
  }
}

// both instances here: the horizon sums and the new dt are FP64 work built
// without contraction in either precision
void launch_step_end(int mixed, cudaStream_t s, const StepArgs& a, const double* pv)
{
  if (mixed) k_step_end<float><<<1, STEP_END_THREADS, 0, s>>>(a, pv);
  else k_step_end<double><<<1, STEP_END_THREADS, 0, s>>>(a, pv);
}

}  // namespace harm
