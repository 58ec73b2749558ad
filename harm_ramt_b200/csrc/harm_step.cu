// HARM finite-volume step on sm_100a: the kernels of one RK2 substep.
//
// Substep pipeline (reference step_ch.c:79-136 for one timeorder):
//   k_flux         fluxcalc x1 and x2 faces + fix_flux + per-block dt minima
//   k_emf          flux_ct corner EMFs (Toth, CORNGDETVERSION 1)
//   k_update       advance_standard zone loop: U(pi), geometric source(pb),
//                  flux divergence with the CT-rewritten B fluxes, RK combine,
//                  2D Newton con-to-prim, fixup1zone
//   k_bound        bound_prim + bound_pflag (ghost zones only)
//   k_poledeath    the POLEDEATH zeroing of the first/last active x2 rows
//   k_gammacheck,
//   k_checksol     fixup_checksolution (parallel fixed-point sweep, exact)
//   k_fixup_*      fixup_utoprim from a snapshot
//   k_bound/k_poledeath again, and k_dt_finalize after the last substep.
#include <cuda_runtime.h>
#include "harm_kernels.cuh"

namespace harm {

// ---------------------------------------------------------------- flags
// get_bsqflags, fixup.c:1197-1295 over the DQZLOOP range [-1,N1]x[-1,N2]
__global__ void k_bsqflags(StepArgs a, const double* __restrict__ pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
  if (i > a.gr.n1 || j > a.gr.n2) return;
  const long long z = a.gr.at(i, j);
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = __ldg(pv + k * a.gr.plane + z);
  Geo<double> g;
  load_geo(a, CENT, z, g);
  State<double> q;
  state_of(pr, g, q);
  double bsq = dot4(q.bcon, q.bcov);
  int f0, f3;
  if (bsq / pr[RHO] > a.pp.bsqorholimit) f0 = 2;
  else if (bsq / pr[RHO] > 0.9 * a.pp.bsqorholimit) f0 = 1;
  else f0 = 0;
  if (bsq / pr[UU] > a.pp.bsqoulimit) f3 = 2;
  else if (bsq / pr[UU] > 0.9 * a.pp.bsqoulimit) f3 = 1;
  else f3 = 0;
  a.bsqf[z] = (unsigned char)(f0 | (f3 << 2));
}

// ---------------------------------------------------------------- fluxes
// Interface states of zone (i, j) along `dir` (step_ch.c:812-823 slopes and
// 893-904 interface values): L = the zone's left-face value (p_r of face i),
// R = its right-face value (p_l of face i+1).
template <typename T, bool PARA>
__device__ __forceinline__ void zone_states(const StepArgs& a, const double* __restrict__ pb, int i, int j, int dir,
                                            T* L, T* R)
{
  const long long s = (dir == 1) ? 1LL : (long long)a.gr.pitch;
  const long long z = a.gr.at(i, j);
#pragma unroll
  for (int k = 0; k < NPR; k++) {
    const double* pk = pb + k * a.gr.plane + z;
    if (!PARA) {
      T ym1 = (T)__ldg(pk - s), y0 = (T)__ldg(pk), yp1 = (T)__ldg(pk + s);
      T dq = mc_slope(ym1, y0, yp1);
      L[k] = y0 - T(0.5) * dq;
      R[k] = y0 + T(0.5) * dq;
    } else {
      T l, r;
      para4((T)__ldg(pk - 2 * s), (T)__ldg(pk - s), (T)__ldg(pk), (T)__ldg(pk + s), (T)__ldg(pk + 2 * s), l, r);
      L[k] = l;
      R[k] = r;
    }
  }
}

// Flux through one face from its two interface states (the rest of the
// fluxcalc face loop, step_ch.c:944-1065).
template <typename T, bool FFDE>
__device__ __forceinline__ void face_flux(const StepArgs& a, int i, int j, int dir, T* p_l, T* p_r, double* Fo,
                                          double& dtij)
{
  const long long z = a.gr.at(i, j);
  Geo<T> g;
  load_geo(a, dir == 1 ? FACE1 : FACE2, z, g);
  // B^dir continuity (BDIRCONT, step_ch.c:944-947)
  const int bd = B1 + dir - 1;
  p_l[bd] = p_r[bd] = T(0.5) * (p_l[bd] + p_r[bd]);
  const T gmax = (T)a.pp.gammamax, gam = (T)a.pp.gam;
  int rc = limit_gamma(gmax, p_l, g);
  if (!rc) rc = limit_gamma(gmax, p_r, g);
  State<T> ql, qr;
  state_of(p_l, g, ql);
  state_of(p_r, g, qr);
  T F_l[NPR], F_r[NPR], U_l[NPR], U_r[NPR];
  flux_of<T, FFDE>(p_l, ql, dir, g, gam, F_l);
  flux_of<T, FFDE>(p_r, qr, dir, g, gam, F_r);
  flux_of<T, FFDE>(p_l, ql, 0, g, gam, U_l);
  flux_of<T, FFDE>(p_r, qr, 0, g, gam, U_r);
  T cmax_l, cmin_l, cmax_r, cmin_r;
  if (!rc) rc = vchar_of(p_l, ql, dir, g, gam, cmax_l, cmin_l);
  if (!rc) rc = vchar_of(p_r, qr, dir, g, gam, cmax_r, cmin_r);
  if (rc) {
    report_fail(a.sc, rc, i, j);
    cmax_l = cmin_l = cmax_r = cmin_r = T(0.);
  }
  // cminmax_calc, step_ch.c:1095-1148
  T lmin = rmin(cmin_l, cmin_r), lmax = rmax(cmax_l, cmax_r);
  lmin = fabs(rmax(T(0.), -lmin));
  lmax = fabs(rmax(T(0.), lmax));
  T cmin = lmin, cmax = lmax, ctop = rmax(lmax, lmin);
  const T hllfrac = (a.pp.fluxmethod == 1) ? T(1.0) : T(0.0);
  const T laxffrac = (a.pp.fluxmethod == 1) ? T(0.0) : T(1.0);
  if (cmax + cmin != T(0.0)) {
#pragma unroll
    for (int k = 0; k < NPR; k++)
      Fo[k] = (double)(hllfrac * ((cmax * F_l[k] + cmin * F_r[k] - cmax * cmin * (U_r[k] - U_l[k])) / (cmax + cmin)) +
                       laxffrac * (T(0.5) * (F_l[k] + F_r[k] - ctop * (U_r[k] - U_l[k]))));
  } else {
#pragma unroll
    for (int k = 0; k < NPR; k++) Fo[k] = (double)(T(0.5) * (F_l[k] + F_r[k] - ctop * (U_r[k] - U_l[k])));
  }
  // face Courant limit, step_ch.c:1062-1065 (kept in FP64)
  double cm = (double)rmax(cmax, cmin);
  dtij = a.pp.cour * (dir == 1 ? a.pp.dx1 : a.pp.dx2) / cm;
}

__device__ __forceinline__ double block_min(double v, double* sh)
{
  // exact minimum (no rounding), NaN-ignoring like `if (x < m) m = x`
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_down_sync(0xffffffffu, v, o);
    v = (w < v) ? w : v;
  }
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31, warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
  if (warp == 0) {
    v = (lane < nw) ? sh[lane] : 1.e9;
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_down_sync(0xffffffffu, v, o);
      v = (w < v) ? w : v;
    }
  }
  return v;
}

// fluxcalc for both directions over i in [-1,N1], j in [-1,N2]: x1 faces
// with i >= 0, x2 faces with j >= 0 (FZLOOP ranges), then the fix_flux
// rules that do not read another face (fixup.c:1357-1410).  Blocks are
// 32 (x1) x FLUX_BY (x2) zones; every zone reconstructs its own interface
// states once: the x1 neighbour's right state arrives by warp shuffle and
// the x2 neighbour's through shared memory (the first lane/row recomputes).
constexpr int FLUX_BY = 4;
template <typename T, bool PARA, bool FFDE>
__global__ void __launch_bounds__(32 * FLUX_BY) k_flux(StepArgs a, const double* __restrict__ pb)
{
  __shared__ double sh[2][32];
  __shared__ T shr[NPR][FLUX_BY][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx - 1;
  const int j = blockIdx.y * FLUX_BY + ty - 1;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  const bool in = (i <= n1) && (j <= n2);
  // threads past the grid work on a clamped (valid) zone; their results are unused
  const int ic = (i <= n1) ? i : n1, jc = (j <= n2) ? j : n2;
  double dt1 = 1.e9, dt2 = 1.e9;
  const long long z = a.gr.at(ic, jc);
  T L[NPR], R[NPR], pl[NPR];
  double Fo[NPR], dtij;
  // ---- x1 faces
  zone_states<T, PARA>(a, pb, ic, jc, 1, L, R);
#pragma unroll
  for (int k = 0; k < NPR; k++) pl[k] = __shfl_up_sync(0xffffffffu, R[k], 1);
  if (tx == 0 && ic >= 0) {
    T Lm[NPR];
    zone_states<T, PARA>(a, pb, ic - 1, jc, 1, Lm, pl);
  }
  if (in && i >= 0) {
    face_flux<T, FFDE>(a, i, j, 1, pl, L, Fo, dtij);
    dt1 = (dtij < dt1) ? dtij : dt1;
    if (i == 0 && j >= -1 && j < n2 && Fo[RHO] > 0) Fo[RHO] = 0;
    if (i == n1 && j >= -1 && j < n2 && Fo[RHO] < 0) Fo[RHO] = 0;
#pragma unroll
    for (int k = 0; k < NPR; k++) a.F1[k * a.gr.plane + z] = Fo[k];
  }
  // ---- x2 faces
  zone_states<T, PARA>(a, pb, ic, jc, 2, L, R);
#pragma unroll
  for (int k = 0; k < NPR; k++) shr[k][ty][tx] = R[k];
  __syncthreads();
  if (ty > 0) {
#pragma unroll
    for (int k = 0; k < NPR; k++) pl[k] = shr[k][ty - 1][tx];
  } else if (jc >= 0) {
    T Lm[NPR];
    zone_states<T, PARA>(a, pb, ic, jc - 1, 2, Lm, pl);
  }
  if (in && j >= 0) {
    face_flux<T, FFDE>(a, i, j, 2, pl, L, Fo, dtij);
    dt2 = (dtij < dt2) ? dtij : dt2;
    const bool polar = (j == 0 || j == n2) && (i < n1);
    const bool equator = (j == (n2 - 1) / 2) && (i >= 0) && (i < n1);
    if (polar || equator) {
#pragma unroll
      for (int k = 0; k < NPR; k++)
        if (k != U2) Fo[k] = 0.;
    }
#pragma unroll
    for (int k = 0; k < NPR; k++) a.F2[k * a.gr.plane + z] = Fo[k];
  }
  dt1 = block_min(dt1, sh[0]);
  dt2 = block_min(dt2, sh[1]);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    a.blockmin[b] = dt1;
    a.blockmin[a.nblocks_flux + b] = dt2;
  }
}

// flux_ct corner EMF, step_ch.c:1214-1234, over i in [0,N1], j in [0,N2].
// F1 on the rows j = -1 and j = N2 carries fix_flux's mirrored B2 for i < N1.
__global__ void k_emf(StepArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i == 0 && j == 0) a.sc->ndeferred = 0;
  if (i > n1 || j > n2) return;
  const long long pl = a.gr.plane;
  const double* F1b2 = a.F1 + B2 * pl;
  const double* F2b1 = a.F2 + B1 * pl;
  double f1a = F1b2[a.gr.at(i, j)];
  if (j == n2 && i < n1) f1a = -F1b2[a.gr.at(i, n2 - 1)];
  double f1b = F1b2[a.gr.at(i, j - 1)];
  if (j - 1 == -1 && i < n1) f1b = -F1b2[a.gr.at(i, 0)];
  double f2a = F2b1[a.gr.at(i, j)], f2b = F2b1[a.gr.at(i - 1, j)];
  const double gc = gdet_at(a, CORN, a.gr.at(i, j));
  const double g1 = gdet_at(a, FACE1, a.gr.at(i, j)), g2 = gdet_at(a, FACE1, a.gr.at(i, j - 1));
  const double g3 = gdet_at(a, FACE2, a.gr.at(i, j)), g4 = gdet_at(a, FACE2, a.gr.at(i - 1, j));
  a.emf[a.gr.at(i, j)] = 0.25 * (gc) * (f1a / (g1) + f1b / (g2) - f2a / (g3) - f2b / (g4));
}

// ---------------------------------------------------------------- update
// Newton iterations a zone may take inside k_update before it is handed to
// k_update_tail (the reference's limit is 200; typical zones need 2-4).
constexpr int NEWTON_MAIN_CAP = 16;

// pflag store + fixup1zone (fixup.c:274-377: floors then the Lorentz factor
// limit) + store of the new primitives
__device__ __forceinline__ void finish_zone(const StepArgs& a, const Geo<double>& g, long long z, int i, int j, double* pfz,
                                            int pfl, double* pf)
{
  const long long pl = a.gr.plane;
  a.pflag[z] = pfl;
  const double frho = __ldg(a.geo + (long long)GEO_FLOOR * pl + z), fu = __ldg(a.geo + (long long)(GEO_FLOOR + 1) * pl + z);
  if (frho > pfz[RHO]) pfz[RHO] = frho;
  if (fu > pfz[UU]) pfz[UU] = fu;
  int rc = limit_gamma(a.pp.gammamax, pfz, g);
  if (rc) report_fail(a.sc, rc, i, j);
#pragma unroll
  for (int k = 0; k < NPR; k++) pf[k * pl + z] = pfz[k];
}

// advance_standard zone loop, advance.c:114-181, for one RK2 substep.
// CUf = {1, 0, c2}: Uf = Ui + c2*dt*dU; on the last substep unew = Uf.
template <bool FFDE>
__global__ void __launch_bounds__(128, 3) k_update(StepArgs a, const double* __restrict__ pi, const double* __restrict__ pb,
                                                double* __restrict__ pf, double c2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.gr.n1 || j >= a.gr.n2) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  const double dt = a.sc->dt;
  Geo<double> g;
  load_geo(a, CENT, z, g);
  const double gam = a.pp.gam;
  double U[NPR], pfz[NPR];
  {
    // Ui = U(pi)
    double pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = __ldg(pi + k * pl + z);
#pragma unroll
    for (int k = 0; k < NPR; k++) pfz[k] = pr[k];
    State<double> q;
    state_of(pr, g, q);
    flux_of<double, FFDE>(pr, q, 0, g, gam, U);
  }
  double dUg[NPR];
  {
    // source_conn, phys.c:520-619: dU[UU+l] = e * sum_j sum_k T^j_k Gamma^k_{lj}
    double pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = __ldg(pb + k * pl + z);
    State<double> q;
    state_of(pr, g, q);
    double acc[4] = {0., 0., 0., 0.};
    const double* cn = a.geo + z;
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      double row[4];
      mhd_row<double, FFDE>(pr, jj, q, gam, row);
#pragma unroll
      for (int l = 0; l < 4; l++)
#pragma unroll
        for (int k = 0; k < 4; k++) acc[l] += row[k] * __ldg(cn + (long long)conn_plane(k, l, jj) * pl);
    }
    dUg[RHO] = 0. + g.g * 0.;
    dUg[B1] = dUg[B2] = dUg[B3] = dUg[RHO];
#pragma unroll
    for (int l = 0; l < 4; l++) dUg[UU + l] = 0. + g.g * acc[l];
  }
  {
    // flux divergence with flux-CT B fluxes (step_ch.c:1403-1413) and the
    // RK combine of dUtoU, advance.c:273-286
    const double idx1 = 1.0 / a.pp.dx1, idx2 = 1.0 / a.pp.dx2;
    const long long zi1 = a.gr.at(i + 1, j), zj1 = a.gr.at(i, j + 1), zij = a.gr.at(i + 1, j + 1);
    const double e00 = a.emf[z], e10 = a.emf[zi1], e01 = a.emf[zj1], e11 = a.emf[zij];
    const double cdt = c2 * dt;
#pragma unroll
    for (int k = 0; k < NPR; k++) {
      double f1p, f1m, f2p, f2m;
      if (k == B1) {
        f1p = 0.;
        f1m = 0.;
        f2m = -0.5 * (e00 + e10);
        f2p = -0.5 * (e01 + e11);
      } else if (k == B2) {
        f1m = 0.5 * (e00 + e01);
        f1p = 0.5 * (e10 + e11);
        f2p = 0.;
        f2m = 0.;
      } else {
        f1p = a.F1[k * pl + zi1];
        f1m = a.F1[k * pl + z];
        f2p = a.F2[k * pl + zj1];
        f2m = a.F2[k * pl + z];
      }
      const double dU1 = (-(f1p - f1m) * idx1);
      const double dU2 = (-(f2p - f2m) * idx2);
      const double dUr = dU1 + dU2;
      U[k] = 1.0 * U[k] + 0.0 * 0.0 + cdt * (dUr + dUg[k]);
    }
  }
  int niter;
  int pfl = utoprim_2d(U, g, pfz, gam, a.pp.gammafail, &niter, NEWTON_MAIN_CAP);
  if (pfl == NEWTON_DEFERRED) {
    // rare slow inversion: hand the zone to k_update_tail so that this warp
    // is not held for up to 200 iterations by one lane
#pragma unroll
    for (int k = 0; k < NPR; k++) a.ubuf[k * pl + z] = U[k];
    a.worklist[atomicAdd(&a.sc->ndeferred, 1)] = (int)z;
    niter = 0;
  } else {
    finish_zone(a, g, z, i, j, pfz, pfl, pf);
  }
  // Newton iteration count (the reference's nstroke), one atomic per warp
  const unsigned mask = __activemask();
  const unsigned it = __reduce_add_sync(mask, (unsigned)niter);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(&a.sc->newton_iters, (unsigned long long)it);
}

// The deferred inversions of k_update, redone with the full iteration limit.
// A deferred zone's pf slot was not written, so pi still holds its guess.
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
    int pfl = utoprim_2d(U, g, pfz, a.pp.gam, a.pp.gammafail, &niter);
    finish_zone(a, g, z, i, j, pfz, pfl, pf);
    atomicAdd(&a.sc->newton_iters, (unsigned long long)niter);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.sc->ndeferred_total += nd;
}

// ---------------------------------------------------------------- bounds
// inflow_check_rel4vel for dir 1 at CENT, fixup.c:1733-1830 (both x1 ends OUTFLOW)
__device__ __forceinline__ int inflow_check_x1(const StepArgs& a, int i, double* pr, const Geo<double>& g)
{
  double ucon[4];
  ucon_of(pr, g, ucon);
  const bool dofix = ((i <= -1) && (ucon[1] > 0.)) || ((i >= a.gr.n1) && (ucon[1] < 0.));
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

// outflow copy + inflow check + gamma limit of an x1 ghost zone (i, j),
// bounds.fishmon.c:28-60 and 192-230 (EXTRAP 0)
__device__ __forceinline__ void x1_ghost(const StepArgs& a, const double* pv, int i, int j, double* pr)
{
  const int is = (i < 0) ? 0 : a.gr.n1 - 1;
  const long long zs = a.gr.at(is, j);
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = pv[k * a.gr.plane + zs];
  Geo<double> g;
  load_geo(a, CENT, a.gr.at(i, j), g);
  int rc = inflow_check_x1(a, i, pr, g);
  if (!rc) rc = limit_gamma(a.pp.gammamax, pr, g);
  if (rc) report_fail(a.sc, rc, i, j);
}

// bound_prim (bounds.fishmon.c:14-330) and bound_pflag (boundsint.c:4-60)
// for every ghost zone; reads only active zones, writes only ghost zones.
// Polar ghosts of the x1 ghost columns take the x1 ghost value of their
// mirror row, as the reference's x1-then-x2 order produces.
__global__ void k_bound(StepArgs a, double* pv, int with_pflag)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - NG;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - NG;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i >= n1 + NG || j >= n2 + NG) return;
  const bool xin = (i >= 0 && i < n1), yin = (j >= 0 && j < n2);
  if (xin && yin) return;
  const long long pl = a.gr.plane, z = a.gr.at(i, j);
  double pr[NPR];
  if (yin) {
    x1_ghost(a, pv, i, j, pr);
    if (j == 0 || j == n2 - 1) {
      pr[U2] *= 0.;
      pr[B2] *= 0.;
    }
  } else {
    const int jm = (j < 0) ? (-j - 1) : (2 * n2 - 1 - j);
    if (xin) {
      const long long zs = a.gr.at(i, jm);
#pragma unroll
      for (int k = 0; k < NPR; k++) pr[k] = pv[k * pl + zs];
    } else {
      x1_ghost(a, pv, i, jm, pr);
    }
    pr[U2] *= 0.;
    pr[B2] *= 0.;
  }
#pragma unroll
  for (int k = 0; k < NPR; k++) pv[k * pl + z] = pr[k];
  if (with_pflag) {
    const int is = (i < 0) ? 0 : ((i >= n1) ? n1 - 1 : i);
    const int js = (j < 0) ? (-j - 1) : ((j >= n2) ? (2 * n2 - 1 - j) : j);
    a.pflag[z] = a.pflag[a.gr.at(is, js)];
  }
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
__global__ void k_gammacheck(StepArgs a, const double* __restrict__ pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < 8 && threadIdx.y == 0) a.sc->chk_changed[threadIdx.x] = 0;
  if (i > a.gr.n1 || j > a.gr.n2) return;
  const long long z = a.gr.at(i, j);
  if (a.bsqf[z] == 0 || a.pflag[z] != 0) return;
  double pr[NPR];
#pragma unroll
  for (int k = 0; k < NPR; k++) pr[k] = pv[k * a.gr.plane + z];
  Geo<double> g;
  load_geo(a, CENT, z, g);
  a.gammacheck[z] = gamma_of(pr, g);
}

// One round of the check-solution vote.  The reference sweeps zones in ZLOOP
// order (i outer, j inner) and a zone flagged there is seen as failed by the
// zones after it.  Here every candidate is decided from the decisions of its
// earlier neighbours in the previous round; the earlier-than relation is
// acyclic, so the sweep's result is the unique fixed point and a round with
// no change proves it has been reached.
__global__ void k_checksol(StepArgs a, const double* __restrict__ pv, int round)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (round > 0 && !a.sc->chk_changed[round - 1]) return;
  if (i == 0 && j == 0) a.sc->chk_final = round;
  if (i >= a.gr.n1 || j >= a.gr.n2) return;
  const long long z = a.gr.at(i, j), pl = a.gr.plane;
  unsigned char* cur = a.chk + (long long)(round & 1) * pl;
  const unsigned char* prev = a.chk + (long long)((round + 1) & 1) * pl;
  if (a.bsqf[z] == 0 || a.pflag[z] != 0) {
    cur[z] = 0;
    return;
  }
  const int di[8] = {0, 0, 1, -1, 1, 1, 1, -1};
  const int dj[8] = {1, -1, 0, 0, 1, -1, 1, -1};
  const double g0 = a.gammacheck[z], u0 = pv[UU * pl + z];
  double pd[8], pd2[8];
#pragma unroll
  for (int l = 0; l < 8; l++) {
    const int ii = i + di[l], jj = j + dj[l];
    const long long zz = a.gr.at(ii, jj);
    bool ok = (a.pflag[zz] == 0);
    // an earlier (ZLOOP order) candidate neighbour counts as failed if flagged
    const bool earlier = (ii < i) || (ii == i && jj < j);
    if (ok && round > 0 && earlier && ii >= 0 && ii < a.gr.n1 && jj >= 0 && jj < a.gr.n2 && prev[zz] != 0) ok = false;
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
  if (round > 0 && d != prev[z]) a.sc->chk_changed[round] = 1;
  if (round == 0 && d != 0) {
    // a flagged zone can only influence later candidates
    bool later_cand = false;
    const int li[4] = {0, 1, 1, 1}, lj[4] = {1, -1, 0, 1};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int ii = i + li[l], jj = j + lj[l];
      if (ii < a.gr.n1 && jj >= 0 && jj < a.gr.n2) {
        const long long zz = a.gr.at(ii, jj);
        if (a.bsqf[zz] != 0 && a.pflag[zz] == 0) later_cand = true;
      }
    }
    if (later_cand) a.sc->chk_changed[0] = 1;
  }
  cur[z] = d;
}

// Sequential ZLOOP sweep for the rare case where the rounds did not settle.
__global__ void k_checksol_serial(StepArgs a, const double* __restrict__ pv, int nrounds)
{
  if (!a.sc->chk_changed[nrounds - 1]) return;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long pl = a.gr.plane;
  const int di[8] = {0, 0, 1, -1, 1, 1, 1, -1};
  const int dj[8] = {1, -1, 0, 0, 1, -1, 1, -1};
  a.sc->chk_final = nrounds - 1;
  unsigned char* out = a.chk + (long long)((nrounds - 1) & 1) * pl;
  for (int i = 0; i < a.gr.n1; i++)
    for (int j = 0; j < a.gr.n2; j++) {
      const long long z = a.gr.at(i, j);
      out[z] = 0;
      if (a.bsqf[z] == 0 || a.pflag[z] != 0) continue;
      const double g0 = a.gammacheck[z], u0 = pv[UU * pl + z];
      double pd[8], pd2[8];
      for (int l = 0; l < 8; l++) {
        const int ii = i + di[l], jj = j + dj[l];
        const long long zz = a.gr.at(ii, jj);
        bool ok = (a.pflag[zz] == 0);
        const bool earlier = (ii < i) || (ii == i && jj < j);
        if (ok && earlier && ii >= 0 && jj >= 0 && jj < a.gr.n2 && out[zz] != 0) ok = false;
        pd[l] = ok ? (a.gammacheck[zz] / g0) : -1;
        pd2[l] = ok ? (pv[UU * pl + zz] / u0) : -1;
      }
      int v0 = 0, v1 = 0, nv = 0;
      for (int l = 0; l < 8; l++)
        if (pd[0] >= 0.0) {
          if ((fabs(pd[l]) > 2.0) || (fabs(pd[l]) < 1.0 / 2.0)) v0++;
          if ((fabs(pd2[l]) > 10.0) || (fabs(pd2[l]) < 1.0 / 10.0)) v1++;
          nv++;
        }
      unsigned char d = 0;
      if (v0 > nv * 0.5) d = PF_GAMMAPERC;
      if (v1 > nv * 0.5) d = PF_UPERC;
      out[z] = d;
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
  const unsigned char* chk = a.chk + (long long)(a.sc->chk_final & 1) * pl;
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
  if (good(i, j + 1) && good(i, j - 1) && good(i + 1, j) && good(i - 1, j)) {
    for (int k = 0; k <= U3; k++) pr[k] = 0.25 * (P(i, j + 1, k) + P(i, j - 1, k) + P(i - 1, j, k) + P(i + 1, j, k));
  } else if (good(i + 1, j + 1) && good(i + 1, j - 1) && good(i - 1, j + 1) && good(i - 1, j - 1)) {
    for (int k = 0; k <= U3; k++) pr[k] = 0.25 * (P(i + 1, j + 1, k) + P(i + 1, j - 1, k) + P(i - 1, j + 1, k) + P(i - 1, j - 1, k));
  } else if (good(i, j + 1) && good(i, j - 1)) {
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i, j + 1, k) + P(i, j - 1, k));
  } else if (good(i + 1, j) && good(i - 1, j)) {
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i + 1, j, k) + P(i - 1, j, k));
  } else if (good(i + 1, j + 1) && good(i - 1, j - 1)) {
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i + 1, j + 1, k) + P(i - 1, j - 1, k));
  } else if (good(i + 1, j - 1) && good(i - 1, j + 1)) {
    for (int k = 0; k <= U3; k++) pr[k] = 0.5 * (P(i + 1, j - 1, k) + P(i - 1, j + 1, k));
  } else {
    const int oi[8] = {1, 1, 1, 0, -1, -1, -1, 0};
    const int oj[8] = {1, 0, -1, -1, -1, 0, 1, 1};
    int m = 0;
    for (; m < 8; m++)
      if (good(i + oi[m], j + oj[m])) break;
    if (m < 8) {
      for (int k = 0; k <= U3; k++) pr[k] = P(i + oi[m], j + oj[m], k);
    } else {
      for (int k = 0; k <= U3; k++)
        pr[k] = 0.5 * (0.25 * (P(i, j + 1, k) + P(i, j - 1, k) + P(i - 1, j, k) + P(i + 1, j, k)) +
                       0.25 * (P(i + 1, j + 1, k) + P(i + 1, j - 1, k) + P(i - 1, j + 1, k) + P(i - 1, j - 1, k)));
    }
  }
  int rc = limit_gamma(gamma, pr, g);
  if (rc) report_fail(a.sc, rc, i, j);
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
  const int c = a.chk[(long long)(a.sc->chk_final & 1) * pl + z];
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

// ---------------------------------------------------------------- dt
// advance.c:190 and step_ch.c:174-183, after the last substep
__global__ void k_dt_finalize(StepArgs a)
{
  __shared__ double sh[2][32];
  double m1 = 1.e9, m2 = 1.e9;
  for (int b = threadIdx.x; b < a.nblocks_flux; b += blockDim.x) {
    double v1 = a.blockmin[b], v2 = a.blockmin[a.nblocks_flux + b];
    m1 = (v1 < m1) ? v1 : m1;
    m2 = (v2 < m2) ? v2 : m2;
  }
  m1 = block_min(m1, sh[0]);
  m2 = block_min(m2, sh[1]);
  if (threadIdx.x == 0) {
    DevScalars* s = a.sc;
    double ndt = a.pp.defcon * 1. / (1. / m1 + 1. / m2);
    s->ndt = ndt;
    s->t += s->dt;
    s->realnstep += 1;
    if (ndt > a.pp.safe * s->dt) ndt = a.pp.safe * s->dt;
    s->dt = ndt;
    if (s->t + s->dt > a.pp.tf) s->dt = a.pp.tf - s->t;
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
    f[4] = 0;
  }
}

// launchers for the templated kernels (used by the host engine)
void launch_flux(int para, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const double* pb)
{
  if (para) k_flux<double, true, false><<<g, b, 0, s>>>(a, pb);
  else k_flux<double, false, false><<<g, b, 0, s>>>(a, pb);
}

void launch_update(dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const double* pi, const double* pb, double* pf,
                   double c2)
{
  k_update<false><<<g, b, 0, s>>>(a, pi, pb, pf, c2);
  k_update_tail<<<148, 64, 0, s>>>(a, pi, pf);
}

}  // namespace harm
