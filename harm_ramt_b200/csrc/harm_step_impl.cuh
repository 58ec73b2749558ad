// Templated kernels of the step, shared by the FP64 translation unit
// (harm_step.cu, built without multiply-add contraction so that it rounds
// as the reference does) and the mixed-precision one (harm_step_mixed.cu,
// built with contraction and fast FP32 division/square root).
#pragma once
#include <cuda_runtime.h>
#include "harm_kernels.cuh"
#include "harm_tma.cuh"

namespace harm {

// ---------------------------------------------------------------- fluxes
// Interface states of a zone along `dir` (step_ch.c:812-823 slopes and
// 893-904 interface values) from its stencil in the block's primitive tile
// (shared memory): L = the zone's left-face value (p_r of face i), R = its
// right-face value (p_l of face i+1).  t points at the zone's value of
// plane 0; planes are `ps` doubles apart, the stencil step is `st` (1 along
// x1, the tile width along x2).
template <typename T, bool PARA>
__device__ __forceinline__ void zone_states(const double* t, int ps, int st, T* L, T* R)
{
#pragma unroll
  for (int k = 0; k < NPR; k++) {
    const double* pk = t + k * ps;
    if (!PARA) {
      T ym1 = (T)pk[-st], y0 = (T)pk[0], yp1 = (T)pk[st];
      T dq = mc_slope(ym1, y0, yp1);
      L[k] = y0 - T(0.5) * dq;
      R[k] = y0 + T(0.5) * dq;
    } else {
      T l, r;
      para4((T)pk[-2 * st], (T)pk[-st], (T)pk[0], (T)pk[st], (T)pk[2 * st], l, r);
      L[k] = l;
      R[k] = r;
    }
  }
}

// Flux through one face from its two interface states (the rest of the
// fluxcalc face loop, step_ch.c:944-1065).  The left state is finished
// (state, fluxes, wavespeeds) before the right one starts, and U_r - U_l is
// formed as soon as U_r exists, so only one state is live at a time; the
// values and the order of the fatal checks (both Lorentz limits, then the
// left and the right wavespeeds) are the reference's.
template <typename T, bool FFDE>
__device__ __forceinline__ void face_flux(const StepArgs& a, int i, int j, int dir, T* p_l, T* p_r, T* Fo,
                                          double& dtij, int rf)
{
  const long long z = a.gr.at(i, j);
  Geo<T> g;
  if constexpr (sizeof(T) == 4) load_geo32(a, dir == 1 ? FACE1 : FACE2, z, g);
  else load_geo(a, dir == 1 ? FACE1 : FACE2, z, g);
  // B^dir continuity (BDIRCONT, step_ch.c:944-947)
  if (dir == 1) p_l[B1] = p_r[B1] = T(0.5) * (p_l[B1] + p_r[B1]);
  else p_l[B2] = p_r[B2] = T(0.5) * (p_l[B2] + p_r[B2]);
  const T gmax = (T)a.pp.gammamax, gam = (T)a.pp.gam;
  int rc = limit_gamma(gmax, p_l, g);
  if (!rc) rc = limit_gamma(gmax, p_r, g);
  T F_l[NPR], F_r[NPR], dU[NPR];
  T cmax_l, cmin_l, cmax_r, cmin_r;
  {
    State<T> q;
    state_of(p_l, g, q);
    flux_of<T, FFDE>(p_l, q, dir, g, gam, F_l);
    flux_of<T, FFDE>(p_l, q, 0, g, gam, dU);  // U_l for now
    if (!rc) rc = vchar_of(p_l, q, dir, g, gam, cmax_l, cmin_l);
  }
  {
    State<T> q;
    T U_r[NPR];
    state_of(p_r, g, q);
    flux_of<T, FFDE>(p_r, q, dir, g, gam, F_r);
    flux_of<T, FFDE>(p_r, q, 0, g, gam, U_r);
#pragma unroll
    for (int k = 0; k < NPR; k++) dU[k] = U_r[k] - dU[k];
    if (!rc) rc = vchar_of(p_r, q, dir, g, gam, cmax_r, cmin_r);
  }
  if (rc) {
    report_fail(a.sc, a.phase0 + (dir == 1 ? PH_FACE1 : PH_FACE2), rc, zone_order(i, j));
    cmax_l = cmin_l = cmax_r = cmin_r = T(0.);
  }
  // cminmax_calc, step_ch.c:1095-1148
  T lmin = rmin(cmin_l, cmin_r), lmax = rmax(cmax_l, cmax_r);
  lmin = fabs(rmax(T(0.), -lmin));
  lmax = fabs(rmax(T(0.), lmax));
  T cmin = lmin, cmax = lmax, ctop = rmax(lmax, lmin);
  // choose_flux, step_ch.c:703-738: rf is fluxmethod, or with FLUXADJUST
  // (HYDROFLUXADJUSTONLY 1) FLAGREALFLUX of zone (i, j), the face's own
  // zone, for the hydro variables
  if (cmax + cmin != T(0.0)) {
#pragma unroll
    for (int k = 0; k < NPR; k++) {
      const int m = (k < B1) ? rf : a.pp.fluxmethod;
      const T hllfrac = (m == 1) ? T(1.0) : T(0.0), laxffrac = (m == 1) ? T(0.0) : T(1.0);
      Fo[k] = hllfrac * ((cmax * F_l[k] + cmin * F_r[k] - cmax * cmin * dU[k]) / (cmax + cmin)) +
              laxffrac * (T(0.5) * (F_l[k] + F_r[k] - ctop * dU[k]));
    }
  } else {
#pragma unroll
    for (int k = 0; k < NPR; k++) Fo[k] = T(0.5) * (F_l[k] + F_r[k] - ctop * dU[k]);
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
// rules that do not read another face (fixup.c:1357-1410; the inner x1 mass
// flux clamp only where that end is OUTFLOW, i.e. for the torus).  Blocks are
// 32 (x1) x BY (x2) zones.  The block's primitive tile -- its zones, the
// two-zone stencil halo on every side and one more row below, for the x2
// neighbour of its first row -- arrives in shared memory by one TMA copy
// (flux_tile_*, below); every zone reconstructs its own interface states
// once from the tile: the x1 neighbour's right state arrives by warp
// shuffle and the x2 neighbour's through shared memory (the first row
// recomputes it).  Lane 0's zone is also the previous block's lane 31
// (blocks step by FLUX_BX = 31 along x1): lane 0 only lends its right state,
// and its faces are the previous block's (block 0's lane 0 is zone -1,
// which has no x1 face but an x2 face).
// BY = 4 or 8 rows per block (flux_rows).  At most 128 registers a thread
// for the FP64 faces (512 threads per SM), 96 for the FP32 ones (five 4-row
// blocks per SM).
template <typename T, bool PARA, bool FFDE, int BY>
__global__ void __launch_bounds__(32 * BY, (sizeof(T) == 8) ? 512 / (32 * BY) : ((BY == FLUX_BY_SMALL) ? 5 : 1))
    k_flux(StepArgs a, const __grid_constant__ CUtensorMap prim_map)
{
  extern __shared__ __align__(128) double tile[];
  __shared__ double sh[2][32];
  __shared__ T shr[NPR][BY][32];
  __shared__ uint64_t bar;
  const int tx = threadIdx.x, ty = threadIdx.y;
  constexpr int ROWS = flux_tile_rows(BY), PS = ROWS * FLUX_TILE_W;
  const int cx = (int)(blockIdx.x * FLUX_BX) & ~1;  // the tile's first column (even)
  if (tx == 0 && ty == 0) {
    mbar_init(&bar, 1);
    mbar_expect_tx(&bar, (uint32_t)flux_tile_bytes(BY));
    tma_load_3d(tile, &prim_map, cx, (int)(blockIdx.y * BY) - 1, 0, &bar);
  }
  const int i = blockIdx.x * FLUX_BX + tx - 1;
  const int j = blockIdx.y * BY + ty - 1;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  const bool in = (i <= n1) && (j <= n2);
  const bool own = (tx > 0) || (blockIdx.x == 0);  // lane 0 of a later block repeats a zone
  const long long z = a.gr.at(in ? i : -1, in ? j : -1);
  double dt1 = 1.e9, dt2 = 1.e9;
  T L[NPR], R[NPR], pl[NPR];
  T Fo[NPR];
  double dtij;
  T* F1 = reinterpret_cast<T*>(a.F1);
  T* F2 = reinterpret_cast<T*>(a.F2);
  __syncthreads();  // the barrier is initialised before anyone polls it
  if (!mbar_wait(&bar, 0)) {
    if (tx == 0 && ty == 0) report_fail(a.sc, a.phase0 + PH_FACE1, FAIL_TMA_TIMEOUT, zone_order(i, j));
    return;
  }
  // the zone's value of plane 0 in the tile: row ty + 3, column tx + 2 + (the
  // block's first column - cx)
  const double* tz = tile + (ty + 3) * FLUX_TILE_W + tx + 2 + ((int)(blockIdx.x * FLUX_BX) - cx);
  // the flux choice of this zone, which both of its faces use: fluxmethod,
  // or with the per-zone switch FLAGREALFLUX, formed here in the first
  // substep of the FP64 step (from the step's p, which is this substep's
  // tile; get_bsqflags, fixup.c:1197-1295, with the b^2 flags the repairs
  // read later) and read back in the second
  int rf = a.pp.fluxmethod;
  if (a.pp.fluxadjust && in) {
    if (a.flags_here) {
      double pr[NPR];
#pragma unroll
      for (int k = 0; k < NPR; k++) pr[k] = tz[k * PS];
      Geo<double> gz;
      load_geo(a, CENT, z, gz);
      unsigned char b = 0;
      if (!a.pp.eom) {
        State<double> q;
        state_of(pr, gz, q);
        b = bsq_flag(a, pr, q);
      }
      const double gamma = gamma_of(pr, gz);
      const int f1 = (gamma > 2.0 * a.pp.gammadamp) ? 2 : ((gamma > a.pp.gammadamp) ? 1 : 0);
      rf = ((b & 3) == 2 || f1 == 2 || (b >> 2) == 2) ? a.pp.fluxmethod - 1 : a.pp.fluxmethod;
      rf = (rf < 0) ? 0 : rf;
      if (own) {
        a.bsqf[z] = b;
        a.fluxf[z] = (unsigned char)rf;
      }
    } else {
      rf = (int)a.fluxf[z];
    }
  }
  if constexpr (sizeof(T) == 4) {
    // FP32 faces (mixed form): both directions through one copy of the face
    // code, dir a run-time value (the direction-dependent reads are
    // selects), which halves the kernel's instruction footprint (the FP32
    // kernel stalls on instruction fetch: 1% on the mixed step).  The FP64
    // faces keep one copy per direction (below): the shared copy's register
    // allocation cost them 0.3%.
#pragma unroll 1
    for (int dir = 1; dir <= 2; dir++) {
      zone_states<T, PARA>(tz, PS, (dir == 1) ? 1 : FLUX_TILE_W, L, R);
      bool act;
      if (dir == 1) {
#pragma unroll
        for (int k = 0; k < NPR; k++) pl[k] = __shfl_up_sync(0xffffffffu, R[k], 1);
        act = in && i >= 0 && tx > 0;
      } else {
#pragma unroll
        for (int k = 0; k < NPR; k++) shr[k][ty][tx] = R[k];
        __syncthreads();
        if (ty > 0) {
#pragma unroll
          for (int k = 0; k < NPR; k++) pl[k] = shr[k][ty - 1][tx];
        } else {
          T Lm[NPR];
          zone_states<T, PARA>(tz - FLUX_TILE_W, PS, FLUX_TILE_W, Lm, pl);
        }
        act = in && j >= 0 && own;
      }
      if (act) {
        face_flux<T, FFDE>(a, i, j, dir, pl, L, Fo, dtij, rf);
        T* F;
        if (dir == 1) {
          // x1: fix_flux's mass-flux sign clamps at the two ends
          dt1 = (dtij < dt1) ? dtij : dt1;
          if (i == 0 && a.pp.bc == 0 && j >= -1 && j < n2 && Fo[RHO] > 0) Fo[RHO] = 0;
          if (i == n1 && j >= -1 && j < n2 && Fo[RHO] < 0) Fo[RHO] = 0;
          F = F1;
        } else {
          // x2: only u~2's flux crosses the polar and equatorial faces
          dt2 = (dtij < dt2) ? dtij : dt2;
          const bool polar = (j == 0 || j == n2) && (i < n1);
          const bool equator = (j == (n2 - 1) / 2) && (i >= 0) && (i < n1);
          if (polar || equator) {
#pragma unroll
            for (int k = 0; k < NPR; k++)
              if (k != U2) Fo[k] = T(0.);
          }
          F = F2;
        }
#pragma unroll
        for (int k = 0; k < NPR; k++) F[k * a.gr.plane + z] = Fo[k];
      }
    }
  } else {
    // ---- x1 faces
    zone_states<T, PARA>(tz, PS, 1, L, R);
#pragma unroll
    for (int k = 0; k < NPR; k++) pl[k] = __shfl_up_sync(0xffffffffu, R[k], 1);
    if (in && i >= 0 && tx > 0) {
      face_flux<T, FFDE>(a, i, j, 1, pl, L, Fo, dtij, rf);
      dt1 = (dtij < dt1) ? dtij : dt1;
      if (i == 0 && a.pp.bc == 0 && j >= -1 && j < n2 && Fo[RHO] > 0) Fo[RHO] = 0;
      if (i == n1 && j >= -1 && j < n2 && Fo[RHO] < 0) Fo[RHO] = 0;
#pragma unroll
      for (int k = 0; k < NPR; k++) F1[k * a.gr.plane + z] = Fo[k];
    }
    // ---- x2 faces
    zone_states<T, PARA>(tz, PS, FLUX_TILE_W, L, R);
#pragma unroll
    for (int k = 0; k < NPR; k++) shr[k][ty][tx] = R[k];
    __syncthreads();
    if (ty > 0) {
#pragma unroll
      for (int k = 0; k < NPR; k++) pl[k] = shr[k][ty - 1][tx];
    } else {
      T Lm[NPR];
      zone_states<T, PARA>(tz - FLUX_TILE_W, PS, FLUX_TILE_W, Lm, pl);
    }
    if (in && j >= 0 && own) {
      face_flux<T, FFDE>(a, i, j, 2, pl, L, Fo, dtij, rf);
      dt2 = (dtij < dt2) ? dtij : dt2;
      const bool polar = (j == 0 || j == n2) && (i < n1);
      const bool equator = (j == (n2 - 1) / 2) && (i >= 0) && (i < n1);
      if (polar || equator) {
#pragma unroll
        for (int k = 0; k < NPR; k++)
          if (k != U2) Fo[k] = T(0.);
      }
#pragma unroll
      for (int k = 0; k < NPR; k++) F2[k * a.gr.plane + z] = Fo[k];
    }
  }
  dt1 = block_min(dt1, sh[0]);
  dt2 = block_min(dt2, sh[1]);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    a.blockmin[b] = dt1;
    a.blockmin[a.nblocks_flux + b] = dt2;
  }
}

// the k_flux instance of the block's row count (b.y); its dynamic shared
// memory limit raised once to the tile's size
template <typename T, bool PARA, bool FFDE, int BY>
inline void flux_launch_by(dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map)
{
  constexpr size_t sm = flux_tile_bytes(BY);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_flux<T, PARA, FFDE, BY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  k_flux<T, PARA, FFDE, BY><<<g, b, sm, s>>>(a, map);
}
template <typename T, bool PARA, bool FFDE>
inline void flux_rows_launch(dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map)
{
  if (b.y == FLUX_BY_LARGE) flux_launch_by<T, PARA, FFDE, FLUX_BY_LARGE>(g, b, s, a, map);
  else flux_launch_by<T, PARA, FFDE, FLUX_BY_SMALL>(g, b, s, a, map);
}

// flux_ct corner EMF, step_ch.c:1214-1234, over i in [0,N1], j in [0,N2].
// F1 on the rows j = -1 and j = N2 carries fix_flux's mirrored B2 for i < N1.
// The grid spans i, j from -1: with bsqf_fused set (the first substep of an
// FP64 GRMHD step) the threads of the ring one zone outside the active grid
// (i or j in {-1, N}) set the b^2 flags of their zone from the step's p, as
// get_bsqflags does over its DQZLOOP range (fixup.c:1197-1233); the first
// substep's k_update sets those of the active zones.
template <typename FT>
__global__ void k_emf(StepArgs a, const double* __restrict__ pv)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - 1;
  const int n1 = a.gr.n1, n2 = a.gr.n2;
  if (i == 0 && j == 0) a.sc->ndeferred = 0;
  if (i > n1 || j > n2) return;
  if (a.bsqf_fused && (i == -1 || i == n1 || j == -1 || j == n2)) {
    const long long z = a.gr.at(i, j);
    double pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = __ldg(pv + k * a.gr.plane + z);
    Geo<double> g;
    load_geo(a, CENT, z, g);
    State<double> q;
    state_of(pr, g, q);
    a.bsqf[z] = bsq_flag(a, pr, q);
  }
  if (i < 0 || j < 0) return;
  const long long pl = a.gr.plane;
  const FT* F1b2 = reinterpret_cast<const FT*>(a.F1) + B2 * pl;
  const FT* F2b1 = reinterpret_cast<const FT*>(a.F2) + B1 * pl;
  double f1a = F1b2[a.gr.at(i, j)];
  if (j == n2 && i < n1) f1a = -(double)F1b2[a.gr.at(i, n2 - 1)];
  double f1b = F1b2[a.gr.at(i, j - 1)];
  if (j - 1 == -1 && i < n1) f1b = -(double)F1b2[a.gr.at(i, 0)];
  double f2a = F2b1[a.gr.at(i, j)], f2b = F2b1[a.gr.at(i - 1, j)];
  const double gc = gdet_at(a, CORN, a.gr.at(i, j));
  const double g1 = gdet_at(a, FACE1, a.gr.at(i, j)), g2 = gdet_at(a, FACE1, a.gr.at(i, j - 1));
  const double g3 = gdet_at(a, FACE2, a.gr.at(i, j)), g4 = gdet_at(a, FACE2, a.gr.at(i - 1, j));
  a.emf[a.gr.at(i, j)] = 0.25 * (gc) * (f1a / (g1) + f1b / (g2) - f2a / (g3) - f2b / (g4));
}

// ---------------------------------------------------------------- update
// Newton iterations a zone may take inside k_update before it is handed to
// k_update_tail, which continues the solve from the saved state (the
// reference's limit is 200; typical zones need 2-4).
#ifndef HARM_NEWTON_CAP
#define HARM_NEWTON_CAP 16
#endif
constexpr int NEWTON_MAIN_CAP = HARM_NEWTON_CAP;

// pflag store + fixup1zone (fixup.c:274-377: floors then the Lorentz factor
// limit) + store of the new primitives; frho, fu: the zone's floors
__device__ __forceinline__ void finish_zone(const StepArgs& a, const Geo<double>& g, long long z, int i, int j, double* pfz,
                                            int pfl, double* pf, double frho, double fu)
{
  const long long pl = a.gr.plane;
  if (a.rec_pinv) {
#pragma unroll
    for (int k = 0; k < NPR; k++) a.rec_pinv[k * pl + z] = pfz[k];
  }
  a.pflag[z] = pfl;
  if (frho > pfz[RHO]) pfz[RHO] = frho;
  if (fu > pfz[UU]) pfz[UU] = fu;
  int rc = limit_gamma(a.pp.gammamax, pfz, g);
  if (rc) report_fail(a.sc, a.phase0 + PH_UPDATE, rc, zone_order(i, j));
#pragma unroll
  for (int k = 0; k < NPR; k++) pf[k * pl + z] = pfz[k];
}

// advance_standard zone loop, advance.c:114-181, for one RK2 substep.
// CUf = {1, 0, c2}: Uf = Ui + c2*dt*dU; on the last substep unew = Uf.
// The connection coefficients and floors arrive by TMA (geo_map, a 3D map
// over the geometry block with the box above) while U(p_i) and the flux
// divergence are formed from global loads; the block width is even.
template <typename FT, bool FFDE>
__global__ void __launch_bounds__(128, 4) k_update(StepArgs a, const __grid_constant__ CUtensorMap geo_map,
                                                const double* __restrict__ pi, const double* __restrict__ pb,
                                                double* __restrict__ pf, double c2)
{
  extern __shared__ __align__(128) double sgeo[];
  __shared__ uint64_t bar;
  const FT* F1 = reinterpret_cast<const FT*>(a.F1);
  const FT* F2 = reinterpret_cast<const FT*>(a.F2);
  // block rows in launch order from both poles inward (0, last, 1, last-1,
  // ...): the zones near the axis take the most Newton iterations, and
  // started first their blocks no longer trail the kernel's last wave
  // (developed 512^2 flow: 0.5256-0.5309 against 0.5333-0.5366 ms a step)
  const unsigned by = (blockIdx.y & 1u) ? gridDim.y - 1u - (blockIdx.y >> 1) : (blockIdx.y >> 1);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int W = upd_box_w(blockDim.x);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    mbar_init(&bar, 1);
    mbar_expect_tx(&bar, (uint32_t)upd_smem_bytes(blockDim.x, blockDim.y));
    tma_load_3d(sgeo, &geo_map, (int)((blockIdx.x * blockDim.x + NG) & ~1u), (int)(by * blockDim.y + NG),
                GEO_CONN, &bar);
  }
  __syncthreads();  // the barrier is initialised before anyone polls it
  const bool active = (i < a.gr.n1 && j < a.gr.n2);
  const long long pl = a.gr.plane, z = a.gr.at(active ? i : 0, active ? j : 0);
  const double dt = a.sc->dt;
  Geo<double> g;
  const double gam = a.pp.gam;
  double U[NPR], pfz[NPR], dUr[NPR];
  if (active) {
    load_geo(a, CENT, z, g);
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
      if (a.bsqf_fused) a.bsqf_fused[z] = bsq_flag(a, pr, q);  // get_bsqflags of the step's p
    }
    {
      // flux divergence with flux-CT B fluxes (step_ch.c:1403-1413)
      const double idx1 = 1.0 / a.pp.dx1, idx2 = 1.0 / a.pp.dx2;
      const long long zi1 = a.gr.at(i + 1, j), zj1 = a.gr.at(i, j + 1), zij = a.gr.at(i + 1, j + 1);
      const double e00 = a.emf[z], e10 = a.emf[zi1], e01 = a.emf[zj1], e11 = a.emf[zij];
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
          f1p = F1[k * pl + zi1];
          f1m = F1[k * pl + z];
          f2p = F2[k * pl + zj1];
          f2m = F2[k * pl + z];
        }
        const double dU1 = (-(f1p - f1m) * idx1);
        const double dU2 = (-(f2p - f2m) * idx2);
        dUr[k] = dU1 + dU2;
      }
    }
  }
  if (!mbar_wait(&bar, 0)) {
    if (active) report_fail(a.sc, a.phase0 + PH_UPDATE, FAIL_TMA_TIMEOUT, zone_order(i, j));
    return;
  }
  if (!active) return;
  const int plane_s = blockDim.y * W;
  const double* sz = sgeo + threadIdx.y * W + threadIdx.x + 1;
  double dUg[NPR];
  {
    // source_conn, phys.c:520-619: dU[UU+l] = e * sum_j sum_k T^j_k Gamma^k_{lj}
    double pr[NPR];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = __ldg(pb + k * pl + z);
    State<double> q;
    state_of(pr, g, q);
    double acc[4] = {0., 0., 0., 0.};
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      double row[4];
      mhd_row<double, FFDE>(pr, jj, q, gam, row);
#pragma unroll
      for (int l = 0; l < 4; l++)
#pragma unroll
        for (int k = 0; k < 4; k++) acc[l] += row[k] * sz[(conn_plane(k, l, jj) - GEO_CONN) * plane_s];
    }
    dUg[RHO] = 0. + g.g * 0.;
    dUg[B1] = dUg[B2] = dUg[B3] = dUg[RHO];
#pragma unroll
    for (int l = 0; l < 4; l++) dUg[UU + l] = 0. + g.g * acc[l];
  }
  {
    // the RK combine of dUtoU, advance.c:273-286
    const double cdt = c2 * dt;
#pragma unroll
    for (int k = 0; k < NPR; k++) U[k] = 1.0 * U[k] + 0.0 * 0.0 + cdt * (dUr[k] + dUg[k]);
  }
  if constexpr (FFDE) {
    // Utoprim_ffde, then fixup1zone's Lorentz-factor limit (the floors are
    // GRMHD-only, fixup.c:293); pflag is left as it was
    int rc = utoprim_ffde(U, g, pfz, a.pp.gammamax);
    if (!rc) rc = limit_gamma(a.pp.gammamax, pfz, g);
    if (rc) report_fail(a.sc, a.phase0 + PH_UPDATE, rc, zone_order(i, j));
#pragma unroll
    for (int k = 0; k < NPR; k++) pf[k * pl + z] = pfz[k];
    return;
  }
  int niter;
  // a deferred solve leaves its Newton state in the repair scratch (idle
  // until k_fixup_compute), NEWTON_STATE planes
  int pfl = utoprim_2d(U, g, pfz, gam, a.pp.gammafail, &niter, NEWTON_MAIN_CAP, a.fixbuf + z, pl);
  if (pfl == NEWTON_DEFERRED || (a.pp.tryagain && pfl != 0)) {
    // rare slow inversion: hand the zone to k_update_tail so that this warp
    // is not held for up to 200 iterations by one lane (with the retry
    // chain on, failed inversions go there too, to be solved afresh)
    if (pfl != NEWTON_DEFERRED) a.fixbuf[(NEWTON_STATE - 1) * pl + z] = -1.0;
#pragma unroll
    for (int k = 0; k < NPR; k++) a.ubuf[k * pl + z] = U[k];
    a.worklist[atomicAdd(&a.sc->ndeferred, 1)] = (int)z;
    niter = 0;
  } else {
    finish_zone(a, g, z, i, j, pfz, pfl, pf, sz[(GEO_FLOOR - GEO_CONN) * plane_s],
                sz[(GEO_FLOOR + 1 - GEO_CONN) * plane_s]);
  }
  // Newton iteration count (the reference's nstroke), one atomic per warp
  const unsigned mask = __activemask();
  const unsigned it = __reduce_add_sync(mask, (unsigned)niter);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(&a.sc->newton_iters, (unsigned long long)it);
}



// launches a k_update instance (its dynamic shared memory limit raised once
// to the largest box of the tile shapes harm_set_tiles accepts: 42 planes x
// at most 128 threads)
template <typename FT, bool FFDE>
inline void update_launch(dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map, const double* pi,
                          const double* pb, double* pf, double c2)
{
  static bool attr = false;
  if (!attr) {
    size_t mx = 0;
    for (int by = 1; by <= 128; by++) {
      const int bx = 128 / by;
      const size_t v = upd_smem_bytes(bx + (bx & 1), by);
      if (v > mx) mx = v;
    }
    cudaFuncSetAttribute(k_update<FT, FFDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
    attr = true;
  }
  k_update<FT, FFDE><<<g, b, upd_smem_bytes(b.x, b.y), s>>>(a, map, pi, pb, pf, c2);
}

// ---------------------------------------------------------------- end of step
// diag_flux() for the global region's inner x1 face (diag.c:576-833): the
// face fluxes in diagnostic form (UtoU UEVOLVE->UDIAG) and the energy-
// equation stress terms 3 and 6 from the zone-centred state pr of row j.
template <typename FT>
__device__ __forceinline__ void horizon_terms(const StepArgs& a, const double* pr, int j, double* t4)
{
  const FT* F1 = reinterpret_cast<const FT*>(a.F1);
  const long long pl = a.gr.plane;
  const double surface = a.pp.dx2 * (2.0 * 3.14159265358979323846);
  const long long z = a.gr.at(0, j);
  const double gf = gdet_at(a, FACE1, z);
  const double Fr = (double)F1[RHO * pl + z] * surface, Fu = (double)F1[UU * pl + z] * surface;
  const double gr = Fr / gf;
  double gu = Fu / gf;
  gu += -gr;
  t4[0] = gr * gf;
  t4[1] = gu * gf;
  Geo<double> g;
  load_geo(a, CENT, z, g);
  State<double> q;
  state_of(pr, g, q);
  double bsq = 0;
#pragma unroll
  for (int l = 0; l < 4; l++) bsq += (q.bcon[l]) * (q.bcov[l]);
  const double surgdet = (g.g) * surface;
  t4[2] = bsq * (q.ucon[1]) * (q.ucov[0]) * surgdet;
  t4[3] = -(q.bcon[1]) * (q.bcov[0]) * surgdet;
}

// The end of a step, by every thread of one block, after the horizon terms
// of every row j sit in t[k * ts + j] (k < 4): their sums in j order as the
// reference's loop adds them (so the sums are exact), pcum += pdot * dt
// (diag.c:576-833); then the new dt from the flux blocks' Courant minima
// (advance.c:190, step_ch.c:174-183) and t += dt.  L2: the terms were
// written by other blocks of the same kernel (read past L1).
template <bool L2>
__device__ __forceinline__ void step_end_finish(const StepArgs& a, const double* t, long long ts)
{
  constexpr int CHUNK = 256;
  __shared__ double sh[2][32];
  __shared__ double acc[4];
  __shared__ double stage[4][CHUNK + 1];  // rows one double apart in banks: the four adding lanes do not conflict
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
  const int n2 = a.gr.n2;
  // chunks of the four term rows are staged in shared memory by the whole
  // block (independent loads), then four threads add them one after another
  // in j order
  double s = 0.;
  for (int j0 = 0; j0 < n2; j0 += CHUNK) {
    const int m = (n2 - j0 < CHUNK) ? n2 - j0 : CHUNK;
#pragma unroll 8
    for (int q = tid; q < 4 * m; q += nt) {
      const int k = q / m, jj = q - k * m;
      const double* src = t + k * ts + j0 + jj;
      stage[k][jj] = L2 ? __ldcg(src) : *src;
    }
    __syncthreads();
    if (tid < 4) {
      const double* b = stage[tid];
      int q = 0;
      for (; q + 8 <= m; q += 8) {
        double v[8];
#pragma unroll
        for (int r = 0; r < 8; r++) v[r] = b[q + r];
#pragma unroll
        for (int r = 0; r < 8; r++) s += v[r];
      }
      for (; q < m; q++) s += b[q];
    }
    __syncthreads();
  }
  if (tid < 4) acc[tid] = s;
  __syncthreads();
  if (tid == 0) {
    DevScalars* sc = a.sc;
    for (int k = 0; k < 4; k++) sc->hz[k] = acc[k];
    sc->hz[4] += acc[0] * sc->dt;
    sc->hz[5] += acc[1] * sc->dt;
    sc->hz[6] += (acc[2] + acc[3]) * sc->dt;
  }
  double m1 = 1.e9, m2 = 1.e9;
#pragma unroll 4
  for (int b = tid; b < a.nblocks_flux; b += nt) {
    double v1 = __ldcg(a.blockmin + b), v2 = __ldcg(a.blockmin + a.nblocks_flux + b);
    m1 = (v1 < m1) ? v1 : m1;
    m2 = (v2 < m2) ? v2 : m2;
  }
  m1 = block_min(m1, sh[0]);
  m2 = block_min(m2, sh[1]);
  if (tid == 0) {
    DevScalars* s = a.sc;
    double ndt = a.pp.defcon * 1. / (1. / m1 + 1. / m2);
    s->ndt = ndt;
    const bool moved = s->dt > 0.;
    s->t += s->dt;
    s->realnstep += 1;
    if (ndt > a.pp.safe * s->dt) ndt = a.pp.safe * s->dt;
    s->dt = ndt;
    if (moved) s->dt_free = ndt;  // a step at dt = 0 (past the end time) keeps the last one
    if (s->t + s->dt > a.pp.tf) s->dt = a.pp.tf - s->t;
  }
}

// After the last substep, one block: the horizon terms of every row j (into
// the inversion scratch ubuf, idle by now), then step_end_finish.
constexpr int STEP_END_THREADS = 512;
template <typename FT>
__global__ void __launch_bounds__(STEP_END_THREADS) k_step_end(StepArgs a, const double* __restrict__ pv)
{
  const long long pl = a.gr.plane;
  for (int j = threadIdx.x; j < a.gr.n2; j += blockDim.x) {
    const long long z = a.gr.at(0, j);
    double pr[NPR], t4[4];
#pragma unroll
    for (int k = 0; k < NPR; k++) pr[k] = pv[k * pl + z];
    horizon_terms<FT>(a, pr, j, t4);
#pragma unroll
    for (int k = 0; k < 4; k++) a.ubuf[k * pl + j] = t4[k];
  }
  __syncthreads();
  step_end_finish<false>(a, a.ubuf, pl);
}

}  // namespace harm
