// HARM step kernels for sm_100a.
//
// Data layout in HBM (structure of arrays, x1 index i fastest):
//   a field plane holds one double per zone over the full grid including
//   NG = 3 ghost zones per side; zone (i, j), i in [-3, n1+3), j in [-3, n2+3),
//   sits at (j+3)*pitch + (i+3), with pitch = n1+6 rounded up to 16 doubles
//   (128 B rows).  Primitive state: 8 consecutive planes (rho, u, u~1..3,
//   B1..3).  Geometry: per location (FACE1, FACE2, CORN, CENT) 10 gcov + 10
//   gcon + 1 gdet planes; 40 connection planes Gamma^k_{(lj)} at CENT; 2 floor
//   planes.  Fluxes: 8 planes per direction.
#pragma once
#include <cuda.h>
#include "harm_device.cuh"

namespace harm {

constexpr int NG = 3;

struct Grid {
  int n1, n2;    // interior zones
  int pitch;     // doubles per row (i direction, with ghosts)
  int rows;      // n2 + 2*NG
  long long plane;
  __host__ __device__ __forceinline__ long long at(int i, int j) const { return (long long)(j + NG) * pitch + (i + NG); }
};

// geometry plane offsets inside the geometry block
constexpr int GEO_PER_LOC = 21;                 // 10 gcov, 10 gcon, gdet
constexpr int GEO_CONN = 4 * GEO_PER_LOC;       // 40 connection planes follow
constexpr int GEO_FLOOR = GEO_CONN + 40;        // 2 floor planes
constexpr int GEO_NPLANES = GEO_FLOOR + 2;

__host__ __device__ constexpr int conn_plane(int k, int l, int j) { return GEO_CONN + k * 10 + sym(l, j); }

// k_update's staged geometry: the 40 connection planes and the 2 floor
// planes (GEO_CONN .. GEO_NPLANES-1, contiguous) of the block's zones, one
// TMA box of (block width + 2) columns x block height rows x 42 planes.  The
// box starts on the even column at or before the block's first zone (the
// block width is even), so the zone of thread (tx, ty) sits at column tx + 1.
constexpr int UPD_STAGED = GEO_NPLANES - GEO_CONN;
__host__ __device__ constexpr int upd_box_w(int bx) { return bx + 2; }
__host__ __device__ inline size_t upd_smem_bytes(int bx, int by) { return (size_t)UPD_STAGED * by * upd_box_w(bx) * sizeof(double); }

struct Params {
  int lim;          // 3 MC, 4 PARA
  int fluxmethod;   // 0 LAXF, 1 HLL
  int eom;          // 0 GRMHD, 1 FFDE
  int currents;     // 1: Faraday slots and J^mu every step
  int bc;           // 0 torus (bounds.fishmon.c), 1 rotating star (bounds.ns.c)
  int tryagain;     // 1: the UTOPRIMTRYAGAIN retry chain after a failed 2D inversion
  int fluxadjust;   // FLUXADJUST: per-zone HLL/LAXF choice of the hydro fluxes (FLAGREALFLUX)
  double cour, gam, dx1, dx2, safe, defcon, gammamax, gammafail, bsqorholimit, bsqoulimit, tf;
  double omegastar; // bc 1: angular frequency of the stellar surface
  double gammadamp; // GAMMADAMP: Lorentz-factor threshold of the flux switch
};

// device-resident scalars of the run (one struct in device memory)
struct DevScalars {
  double t, dt, ndt;
  double dt_free;        // the next dt before the end-time clamp
  long long realnstep;
  unsigned long long fail_inv;  // ~key of the first fatal check in the reference's order (0 = none; see fail_key)
  unsigned long long newton_iters;   // Newton iterations since the last reset
  int nchk;              // check-solution zones whose vote may change after round 0 (this substep)
  int fixups;            // zones repaired by fixup_utoprim since the last harm_set_time
  double hz[7];          // horizon accounting of the last step (see k_step_end); hz[6]:
                         // sum of dt (b^2 u^r u_t - b^r b_t) terms since the last harm_set_time
  int ndeferred;         // zones whose inversion went to the tail kernel (this substep)
  int ndeferred_total;   // same, summed since the last harm_set_time
  int cur_ring;          // currents: ring level holding the newest F^{i t}
  long long ccalls;      // currents: calls of current_calc_1 (its static count)
  double clastdt;        // currents: dt of the previous call (its static lastdt)
  int chk_multi;         // substeps whose check-solution sweep needed rounds after the first
  unsigned blocks_done;  // blocks of k_bound_fix finished (its last block ends the step; reset by that block)
};

struct StepArgs {
  Grid gr;
  Params pp;
  const double* geo;     // GEO_NPLANES planes
  const float* geo32;    // mixed precision: FACE1 and FACE2 geometry (2 x 21 float planes)
  double* F1;            // 8 planes (of float in mixed precision)
  double* F2;            // 8 planes (of float in mixed precision)
  double* emf;           // 1 plane
  int* pflag;            // 1 plane (FLAGUTOPRIMFAIL)
  unsigned char* bsqf;   // 1 plane: (b^2/rho flag) | (b^2/u flag) << 2
  unsigned char* fluxf;  // 1 plane (fluxadjust only): FLAGREALFLUX of the zone, 0 LAXF or 1 HLL
  double* gammacheck;    // 1 plane, persistent
  unsigned char* chk;    // 2 planes: check-solution decisions (double buffer)
  double* fixbuf;        // 5 planes: repaired rho..u3
  double* blockmin;      // per-block dt minima: [2][nblocks]
  double* ubuf;          // 8 planes: conserved state of zones deferred to the tail kernel
  int* worklist;         // deferred zone indices (capacity: one plane)
  const double* pstep;   // the step's p (the star's inner ghost field is held at it)
  double* cur;           // currents (25 planes): F^{i t} ring 3x3, F^{i r} 3, F^{i h} 3, fcon 6, jcon 4
  unsigned char* bsqf_fused;  // (or null) k_update sets the b^2 flags of its zones here (first substep, FP64)
  double* rec_pinv;      // adjoint recording (or null): inverted prims before the floors, 8 planes
  unsigned char* rec_fixset;  // adjoint recording (or null): neighbour set of each repaired zone
  int nblocks_flux;
  int phase0;            // PH_PER_SUBSTEP * substep: the fail-key phase of this launch's substep
  int flags_here;        // k_flux forms every zone's b^2 flags and flux choice (the first substep, FP64, fluxadjust)
  DevScalars* sc;
};

// get_bsqflags (fixup.c:1214-1233): (b^2/rho flag) | (b^2/u flag) << 2 of a
// zone-centred state
__device__ __forceinline__ unsigned char bsq_flag(const StepArgs& a, const double* pr, const State<double>& q)
{
  const double bsq = dot4(q.bcon, q.bcov);
  int f0, f3;
  if (bsq / pr[RHO] > a.pp.bsqorholimit) f0 = 2;
  else if (bsq / pr[RHO] > 0.9 * a.pp.bsqorholimit) f0 = 1;
  else f0 = 0;
  if (bsq / pr[UU] > a.pp.bsqoulimit) f3 = 2;
  else if (bsq / pr[UU] > 0.9 * a.pp.bsqoulimit) f3 = 1;
  else f3 = 0;
  return (unsigned char)(f0 | (f3 << 2));
}

// Phases of a substep in the order the reference runs them; a fatal check
// ends the reference's step at the first zone of the first phase in loop
// order (fail(), fail.c:4-57, then every caller returns), so the device
// keeps the smallest key over all reports -- (step, substep phase, position
// of the zone in that phase's loop, code) -- and the reported zone and code
// are those of the reference whatever the order in which threads reach them.
enum { PH_FACE1 = 0, PH_FACE2 = 1, PH_UPDATE = 2, PH_BOUND1 = 3, PH_FIXUP = 4, PH_BOUND2 = 5, PH_PER_SUBSTEP = 8 };
// position in ZLOOP / FZLOOP order (i outer, j inner)
__host__ __device__ __forceinline__ unsigned zone_order(int i, int j)
{
  return ((unsigned)((i + NG) & 0x7fff) << 15) | (unsigned)((j + NG) & 0x7fff);
}
// position in bound_prim's x1 ghost loops (bounds.fishmon.c:30-110, 113-200):
// the inner ghosts first (j outer, i = -1, -2, -3), then the outer ones
__host__ __device__ __forceinline__ unsigned bound_order(int n1, int n2, int i, int j)
{
  return (i < 0) ? (unsigned)(j * NG + (-1 - i)) : (unsigned)(n2 * NG + j * NG + (i - n1));
}
__host__ __device__ __forceinline__ unsigned long long fail_key(long long step, int phase, unsigned order, int code)
{
  const unsigned long long st = (step < 0) ? 0ULL : ((step > 0xffffffLL) ? 0xffffffULL : (unsigned long long)step);
  return (st << 40) | ((unsigned long long)(phase & 15) << 36) | ((unsigned long long)(order & 0x3fffffffu) << 6) |
         (unsigned long long)(code & 63);
}
__device__ __forceinline__ void report_fail(DevScalars* sc, int phase, int code, unsigned order)
{
  atomicMax(&sc->fail_inv, ~fail_key(sc->realnstep, phase, order, code));
}

// FP32 copy of a face location's geometry (mixed precision)
__device__ __forceinline__ void load_geo32(const StepArgs& a, int loc, long long z, Geo<float>& g)
{
  const float* base = a.geo32 + (long long)loc * GEO_PER_LOC * a.gr.plane + z;
#pragma unroll
  for (int c = 0; c < 10; c++) g.gcov[c] = __ldg(base + c * a.gr.plane);
#pragma unroll
  for (int c = 0; c < 10; c++) g.gcon[c] = __ldg(base + (10 + c) * a.gr.plane);
  g.g = __ldg(base + 20 * a.gr.plane);
}

template <typename T>
__device__ __forceinline__ void load_geo(const StepArgs& a, int loc, long long z, Geo<T>& g)
{
  const double* base = a.geo + (long long)loc * GEO_PER_LOC * a.gr.plane + z;
#pragma unroll
  for (int c = 0; c < 10; c++) g.gcov[c] = (T)__ldg(base + c * a.gr.plane);
#pragma unroll
  for (int c = 0; c < 10; c++) g.gcon[c] = (T)__ldg(base + (10 + c) * a.gr.plane);
  g.g = (T)__ldg(base + 20 * a.gr.plane);
}

__device__ __forceinline__ double gdet_at(const StepArgs& a, int loc, long long z)
{
  return __ldg(a.geo + ((long long)loc * GEO_PER_LOC + 20) * a.gr.plane + z);
}

// k_flux blocks: 32 zones along x1 (one warp) x 4 or 8 rows.  Neighbouring
// blocks overlap by one zone along x1, so that each covers FLUX_BX x1 faces
// without recomputing a neighbour's interface state.  8 rows (two 256-thread
// blocks per SM at 128 registers: one block's tile copy overlaps the other's
// faces) are used when that grid still fills three waves of the 148 SMs, 4
// rows (four 128-thread blocks per SM) on smaller grids.  Measured on the
// developed 512^2 torus (step time, three runs each): 8 rows 0.5373-0.5405
// ms, 16 rows (one 512-thread block per SM) 0.5427-0.5463, 15 rows (one
// block per SM, 4.0 waves) 0.5770-0.5799.  The FP32 faces of the mixed form
// fit 128 registers without spilling and run best as 4-row blocks at four
// per SM on any grid.
#ifndef HARM_FLUX_BY_LARGE
#define HARM_FLUX_BY_LARGE 8
#endif
constexpr int FLUX_BX = 31, FLUX_BY_SMALL = 4, FLUX_BY_LARGE = HARM_FLUX_BY_LARGE;
// k_flux's primitive tile (one TMA box over a state's 8 planes): the 32
// columns of the block's zones and 2 more on each side (PARA's stencil) = 36,
// starting on the even column at or before the first (TMA copies start on
// 16-byte boundaries) = 37, rounded to 38 (a row of the box is a multiple of
// 16 bytes); BY rows, 2 more on each side, and one more below for the x2
// neighbour of the first row.  The box's first row is the zone row of the
// block's first zones minus 3 (row -1 of the plane for the first blocks,
// which reads as zero and is never used).
constexpr int FLUX_TILE_W = 38;
__host__ __device__ constexpr int flux_tile_rows(int by) { return by + 5; }
__host__ __device__ constexpr size_t flux_tile_bytes(int by)
{
  return (size_t)NPR * flux_tile_rows(by) * FLUX_TILE_W * sizeof(double);
}
inline dim3 flux_grid(int n1, int n2, int by) { return dim3((n1 + 1 + FLUX_BX - 1) / FLUX_BX, (n2 + 2 + by - 1) / by); }
inline int flux_rows(int n1, int n2, bool fp32_faces)
{
  if (fp32_faces) return FLUX_BY_SMALL;
  const dim3 g = flux_grid(n1, n2, FLUX_BY_LARGE);
  return (g.x * g.y >= 3 * 148) ? FLUX_BY_LARGE : FLUX_BY_SMALL;
}

// plane offsets of the currents block
constexpr int CUR_RING = 0, CUR_S1 = 9, CUR_S2 = 12, CUR_FCON = 15, CUR_JCON = 21, CUR_NPLANES = 25;

// launchers of the templated step kernels (harm_step.cu: FP64 instantiations
// and dispatch; harm_step_mixed.cu: the mixed-precision instantiations)
void launch_flux(int para, int mixed, int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a,
                 const CUtensorMap& prim_map);
void launch_emf(int mixed, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const double* pv);
void launch_update(int mixed, int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map,
                   const double* pi, const double* pb, double* pf, double c2);
void launch_step_end(int mixed, cudaStream_t s, const StepArgs& a, const double* pv);
void launch_bound_fix(int mixed, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, double* pv, int step_end);
void launch_flux_mixed(int para, int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a,
                       const CUtensorMap& prim_map);
void launch_emf_mixed(dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const double* pv);
void launch_update_mixed(int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map,
                         const double* pi, const double* pb, double* pf, double c2);

}  // namespace harm
