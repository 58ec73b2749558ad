// Host engine and C ABI (include/harm_b200.h) of the B200 HARM step.
//
// The engine owns the device arrays (structure-of-arrays planes, see
// harm_kernels.cuh), converts the reference-layout host arrays on upload and
// download, and enqueues one step of step_ch() (step_ch.c:35-188 with the
// midpoint RK2 of setup_rktimestep, step_ch.c:412-429) as a fixed sequence
// of kernels on its stream.  The sequence is captured once into a CUDA graph
// and replayed; dt and t live in device memory, so steps chain without host
// round trips.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <functional>
#include <vector>

#include "../../include/harm_b200.h"
#include "harm_kernels.cuh"
#include "harm_tma.cuh"
#include <cudaTypedefs.h>

namespace harm {
__global__ void k_bsqflags(StepArgs a, const double* pv);
__global__ void k_bound(StepArgs a, double* pv, int with_pflag);
__global__ void k_poledeath(StepArgs a, double* pv);
__global__ void k_gammacheck(StepArgs a, double* pv, int poledeath);
__global__ void k_bound_gc(StepArgs a, double* pv);
__global__ void k_checksol(StepArgs a, double* pv, int poledeath);
__global__ void k_checksol_rounds(StepArgs a, const double* pv);
__global__ void k_fixup_compute(StepArgs a, const double* pv);
__global__ void k_fixup_apply(StepArgs a, double* pv, int grmhd);
__global__ void k_faraday(StepArgs a, const double* pv);
__global__ void k_current(StepArgs a);
__global__ void k_currents_commit(StepArgs a);
__global__ void k_dump_columns(StepArgs a, const double* pv, double* out, int* nfail);
__global__ void k_adj_seed_edot(StepArgs a, const double* pv, double* lam, double wfac);
__global__ void k_adj_poledeath(StepArgs a, double* lam);
__global__ void k_adj_ghosts(StepArgs a, double* lam, const double* src);
__global__ void k_adj_fixup(StepArgs a, const double* lam_in, double* lam_snap, const double* snap, const int* flag,
                            const unsigned char* fixset);
__global__ void k_adj_update(StepArgs a, const double* lam, const double* pinv, const int* flaginv, double cfac,
                             double* ubar, double* lam_dU);
__global__ void k_adj_upi(StepArgs a, const double* ubar, const double* pi, double* lam_pi);
__global__ void k_adj_source(StepArgs a, const double* pb, const double* lam_dU, double* lam_b);
__global__ void k_adj_corner(StepArgs a, const double* lam_dU, double* lam_e);
template <int dir>
__global__ void k_adj_faces(StepArgs a, const double* pb, const double* lam_dU, const double* lam_e, double* sl,
                            double* sr, double seed_fac);
template <int dir>
__global__ void k_adj_recon(StepArgs a, const double* pb, const double* sl, const double* sr, double* lam_b);
__global__ void k_set_dt(StepArgs a, const double* dts, int k);
__global__ void k_invert_zones(StepArgs a, int which, int nz, const int* zones, const double* U, double* pr, int* pfl);
__global__ void k_get_dt(StepArgs a, double* dts, int k);
__global__ void k_axpy(double* y, const double* x, long long n);
__global__ void k_mask_ghosts(StepArgs a, double* lam);
__global__ void k_dot_active(StepArgs a, const double* lam, const double* pv, double* out);
constexpr int DUMP_DYNCOLS = 50;
__global__ void k_ref_to_planes(StepArgs a, const double* ref, const int* refflag, double* pv);
__global__ void k_planes_to_ref(StepArgs a, const double* pv, double* ref, int* refflag);
}  // namespace harm

using namespace harm;


struct harm_ctx {
  harm_config cfg;
  cudaStream_t stream;
  Grid gr;
  int n1m, n2m;
  // device buffers
  double *d_p, *d_pk0, *d_geo, *d_F1, *d_F2, *d_emf, *d_gammacheck, *d_fixbuf, *d_blockmin, *d_ubuf, *d_cur;
  float* d_geo32;
  int *d_pflag, *d_worklist;
  double* d_stage;   // reference-layout prims staging buffer
  int* d_stagef;     // reference-layout pflag staging buffer
  unsigned char *d_bsqf, *d_chk, *d_fluxf;
  DevScalars* d_sc;
  int nblocks_flux;
  int flux_by;       // k_flux rows per block (flux_rows)
  bool geo_ok;
  cudaGraph_t graph;
  cudaGraphExec_t gexec;
  bool have_graph;
  dim3 tile_update;  // k_update block (at most 128 threads, even width)
  CUtensorMap geo_map;  // k_update's TMA box over the geometry block (tile_update + 2 columns)
  CUtensorMap map_p, map_pk0;  // k_flux's TMA boxes over the state p and the midpoint state pk[0]
  dim3 tile_small;   // block of the stencil/fixup/boundary kernels
  StepArgs args() const
  {
    StepArgs a{};
    a.gr = gr;
    a.pp.lim = cfg.lim;
    a.pp.fluxmethod = cfg.fluxmethod;
    a.pp.eom = cfg.eom;
    a.pp.bc = cfg.bc;
    a.pp.omegastar = cfg.omegastar;
    a.pp.cour = cfg.cour;
    a.pp.gam = cfg.gam;
    a.pp.dx1 = cfg.dx1;
    a.pp.dx2 = cfg.dx2;
    a.pp.safe = cfg.safe;
    a.pp.defcon = cfg.defcon;
    a.pp.gammamax = cfg.gammamax;
    a.pp.gammafail = cfg.gammafail;
    a.pp.bsqorholimit = cfg.bsqorholimit;
    a.pp.bsqoulimit = cfg.bsqoulimit;
    a.pp.tf = cfg.tf;
    a.geo = d_geo;
    a.geo32 = d_geo32;
    a.F1 = d_F1;
    a.F2 = d_F2;
    a.emf = d_emf;
    a.pflag = d_pflag;
    a.bsqf = d_bsqf;
    a.gammacheck = d_gammacheck;
    a.chk = d_chk;
    a.fixbuf = d_fixbuf;
    a.blockmin = d_blockmin;
    a.ubuf = d_ubuf;
    a.worklist = d_worklist;
    a.pstep = d_p;
    a.cur = d_cur;
    a.pp.currents = cfg.currents;
    a.pp.tryagain = cfg.tryagain;
    a.pp.fluxadjust = cfg.fluxadjust;
    a.pp.gammadamp = cfg.gammadamp;
    a.fluxf = d_fluxf;
    a.rec_pinv = nullptr;
    a.rec_fixset = nullptr;
    a.bsqf_fused = nullptr;
    a.nblocks_flux = nblocks_flux;
    a.sc = d_sc;
    return a;
  }
};

#define CK(call)                                     \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) {                         \
      fprintf(stderr, "harm_b200: %s: %s\n", #call, cudaGetErrorString(e_)); \
      return HARM_ECUDA;                             \
    }                                                \
  } while (0)

static dim3 grid2(int ni, int nj, dim3 b) { return dim3((ni + b.x - 1) / b.x, (nj + b.y - 1) / b.y); }

namespace harm {
bool tma_encode_planes(CUtensorMap* map, const double* base, int pitch, int rows, int nplanes, long long plane, int bx,
                       int by, int bz)
{
  static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
  if (!enc) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)rows, (cuuint64_t)nplanes};
  const cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(double), (cuuint64_t)plane * sizeof(double)};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace harm

// k_flux's map over a state's 8 planes, the box of one block's tile
static bool encode_prim_map(CUtensorMap* map, const double* prims, const Grid& gr, int flux_by)
{
  if ((uintptr_t)prims & 15) return false;
  return tma_encode_planes(map, prims, gr.pitch, gr.rows, NPR, gr.plane, FLUX_TILE_W, flux_tile_rows(flux_by), NPR);
}

// k_update's map: the geometry block, boxes of the block's zones (and one
// column more on each side) over the 42 connection and floor planes
static bool encode_geo_map(CUtensorMap* map, const double* geo, const Grid& gr, dim3 ub)
{
  if ((ub.x & 1) || ((uintptr_t)geo & 15)) return false;
  return tma_encode_planes(map, geo, gr.pitch, gr.rows, GEO_NPLANES, gr.plane, (int)upd_box_w(ub.x), (int)ub.y,
                           UPD_STAGED);
}

// kernel classes of one step, in launch order (for per-kernel timing)
enum { KC_BSQ = 0, KC_FLUX, KC_EMF, KC_UPDATE, KC_BOUND, KC_POLE, KC_GCHECK, KC_CHECKSOL, KC_CHECKSERIAL, KC_FIXC,
       KC_FIXA, KC_DT, KC_HORIZON, KC_FARADAY, KC_CURRENT, KC_COUNT };
// (KC_FIXA: k_fixup_apply on the adjoint's recording path, k_bound_fix --
// repairs, second bound and POLEDEATH in one kernel -- on every other)
static const char* const KC_NAMES[KC_COUNT] = {"k_bsqflags", "k_flux", "k_emf", "k_update", "k_bound", "k_poledeath",
                                               "k_gammacheck", "k_checksol", "k_checksol_rounds", "k_fixup_compute",
                                               "k_bound_fix", "k_step_end", "k_horizon", "k_faraday",
                                               "k_current"};

struct Timer {
  // records an event after every launch (or pair of launches) when active
  cudaEvent_t ev[64];
  int cls[64];
  int nk[64];  // kernels launched since the previous event
  int n = 0;
  bool on = false;
  void mark(cudaStream_t s, int k, int kernels = 1)
  {
    if (!on || n >= 63) return;
    cudaEventRecord(ev[n + 1], s);
    cls[n + 1] = k;
    nk[n + 1] = kernels;
    n++;
  }
};

// What the adjoint's forward recomputation of a step keeps (per substep):
// the inverted primitives before floors, the update's output and pflag, the
// state after the first bound (what the repairs read), the state after the
// repairs and the final pflag, and the neighbour set of each repair.
struct Rec {
  double* pn;  // the step's p
  double* ph;  // the midpoint state (pk[0]) the second substep reads
  double* pinv[2];
  double* upd[2];
  double* snap[2];
  double* pre2[2];
  int* flaginv[2];
  int* flag[2];
  unsigned char* fixset[2];
};

static int enqueue_step(harm_ctx* c, Timer* tm = nullptr, const Rec* rec = nullptr)
{
  Timer dummy;
  Timer& T = tm ? *tm : dummy;
  const StepArgs a0 = c->args();
  StepArgs a = a0;
  const int n1 = c->cfg.n1, n2 = c->cfg.n2;
  const dim3 fb(32, c->flux_by);  // k_flux's shape is fixed by its warp/shared-memory state sharing
  const dim3 b = c->tile_small;   // the other stencil kernels
  const dim3 ub = c->tile_update;
  cudaStream_t s = c->stream;
  const size_t pbytes = (size_t)NPR * c->gr.plane * sizeof(double), fbytes = (size_t)c->gr.plane * sizeof(int);
  if (rec) cudaMemcpyAsync(rec->pn, c->d_p, pbytes, cudaMemcpyDeviceToDevice, s);
  // b^2 flags of the step's p: GRMHD sets them inside the first substep,
  // the active zones' in k_update (from the state it forms anyway) and the
  // one-zone ring's in k_emf (in the mixed form these FP64 flags are built
  // with contraction, like the rest of its kernels); the force-free step
  // has none (k_bsqflags clears them).  (With the
  // flux switch every flag of the DQZLOOP range is needed by the first
  // substep's fluxes: each k_flux thread forms its zone's, which its faces
  // use.)
  const bool fuse_bsq = (c->cfg.eom == HARM_EOM_GRMHD) && !c->cfg.fluxadjust;
  // with the switch, the first substep's k_flux forms all of them
  const bool flags_in_flux = c->cfg.fluxadjust != 0;
  if (!fuse_bsq && !flags_in_flux) {
    k_bsqflags<<<grid2(n1 + 2, n2 + 2, b), b, 0, s>>>(a, c->d_p);
    T.mark(s, KC_BSQ);
  }
  bool step_ended = false;
  for (int sub = 0; sub < 2; sub++) {
    if (rec) {
      a.rec_pinv = rec->pinv[sub];
      a.rec_fixset = rec->fixset[sub];
    }
    a.bsqf_fused = (fuse_bsq && sub == 0) ? a0.bsqf : nullptr;
    a.phase0 = sub * PH_PER_SUBSTEP;
    a.flags_here = (flags_in_flux && sub == 0) ? 1 : 0;
    const double* pi = c->d_p;
    const double* pb = (sub == 0) ? c->d_p : c->d_pk0;
    double* pf = (sub == 0) ? c->d_pk0 : c->d_p;
    const double c2 = (sub == 0) ? 0.5 : 1.0;
    const int mixed = c->cfg.precision == HARM_PREC_MIXED;
    const int ffde = c->cfg.eom == HARM_EOM_FFDE;
    const bool poledeath = c->cfg.bc == HARM_BC_TORUS;
    launch_flux(c->cfg.lim == HARM_LIM_PARA, mixed, ffde, flux_grid(n1, n2, c->flux_by), fb, s, a,
                (sub == 0) ? c->map_p : c->map_pk0);
    T.mark(s, KC_FLUX);
    launch_emf(mixed, grid2(n1 + 2, n2 + 2, b), b, s, a, c->d_p);
    T.mark(s, KC_EMF);
    launch_update(mixed, ffde, grid2(n1, n2, ub), ub, s, a, c->geo_map, pi, pb, pf, c2);
    T.mark(s, KC_UPDATE, ffde ? 1 : 2);  // k_update and k_update_tail
    if (rec) {
      cudaMemcpyAsync(rec->upd[sub], pf, pbytes, cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(rec->flaginv[sub], c->d_pflag, fbytes, cudaMemcpyDeviceToDevice, s);
    }
    if (!ffde && !rec) {
      // GRMHD: the first bound with the check-solution gamma table, the vote
      // (which also writes the POLEDEATH zeroing that follows this bound),
      // its later rounds, the repairs, and the repairs applied with the
      // second bound -- after the last substep also the end of the step
      const bool last = (sub == 1) && !c->cfg.currents;
      k_bound_gc<<<grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, 0, s>>>(a, pf);
      T.mark(s, KC_BOUND);
      k_checksol<<<grid2(n1, n2, b), b, 0, s>>>(a, pf, poledeath ? 1 : 0);
      T.mark(s, KC_CHECKSOL);
      k_checksol_rounds<<<1, 1024, 0, s>>>(a, pf);
      T.mark(s, KC_CHECKSERIAL);
      k_fixup_compute<<<grid2(n1, n2, b), b, 0, s>>>(a, pf);
      T.mark(s, KC_FIXC);
      launch_bound_fix(mixed, grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, s, a, pf, last ? 1 : 0);
      T.mark(s, KC_FIXA);
      if (last) step_ended = true;
      continue;
    }
    k_bound<<<grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, 0, s>>>(a, pf, 1);
    T.mark(s, KC_BOUND);
    // force-free: no b^2 flags (so no check-solution votes) and no
    // fixup_utoprim (fixup.c:542); the second bound would repeat the first
    if (ffde) {
      if (poledeath) {
        k_poledeath<<<dim3((n1 + 127) / 128, 2), 128, 0, s>>>(a, pf);
        T.mark(s, KC_POLE);
      }
      if (rec) cudaMemcpyAsync(rec->snap[sub], pf, pbytes, cudaMemcpyDeviceToDevice, s);
      continue;
    }
    // the adjoint's recording keeps the states between the bounds, the
    // zeroing and the repairs, so it runs them as separate kernels (the
    // POLEDEATH zeroing after the first bound inside k_gammacheck)
    k_gammacheck<<<grid2(n1 + 2, n2 + 2, b), b, 0, s>>>(a, pf, poledeath ? 1 : 0);
    T.mark(s, KC_GCHECK);
    cudaMemcpyAsync(rec->snap[sub], pf, pbytes, cudaMemcpyDeviceToDevice, s);
    k_checksol<<<grid2(n1, n2, b), b, 0, s>>>(a, pf, 0);
    T.mark(s, KC_CHECKSOL);
    k_checksol_rounds<<<1, 1024, 0, s>>>(a, pf);
    T.mark(s, KC_CHECKSERIAL);
    k_fixup_compute<<<grid2(n1, n2, b), b, 0, s>>>(a, pf);
    T.mark(s, KC_FIXC);
    k_fixup_apply<<<grid2(n1, n2, b), b, 0, s>>>(a, pf, 1);
    cudaMemcpyAsync(rec->pre2[sub], pf, pbytes, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(rec->flag[sub], c->d_pflag, fbytes, cudaMemcpyDeviceToDevice, s);
    k_bound<<<grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, 0, s>>>(a, pf, 0);
    if (poledeath) k_poledeath<<<dim3((n1 + 127) / 128, 2), 128, 0, s>>>(a, pf);
  }
  a = a0;
  if (rec) cudaMemcpyAsync(rec->ph, c->d_pk0, pbytes, cudaMemcpyDeviceToDevice, s);
  if (c->cfg.currents) {
    // step_ch.c:143-156: Faraday slots and J^mu at the new time
    k_faraday<<<grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, 0, s>>>(a, c->d_p);
    T.mark(s, KC_FARADAY);
    k_current<<<grid2(n1 + 2 * NG - 2, n2 + 2 * NG - 2, b), b, 0, s>>>(a);
    k_currents_commit<<<1, 1, 0, s>>>(a);
    T.mark(s, KC_CURRENT, 2);
  }
  // horizon accounting and the new dt (unless the last k_bound_fix did it)
  if (!step_ended) {
    launch_step_end(c->cfg.precision == HARM_PREC_MIXED, s, a, c->d_p);
    T.mark(s, KC_DT);
  }
  return cudaGetLastError() == cudaSuccess ? HARM_OK : HARM_ECUDA;
}

extern "C" {

const char* harm_error_string(int code)
{
  switch (code) {
    case HARM_OK: return "ok";
    case HARM_EINVAL: return "invalid argument";
    case HARM_ENODEVICE: return "no usable CUDA device (sm_100 required)";
    case HARM_ECUDA: return "CUDA runtime error";
    case HARM_ENOMEM: return "device allocation failed";
    case HARM_EGEOMETRY: return "geometry tables missing or not symmetric";
    case HARM_EFAIL: return "fatal check of the reference step fired";
    default: return "unknown error";
  }
}

int harm_create(const harm_config* cfg, void* stream, harm_ctx** out)
{
  if (!cfg || !out) return HARM_EINVAL;
  *out = nullptr;
  if (cfg->n1 < 4 || cfg->n2 < 4) return HARM_EINVAL;
  if (cfg->precision != HARM_PREC_FP64 && cfg->precision != HARM_PREC_MIXED) return HARM_EINVAL;
  if (cfg->lim != HARM_LIM_MC && cfg->lim != HARM_LIM_PARA) return HARM_EINVAL;
  if (cfg->fluxmethod != HARM_FLUX_HLL && cfg->fluxmethod != HARM_FLUX_LAXF) return HARM_EINVAL;
  if (cfg->eom != HARM_EOM_GRMHD && cfg->eom != HARM_EOM_FFDE) return HARM_EINVAL;
  if (cfg->bc != HARM_BC_TORUS && cfg->bc != HARM_BC_STAR) return HARM_EINVAL;
  if ((cfg->tryagain != 0 && cfg->tryagain != 1) || (cfg->tryagain && cfg->eom != HARM_EOM_GRMHD)) return HARM_EINVAL;
  if (cfg->fluxadjust < 0 || cfg->fluxadjust > 3 || (cfg->fluxadjust && !(cfg->gammadamp > 0.0))) return HARM_EINVAL;
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HARM_ENODEVICE;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major != 10) return HARM_ENODEVICE;
  harm_ctx* c = new harm_ctx();
  memset(c, 0, sizeof(*c));
  c->cfg = *cfg;
  c->stream = (cudaStream_t)stream;
  c->n1m = cfg->n1 + 2 * NG;
  c->n2m = cfg->n2 + 2 * NG;
  c->gr.n1 = cfg->n1;
  c->gr.n2 = cfg->n2;
  c->gr.pitch = ((c->n1m + 15) / 16) * 16;
  c->gr.rows = c->n2m;
  c->gr.plane = (long long)c->gr.pitch * c->gr.rows;
  const size_t pd = (size_t)c->gr.plane * sizeof(double);
  const dim3 b(32, 4);
  c->flux_by = flux_rows(cfg->n1, cfg->n2, cfg->precision == HARM_PREC_MIXED);
  dim3 gf = flux_grid(cfg->n1, cfg->n2, c->flux_by);
  c->nblocks_flux = gf.x * gf.y;
  c->tile_update = dim3(32, 4);
  c->tile_small = dim3(32, 4);
  bool ok = true;
  ok &= cudaMalloc(&c->d_p, NPR * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_pk0, NPR * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_geo, GEO_NPLANES * pd) == cudaSuccess;
  if (cfg->precision == HARM_PREC_MIXED)
    ok &= cudaMalloc(&c->d_geo32, 2 * GEO_PER_LOC * (size_t)c->gr.plane * sizeof(float)) == cudaSuccess;
  ok &= cudaMalloc(&c->d_F1, NPR * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_F2, NPR * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_emf, pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_gammacheck, pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_fixbuf, 5 * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_blockmin, 2 * (size_t)c->nblocks_flux * sizeof(double)) == cudaSuccess;
  ok &= cudaMalloc(&c->d_pflag, (size_t)c->gr.plane * sizeof(int)) == cudaSuccess;
  ok &= cudaMalloc(&c->d_bsqf, (size_t)c->gr.plane) == cudaSuccess;
  ok &= cudaMalloc(&c->d_chk, 2 * (size_t)c->gr.plane) == cudaSuccess;
  if (cfg->fluxadjust) ok &= cudaMalloc(&c->d_fluxf, (size_t)c->gr.plane) == cudaSuccess;
  ok &= cudaMalloc(&c->d_sc, sizeof(DevScalars)) == cudaSuccess;
  ok &= cudaMalloc(&c->d_ubuf, NPR * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_worklist, (size_t)c->gr.plane * sizeof(int)) == cudaSuccess;
  if (cfg->currents) ok &= cudaMalloc(&c->d_cur, (size_t)CUR_NPLANES * pd) == cudaSuccess;
  ok &= cudaMalloc(&c->d_stage, (size_t)c->n1m * c->n2m * NPR * sizeof(double)) == cudaSuccess;
  ok &= cudaMalloc(&c->d_stagef, (size_t)c->n1m * c->n2m * 5 * sizeof(int)) == cudaSuccess;
  if (!ok) {
    harm_destroy(c);
    return HARM_ENOMEM;
  }
  if (!encode_geo_map(&c->geo_map, c->d_geo, c->gr, c->tile_update) ||
      !encode_prim_map(&c->map_p, c->d_p, c->gr, c->flux_by) || !encode_prim_map(&c->map_pk0, c->d_pk0, c->gr, c->flux_by)) {
    fprintf(stderr, "harm_b200: a TMA map (geometry or state planes) could not be encoded\n");
    harm_destroy(c);
    return HARM_ECUDA;
  }
  cudaMemsetAsync(c->d_p, 0, NPR * pd, c->stream);
  cudaMemsetAsync(c->d_pk0, 0, NPR * pd, c->stream);
  cudaMemsetAsync(c->d_geo, 0, GEO_NPLANES * pd, c->stream);
  cudaMemsetAsync(c->d_F1, 0, NPR * pd, c->stream);
  cudaMemsetAsync(c->d_F2, 0, NPR * pd, c->stream);
  cudaMemsetAsync(c->d_emf, 0, pd, c->stream);
  cudaMemsetAsync(c->d_gammacheck, 0, pd, c->stream);
  cudaMemsetAsync(c->d_fixbuf, 0, 5 * pd, c->stream);
  cudaMemsetAsync(c->d_pflag, 0, (size_t)c->gr.plane * sizeof(int), c->stream);
  cudaMemsetAsync(c->d_bsqf, 0, (size_t)c->gr.plane, c->stream);
  cudaMemsetAsync(c->d_chk, 0, 2 * (size_t)c->gr.plane, c->stream);
  if (c->d_fluxf) cudaMemsetAsync(c->d_fluxf, 0, (size_t)c->gr.plane, c->stream);
  cudaMemsetAsync(c->d_sc, 0, sizeof(DevScalars), c->stream);
  if (c->d_cur) cudaMemsetAsync(c->d_cur, 0, (size_t)CUR_NPLANES * pd, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    harm_destroy(c);
    return HARM_ECUDA;
  }
  *out = c;
  return HARM_OK;
}

void harm_destroy(harm_ctx* c)
{
  if (!c) return;
  if (c->have_graph) {
    cudaGraphExecDestroy(c->gexec);
    cudaGraphDestroy(c->graph);
  }
  cudaFree(c->d_p);
  cudaFree(c->d_pk0);
  cudaFree(c->d_geo);
  cudaFree(c->d_geo32);
  cudaFree(c->d_F1);
  cudaFree(c->d_F2);
  cudaFree(c->d_emf);
  cudaFree(c->d_gammacheck);
  cudaFree(c->d_fixbuf);
  cudaFree(c->d_blockmin);
  cudaFree(c->d_pflag);
  cudaFree(c->d_bsqf);
  cudaFree(c->d_chk);
  cudaFree(c->d_fluxf);
  cudaFree(c->d_sc);
  cudaFree(c->d_ubuf);
  cudaFree(c->d_worklist);
  cudaFree(c->d_cur);
  cudaFree(c->d_stage);
  cudaFree(c->d_stagef);
  delete c;
}

int harm_upload_geometry(harm_ctx* c, const double* gcov, const double* gcon, const double* gdet, const double* conn,
                         const double* floors)
{
  if (!c || !gcov || !gcon || !gdet || !conn || !floors) return HARM_EINVAL;
  const int n1m = c->n1m, n2m = c->n2m;
  const long long pl = c->gr.plane;
  std::vector<double> h((size_t)GEO_NPLANES * pl, 0.0);
  for (int ii = 0; ii < n1m; ii++)
    for (int jj = 0; jj < n2m; jj++) {
      const long long zr = (long long)ii * n2m + jj;                 // reference zone
      const long long zd = c->gr.at(ii - NG, jj - NG);               // device zone
      for (int loc = 0; loc < 4; loc++) {
        const double* gv = gcov + (zr * 4 + loc) * 16;
        const double* gn = gcon + (zr * 4 + loc) * 16;
        for (int a = 0; a < 4; a++)
          for (int b = a; b < 4; b++) {
            // the step kernels use the packed symmetric form; the reference
            // reads both triangles, so they must agree bit for bit
            if (gv[a * 4 + b] != gv[b * 4 + a] || gn[a * 4 + b] != gn[b * 4 + a]) return HARM_EGEOMETRY;
            h[((size_t)loc * GEO_PER_LOC + sym(a, b)) * pl + zd] = gv[a * 4 + b];
            h[((size_t)loc * GEO_PER_LOC + 10 + sym(a, b)) * pl + zd] = gn[a * 4 + b];
          }
        h[((size_t)loc * GEO_PER_LOC + 20) * pl + zd] = gdet[zr * 4 + loc];
      }
      const double* cn = conn + zr * 64;
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++)
          for (int j = l; j < 4; j++) {
            if (cn[(k * 4 + l) * 4 + j] != cn[(k * 4 + j) * 4 + l]) return HARM_EGEOMETRY;
            h[(size_t)conn_plane(k, l, j) * pl + zd] = cn[(k * 4 + l) * 4 + j];
          }
      h[(size_t)GEO_FLOOR * pl + zd] = floors[zr * 2 + 0];
      h[(size_t)(GEO_FLOOR + 1) * pl + zd] = floors[zr * 2 + 1];
    }
  CK(cudaMemcpyAsync(c->d_geo, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  std::vector<float> h32;
  if (c->d_geo32) {
    // FP32 copies of the two face locations (FACE1, FACE2 are the first 42 planes)
    h32.resize((size_t)2 * GEO_PER_LOC * pl);
    for (size_t k = 0; k < h32.size(); k++) h32[k] = (float)h[k];
    CK(cudaMemcpyAsync(c->d_geo32, h32.data(), h32.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->geo_ok = true;
  return HARM_OK;
}

int harm_set_prims(harm_ctx* c, const double* prims, const int* pflag, int reset_gammacheck)
{
  if (!c || !prims) return HARM_EINVAL;
  const size_t nz = (size_t)c->n1m * c->n2m;
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  // one contiguous host->device copy, then the layout change on the device
  CK(cudaMemcpyAsync(c->d_stage, prims, nz * NPR * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (pflag) CK(cudaMemcpyAsync(c->d_stagef, pflag, nz * 5 * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  else CK(cudaMemsetAsync(c->d_pflag, 0, (size_t)c->gr.plane * sizeof(int), c->stream));
  k_ref_to_planes<<<grid2(c->n1m, c->n2m, b), b, 0, c->stream>>>(a, c->d_stage, pflag ? c->d_stagef : nullptr, c->d_p);
  CK(cudaGetLastError());
  if (reset_gammacheck) CK(cudaMemsetAsync(c->d_gammacheck, 0, (size_t)c->gr.plane * sizeof(double), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return HARM_OK;
}

int harm_get_prims(harm_ctx* c, double* prims, int* pflag)
{
  if (!c) return HARM_EINVAL;
  const size_t nz = (size_t)c->n1m * c->n2m;
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  k_planes_to_ref<<<grid2(c->n1m, c->n2m, b), b, 0, c->stream>>>(a, c->d_p, c->d_stage, pflag ? c->d_stagef : nullptr);
  CK(cudaGetLastError());
  if (prims) CK(cudaMemcpyAsync(prims, c->d_stage, nz * NPR * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (pflag) CK(cudaMemcpyAsync(pflag, c->d_stagef, nz * 5 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return HARM_OK;
}

int harm_bound_prims(harm_ctx* c)
{
  if (!c) return HARM_EINVAL;
  if (!c->geo_ok) return HARM_EGEOMETRY;
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  k_bound<<<grid2(c->cfg.n1 + 2 * NG, c->cfg.n2 + 2 * NG, b), b, 0, c->stream>>>(a, c->d_p, 1);
  // POLEDEATH belongs to the torus's bound (bounds.fishmon.c); the star's
  // (bounds.ns.c) keeps the first and last rows as they are
  if (c->cfg.bc == HARM_BC_TORUS) k_poledeath<<<dim3((c->cfg.n1 + 127) / 128, 2), 128, 0, c->stream>>>(a, c->d_p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return HARM_OK;
}

int harm_invert_zones(harm_ctx* c, int which, int nz, const int* zones, const double* U, double* pr, int* pflag)
{
  if (!c || nz < 0 || (nz > 0 && (!zones || !U || !pr || !pflag))) return HARM_EINVAL;
  if (c->cfg.eom != HARM_EOM_GRMHD || which < -1 || which == 1 || which > 7) return HARM_EINVAL;
  for (int k = 0; k < nz; k++)
    if (zones[2 * k] < 0 || zones[2 * k] >= c->cfg.n1 || zones[2 * k + 1] < 0 || zones[2 * k + 1] >= c->cfg.n2)
      return HARM_EINVAL;
  if (nz == 0) return HARM_OK;
  int* dz = nullptr;
  double *dU = nullptr, *dp = nullptr;
  int* df = nullptr;
  int rc = HARM_OK;
  const size_t nd = (size_t)NPR * nz * sizeof(double);
  if (cudaMalloc(&dz, 2 * nz * sizeof(int)) != cudaSuccess || cudaMalloc(&dU, nd) != cudaSuccess ||
      cudaMalloc(&dp, nd) != cudaSuccess || cudaMalloc(&df, nz * sizeof(int)) != cudaSuccess)
    rc = HARM_ENOMEM;
  cudaStream_t s = c->stream;
  if (rc == HARM_OK) {
    cudaMemcpyAsync(dz, zones, 2 * nz * sizeof(int), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dU, U, nd, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dp, pr, nd, cudaMemcpyHostToDevice, s);
    k_invert_zones<<<(nz + 63) / 64, 64, 0, s>>>(c->args(), which, nz, dz, dU, dp, df);
    cudaMemcpyAsync(pr, dp, nd, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(pflag, df, nz * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = HARM_ECUDA;
  }
  cudaFree(dz);
  cudaFree(dU);
  cudaFree(dp);
  cudaFree(df);
  return rc;
}

int harm_set_time(harm_ctx* c, double t, double dt, long long realnstep)
{
  if (!c) return HARM_EINVAL;
  DevScalars h;
  memset(&h, 0, sizeof(h));
  h.t = t;
  h.dt = dt;
  h.dt_free = dt;
  h.realnstep = realnstep;
  CK(cudaMemcpyAsync(c->d_sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  if (c->cfg.currents) {
    // the t = 0 evaluation of initbase.c:653-658 on the uploaded state, from
    // cleared slots (the reference's arrays start at zero)
    const StepArgs a = c->args();
    const dim3 b(32, 4);
    CK(cudaMemsetAsync(c->d_cur, 0, (size_t)CUR_NPLANES * c->gr.plane * sizeof(double), c->stream));
    k_faraday<<<grid2(c->cfg.n1 + 2 * NG, c->cfg.n2 + 2 * NG, b), b, 0, c->stream>>>(a, c->d_p);
    k_current<<<grid2(c->cfg.n1 + 2 * NG - 2, c->cfg.n2 + 2 * NG - 2, b), b, 0, c->stream>>>(a);
    k_currents_commit<<<1, 1, 0, c->stream>>>(a);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  return HARM_OK;
}

int harm_set_end_time(harm_ctx* c, double tf)
{
  if (!c || !(tf == tf)) return HARM_EINVAL;
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->d_sc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // the clamp of step_ch.c:183 redone for the new end time on the unclamped dt
  h.dt = (h.t + h.dt_free > tf) ? tf - h.t : h.dt_free;
  CK(cudaMemcpyAsync(c->d_sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->cfg.tf = tf;
  if (c->have_graph) {  // the end time is a launch parameter of the captured step
    cudaGraphExecDestroy(c->gexec);
    cudaGraphDestroy(c->graph);
    c->have_graph = false;
  }
  return HARM_OK;
}

int harm_step(harm_ctx* c, int nsteps)
{
  if (!c || nsteps < 0) return HARM_EINVAL;
  if (!c->geo_ok) return HARM_EGEOMETRY;
  if (!c->have_graph) {
    cudaStream_t cap = c->stream;
    bool own = false;
    if (cap == 0) {
      // the legacy default stream cannot be captured: capture on a private one
      CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      own = true;
    }
    harm_ctx tmp = *c;
    tmp.stream = cap;
    CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(&tmp);
    cudaGraph_t g;
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    if (own) cudaStreamDestroy(cap);
    if (rc != HARM_OK || e != cudaSuccess) return HARM_ECUDA;
    CK(cudaGraphInstantiate(&c->gexec, g, 0));
    c->graph = g;
    c->have_graph = true;
  }
  for (int n = 0; n < nsteps; n++) CK(cudaGraphLaunch(c->gexec, c->stream));
  return HARM_OK;
}

// the run state of the device scalars; the first fatal check is decoded
// from its key (fail_key: step, phase, position in the phase's loop, code)
static void fill_status(const DevScalars& h, int n1, int n2, harm_status* st)
{
  if (!st) return;
  const unsigned long long key = ~h.fail_inv;
  st->fail_code = 0;
  st->fail_i = st->fail_j = 0;
  st->fail_step = -1;
  if (h.fail_inv) {
    const int phase = (int)((key >> 36) & 15) % PH_PER_SUBSTEP;
    const unsigned o = (unsigned)((key >> 6) & 0x3fffffffu);
    st->fail_code = (int)(key & 63);
    st->fail_step = (long long)(key >> 40);
    if (phase == PH_BOUND1 || phase == PH_BOUND2) {
      const bool outer = o >= (unsigned)(n2 * NG);
      const unsigned r = outer ? o - (unsigned)(n2 * NG) : o;
      st->fail_j = (int)(r / NG);
      st->fail_i = outer ? n1 + (int)(r % NG) : -1 - (int)(r % NG);
    } else {
      st->fail_i = (int)(o >> 15) - NG;
      st->fail_j = (int)(o & 0x7fff) - NG;
    }
  }
  st->fixups = h.fixups;
  st->realnstep = h.realnstep;
  st->t = h.t;
  st->dt = h.dt;
  st->newton_iters = h.newton_iters;
  st->chk_multi = h.chk_multi;
  st->deferred = h.ndeferred_total;
}

int harm_sync(harm_ctx* c, harm_status* st)
{
  if (!c) return HARM_EINVAL;
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->d_sc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  fill_status(h, c->cfg.n1, c->cfg.n2, st);
  return h.fail_inv ? HARM_EFAIL : HARM_OK;
}

int harm_get_currents(harm_ctx* c, double* jcon, double* fcon, double* cfaraday)
{
  if (!c) return HARM_EINVAL;
  if (!c->cfg.currents) return HARM_EINVAL;
  const long long pl = c->gr.plane;
  std::vector<double> h((size_t)CUR_NPLANES * pl);
  DevScalars sc;
  CK(cudaMemcpyAsync(&sc, c->d_sc, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(h.data(), c->d_cur, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // reference slots: 0 = newest F^{it}, 4 = the previous, 3 = two back
  const int lev[5] = {sc.cur_ring, -1, -1, (sc.cur_ring + 1) % 3, (sc.cur_ring + 2) % 3};
  for (int ii = 0; ii < c->n1m; ii++)
    for (int jj = 0; jj < c->n2m; jj++) {
      const long long zd = (long long)jj * c->gr.pitch + ii, zr = (long long)ii * c->n2m + jj;
      if (jcon)
        for (int k = 0; k < 4; k++) jcon[zr * 4 + k] = h[(CUR_JCON + k) * pl + zd];
      if (fcon)
        for (int k = 0; k < 6; k++) fcon[zr * 6 + k] = h[(CUR_FCON + k) * pl + zd];
      if (cfaraday)
        for (int sl = 0; sl < 5; sl++)
          for (int k = 0; k < 3; k++) {
            const int plane = (sl == 1) ? CUR_S1 + k : (sl == 2) ? CUR_S2 + k : CUR_RING + 3 * lev[sl] + k;
            cfaraday[(zr * 5 + sl) * 3 + k] = h[plane * pl + zd];
          }
    }
  return HARM_OK;
}

int harm_write_dump(harm_ctx* c, const char* path, const harm_dump_header* hdr, const double* coords)
{
  if (!c || !path || !hdr || !coords || !c->cfg.currents) return HARM_EINVAL;
  const int n1 = c->cfg.n1, n2 = c->cfg.n2;
  const size_t nz = (size_t)n1 * n2;
  double* d_out = nullptr;
  int* d_nf = nullptr;
  CK(cudaMalloc(&d_out, nz * DUMP_DYNCOLS * sizeof(double)));
  if (cudaMalloc(&d_nf, sizeof(int)) != cudaSuccess) {
    cudaFree(d_out);
    return HARM_ENOMEM;
  }
  std::vector<double> cols(nz * DUMP_DYNCOLS);
  DevScalars sc;
  int nf = 0;
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  cudaError_t e = cudaMemsetAsync(d_nf, 0, sizeof(int), c->stream);
  if (e == cudaSuccess) {
    k_dump_columns<<<grid2(n1, n2, b), b, 0, c->stream>>>(a, c->d_p, d_out, d_nf);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cols.data(), d_out, cols.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nf, d_nf, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&sc, c->d_sc, sizeof(sc), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_out);
  cudaFree(d_nf);
  if (e != cudaSuccess) {
    fprintf(stderr, "harm_b200: harm_write_dump: %s\n", cudaGetErrorString(e));
    return HARM_ECUDA;
  }
  if (nf) return HARM_EFAIL;
  FILE* f = fopen(path, "wt");
  if (!f) return HARM_EINVAL;
  fprintf(f,
          "%21.15g %d %d %21.15g %21.15g %21.15g %21.15g %ld %21.15g %21.15g %21.15g %21.15g %21.15g %21.15g %21.15g "
          "%d\n",
          sc.t, n1, n2, hdr->startx1, hdr->startx2, c->cfg.dx1, c->cfg.dx2, (long)sc.realnstep, c->cfg.gam, hdr->a,
          hdr->R0, hdr->Rin, hdr->Rout, hdr->hslope, sc.dt, hdr->defcoord);
  // rows formatted in parallel chunks, written in order
  const int nth = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::string> chunk(nth);
  std::vector<std::thread> th;
  const int n2m = n2 + 2 * NG;
  for (int t = 0; t < nth; t++)
    th.emplace_back([&, t]() {
      const size_t lo = nz * t / nth, hi = nz * (t + 1) / nth;
      std::string& s = chunk[t];
      s.reserve((hi - lo) * 56 * 22 + 16);
      char buf[64];
      for (size_t zz = lo; zz < hi; zz++) {
        const int j = (int)(zz / n1), i = (int)(zz % n1);
        const double* xr = coords + ((size_t)(i + NG) * n2m + (j + NG)) * 4;
        const double head[6] = {(double)i, (double)j, xr[0], xr[1], xr[2], xr[3]};
        for (int k = 0; k < 6; k++) s.append(buf, snprintf(buf, sizeof(buf), "%21.15g ", head[k]));
        const double* v = cols.data() + zz * DUMP_DYNCOLS;
        for (int k = 0; k < DUMP_DYNCOLS; k++) s.append(buf, snprintf(buf, sizeof(buf), "%21.15g ", v[k]));
        s.push_back('\n');
      }
    });
  for (auto& x : th) x.join();
  bool ok = true;
  for (auto& s : chunk) ok &= fwrite(s.data(), 1, s.size(), f) == s.size();
  ok &= fclose(f) == 0;
  return ok ? HARM_OK : HARM_EINVAL;
}

static void drop_graph(harm_ctx* c)
{
  if (c->have_graph) {
    cudaGraphExecDestroy(c->gexec);
    cudaGraphDestroy(c->graph);
    c->have_graph = false;
  }
}

int harm_set_tiles(harm_ctx* c, const harm_tiles* t)
{
  if (!c || !t) return HARM_EINVAL;
  const long long nu = (long long)t->update_x * t->update_y, ns = (long long)t->small_x * t->small_y;
  if (t->update_x < 2 || (t->update_x & 1) || t->update_y < 1 || nu > 128 || t->small_x < 1 || t->small_y < 1 ||
      ns > 1024)
    return HARM_EINVAL;
  CK(cudaStreamSynchronize(c->stream));
  CUtensorMap m;
  if (!encode_geo_map(&m, c->d_geo, c->gr, dim3(t->update_x, t->update_y))) return HARM_ECUDA;
  c->geo_map = m;
  c->tile_update = dim3(t->update_x, t->update_y);
  c->tile_small = dim3(t->small_x, t->small_y);
  drop_graph(c);
  return HARM_OK;
}

int harm_get_tiles(harm_ctx* c, harm_tiles* t)
{
  if (!c || !t) return HARM_EINVAL;
  t->update_x = c->tile_update.x;
  t->update_y = c->tile_update.y;
  t->small_x = c->tile_small.x;
  t->small_y = c->tile_small.y;
  return HARM_OK;
}

// ---------------------------------------------------------------- ensembles
struct harm_ensemble {
  std::vector<harm_ctx*> m;
  int per_launch;
  cudaStream_t stream;
  bool own_stream;
  cudaGraph_t graph;
  cudaGraphExec_t gexec;
};

void harm_ensemble_destroy(harm_ensemble* e)
{
  if (!e) return;
  cudaStreamSynchronize(e->stream);
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->own_stream) cudaStreamDestroy(e->stream);
  delete e;
}

int harm_ensemble_create(harm_ctx* const* members, int n, int per_launch, void* stream, harm_ensemble** out)
{
  if (!members || n < 1 || per_launch < 1 || !out) return HARM_EINVAL;
  for (int k = 0; k < n; k++)
    if (!members[k] || !members[k]->geo_ok) return HARM_EINVAL;
  harm_ensemble* e = new harm_ensemble();
  e->m.assign(members, members + n);
  e->per_launch = per_launch;
  e->stream = (cudaStream_t)stream;
  e->own_stream = false;
  e->graph = nullptr;
  e->gexec = nullptr;
  if (!e->stream) {
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete e;
      return HARM_ECUDA;
    }
    e->own_stream = true;
  }
  // members' pending work (uploads, set-up) completes before the first launch
  for (int k = 0; k < n; k++)
    if (cudaStreamSynchronize(members[k]->stream) != cudaSuccess) {
      harm_ensemble_destroy(e);
      return HARM_ECUDA;
    }
  // capture: fork from the ensemble stream into one branch stream per
  // member, each branch the member's step sequence, joined at the end
  std::vector<cudaStream_t> br(n, nullptr);
  std::vector<cudaEvent_t> ev(n + 1, nullptr);
  int rc = HARM_OK;
  bool ok = true;
  for (int k = 0; k < n && ok; k++) ok = cudaStreamCreateWithFlags(&br[k], cudaStreamNonBlocking) == cudaSuccess;
  for (int k = 0; k <= n && ok; k++) ok = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) == cudaSuccess;
  if (ok) ok = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    bool cap_ok = cudaEventRecord(ev[n], e->stream) == cudaSuccess;
    for (int k = 0; k < n && cap_ok; k++) {
      cap_ok = cudaStreamWaitEvent(br[k], ev[n], 0) == cudaSuccess;
      harm_ctx tmp = *e->m[k];
      tmp.stream = br[k];
      for (int sidx = 0; sidx < per_launch && cap_ok; sidx++) cap_ok = enqueue_step(&tmp) == HARM_OK;
      if (cap_ok) cap_ok = cudaEventRecord(ev[k], br[k]) == cudaSuccess;
      if (cap_ok) cap_ok = cudaStreamWaitEvent(e->stream, ev[k], 0) == cudaSuccess;
    }
    cudaGraph_t g = nullptr;
    const bool end_ok = cudaStreamEndCapture(e->stream, &g) == cudaSuccess;
    ok = cap_ok && end_ok;
    if (ok) ok = cudaGraphInstantiate(&e->gexec, g, 0) == cudaSuccess;
    e->graph = g;
  }
  for (int k = 0; k < n; k++)
    if (br[k]) cudaStreamDestroy(br[k]);
  for (int k = 0; k <= n; k++)
    if (ev[k]) cudaEventDestroy(ev[k]);
  if (!ok) {
    fprintf(stderr, "harm_b200: harm_ensemble_create: graph capture failed (%s)\n",
            cudaGetErrorString(cudaGetLastError()));
    harm_ensemble_destroy(e);
    return HARM_ECUDA;
  }
  (void)rc;
  *out = e;
  return HARM_OK;
}

int harm_ensemble_step(harm_ensemble* e, int nsteps)
{
  if (!e || nsteps < 0 || nsteps % e->per_launch) return HARM_EINVAL;
  for (int k = 0; k < nsteps / e->per_launch; k++) CK(cudaGraphLaunch(e->gexec, e->stream));
  return HARM_OK;
}

int harm_ensemble_sync(harm_ensemble* e, harm_status* st)
{
  if (!e) return HARM_EINVAL;
  CK(cudaStreamSynchronize(e->stream));
  int worst = HARM_OK;
  for (size_t k = 0; k < e->m.size(); k++) {
    harm_status s;
    const int rc = harm_sync(e->m[k], &s);
    if (st) st[k] = s;
    if (rc == HARM_EFAIL) worst = HARM_EFAIL;
    else if (rc != HARM_OK) return rc;
  }
  return worst;
}

// ---------------------------------------------------------------- adjoint
namespace {

// The reverse pass keeps two record sets: while the adjoint of one
// checkpoint segment runs from one set (on its own stream), the replay of
// the segment before it records into the other (on the context's stream).
struct AdjWork {
  std::vector<void*> mem;
  std::vector<Rec> rec[2];        // one per step of a checkpoint segment, per set
  std::vector<double*> pnext[2];  // the state after each slot's step (the next slot's pn; an extra one at the end)
  std::vector<cudaGraphExec_t> recg[2];  // the recording step of each slot, captured
  std::vector<cudaGraphExec_t> adjg[2];  // the adjoint step of each slot, captured
  double *La, *Lc, *Lb, *Lsnap, *LdU, *Le, *Sr, *dts, *dot;
  DevScalars* sc_adj;  // the adjoint stream's scalars (its steps' dt), apart from the replay's
  bool ok = true;
  void* get(size_t bytes)
  {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    mem.push_back(p);
    return p;
  }
  ~AdjWork()
  {
    for (int x = 0; x < 2; x++) {
      for (cudaGraphExec_t g : recg[x])
        if (g) cudaGraphExecDestroy(g);
      for (cudaGraphExec_t g : adjg[x])
        if (g) cudaGraphExecDestroy(g);
    }
    for (void* p : mem) cudaFree(p);
  }
};

// the step's state the adjoint restores: p and the check-solution gamma table
struct Saved {
  double* p;
  double* gc;
};

// blocks of k_dot_active (one partial sum each)
size_t dot_blocks(const harm_ctx* c)
{
  const dim3 g = grid2(c->cfg.n1, c->cfg.n2, dim3(32, 4));
  return (size_t)g.x * g.y;
}

// nslots: steps per checkpoint segment.  Each keeps its own record, about
// 10 state-sized arrays, in each of the two sets: a 16-step segment of a
// 512^2 grid holds ~3 GB per set.  nsets: 2 when there is more than one
// segment (replay and adjoint overlap), else 1.
int adj_alloc(harm_ctx* c, AdjWork& w, int nsteps, int nslots, int nsets)
{
  const size_t pl = (size_t)c->gr.plane, P = NPR * pl * sizeof(double);
  for (int x = 0; x < nsets; x++) {
    w.rec[x].resize(nslots);
    for (Rec& r : w.rec[x]) {
      r.pn = (double*)w.get(P);
      r.ph = (double*)w.get(P);
      for (int s = 0; s < 2; s++) {
        r.pinv[s] = (double*)w.get(P);
        r.upd[s] = (double*)w.get(P);
        r.snap[s] = (double*)w.get(P);
        r.pre2[s] = (double*)w.get(P);
        r.flaginv[s] = (int*)w.get(pl * sizeof(int));
        r.flag[s] = (int*)w.get(pl * sizeof(int));
        r.fixset[s] = (unsigned char*)w.get(pl);
      }
    }
    double* plast = (double*)w.get(P);
    for (int m = 0; m < nslots; m++) w.pnext[x].push_back(m + 1 < nslots ? w.rec[x][m + 1].pn : plast);
  }
  w.sc_adj = (DevScalars*)w.get(sizeof(DevScalars));
  w.La = (double*)w.get(P);
  w.Lc = (double*)w.get(P);
  w.Lb = (double*)w.get(P);
  w.Lsnap = (double*)w.get(P);
  w.LdU = (double*)w.get(P);
  w.Sr = (double*)w.get(P);
  w.Le = (double*)w.get(pl * sizeof(double));
  w.dts = (double*)w.get((size_t)nsteps * sizeof(double));
  w.dot = (double*)w.get(dot_blocks(c) * sizeof(double));
  return w.ok ? HARM_OK : HARM_ENOMEM;
}

void save_state(harm_ctx* c, const Saved& s)
{
  const size_t pl = (size_t)c->gr.plane;
  cudaMemcpyAsync(s.p, c->d_p, NPR * pl * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(s.gc, c->d_gammacheck, pl * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
}

void load_state(harm_ctx* c, const Saved& s)
{
  const size_t pl = (size_t)c->gr.plane;
  cudaMemcpyAsync(c->d_p, s.p, NPR * pl * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_gammacheck, s.gc, pl * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
}

// one substep's adjoint: lam_in (the substep output's adjoint, ghosts
// included; consumed) -> lam_pi_acc (+=, pi), out (the pb adjoint, set).
// The update's c dt is cfac times the step's dt (a.sc->dt).
void adjoint_substep(harm_ctx* c, AdjWork& w, const Rec& r, int sub, double* lam_in, double* out, const double* pi,
                     const double* pb, double cfac, double seed_fac, double* lam_pi_acc)
{
  const StepArgs a = c->args();
  const int n1 = c->cfg.n1, n2 = c->cfg.n2;
  const dim3 b(32, 4);
  cudaStream_t s = c->stream;
  const size_t P = (size_t)NPR * c->gr.plane * sizeof(double);
  k_adj_poledeath<<<dim3((n1 + 127) / 128, 2), 128, 0, s>>>(a, lam_in);
  k_adj_ghosts<<<grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, 0, s>>>(a, lam_in, r.pre2[sub]);
  cudaMemsetAsync(w.Lsnap, 0, P, s);
  k_adj_fixup<<<grid2(n1, n2, b), b, 0, s>>>(a, lam_in, w.Lsnap, r.snap[sub], r.flag[sub], r.fixset[sub]);
  k_adj_poledeath<<<dim3((n1 + 127) / 128, 2), 128, 0, s>>>(a, w.Lsnap);
  k_adj_ghosts<<<grid2(n1 + 2 * NG, n2 + 2 * NG, b), b, 0, s>>>(a, w.Lsnap, r.upd[sub]);
  cudaMemsetAsync(out, 0, P, s);
  k_adj_update<<<grid2(n1, n2, b), b, 0, s>>>(a, w.Lsnap, r.pinv[sub], r.flaginv[sub], cfac, w.Sr, w.LdU);
  k_adj_upi<<<grid2(n1, n2, b), b, 0, s>>>(a, w.Sr, pi, lam_pi_acc);
  k_adj_source<<<grid2(n1, n2, b), b, 0, s>>>(a, pb, w.LdU, out);
  k_adj_corner<<<grid2(n1 + 1, n2 + 1, b), b, 0, s>>>(a, w.LdU, w.Le);
  // the face-state adjoints go to Lsnap (free after the update) and Sr
  k_adj_faces<1><<<grid2(n1 + 1, n2 + 2, b), b, 0, s>>>(a, pb, w.LdU, w.Le, w.Lsnap, w.Sr, seed_fac);
  k_adj_recon<1><<<grid2(n1 + 2, n2 + 2, b), b, 0, s>>>(a, pb, w.Lsnap, w.Sr, out);
  k_adj_faces<2><<<grid2(n1 + 2, n2 + 1, b), b, 0, s>>>(a, pb, w.LdU, w.Le, w.Lsnap, w.Sr, 0.);
  k_adj_recon<2><<<grid2(n1 + 2, n2 + 2, b), b, 0, s>>>(a, pb, w.Lsnap, w.Sr, out);
}

// step n's adjoint from its record r and its output state pout (p^{n+1}),
// dt the step's (a.sc->dt): w.La = lambda_{n+1} -> lambda_n.  Fixed roles
// (La in and out, Lb the midpoint state's adjoint, Lc the accumulator), so
// that a slot's adjoint step can be captured once and replayed.
void adjoint_step(harm_ctx* c, AdjWork& w, const Rec& r, const double* pout, double wm, double we)
{
  const StepArgs a = c->args();
  cudaStream_t s = c->stream;
  const long long nval = (long long)NPR * c->gr.plane;
  const size_t P = (size_t)nval * sizeof(double);
  const double surface = c->cfg.dx2 * (2.0 * 3.14159265358979323846);
  k_adj_seed_edot<<<(c->cfg.n2 + 127) / 128, 128, 0, s>>>(a, pout, w.La, we);
  cudaMemsetAsync(w.Lc, 0, P, s);
  adjoint_substep(c, w, r, 1, w.La, w.Lb, r.pn, r.ph, 1.0, wm * surface, w.Lc);
  adjoint_substep(c, w, r, 0, w.Lb, w.La, r.pn, r.pn, 0.5, 0., w.Lc);
  k_axpy<<<(unsigned)((nval + 255) / 256), 256, 0, s>>>(w.La, w.Lc, nval);
}

// captures what `enqueue` issues on c's stream into a graph (on a private
// stream) and instantiates it
int capture_graph(harm_ctx* c, const std::function<int(harm_ctx*)>& enqueue, cudaGraphExec_t* out)
{
  cudaStream_t cap;
  CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  harm_ctx tmp = *c;
  tmp.stream = cap;
  int rc = HARM_OK;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = HARM_ECUDA;
  if (rc == HARM_OK) {
    rc = enqueue(&tmp);
    if (cudaStreamEndCapture(cap, &g) != cudaSuccess) rc = HARM_ECUDA;
  }
  cudaStreamDestroy(cap);
  if (rc == HARM_OK && cudaGraphInstantiate(out, g, 0) != cudaSuccess) rc = HARM_ECUDA;
  if (g) cudaGraphDestroy(g);
  return rc;
}

// <lam, p> over the active zones, lam given in the reference layout (host)
int host_lambda_to_planes(harm_ctx* c, const double* lam_host, double* planes)
{
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  CK(cudaMemcpyAsync(c->d_stage, lam_host, (size_t)c->n1m * c->n2m * NPR * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  k_ref_to_planes<<<grid2(c->n1m, c->n2m, b), b, 0, c->stream>>>(a, c->d_stage, nullptr, planes);
  CK(cudaGetLastError());
  return HARM_OK;
}

int objective(harm_ctx* c, AdjWork& w, double wm, double we, bool with_lam, double* J)
{
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  double dot = 0.;
  std::vector<double> part(dot_blocks(c));
  if (with_lam) {
    k_dot_active<<<grid2(c->cfg.n1, c->cfg.n2, b), b, 0, c->stream>>>(a, w.La, c->d_p, w.dot);
    CK(cudaMemcpyAsync(part.data(), w.dot, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->d_sc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (with_lam)
    for (double x : part) dot += x;  // block partials in a fixed order: the same J on every run
  *J = wm * h.hz[4] + we * h.hz[6] + dot;
  return HARM_OK;
}

int zero_accumulators(harm_ctx* c)
{
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->d_sc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  h.hz[4] = h.hz[5] = h.hz[6] = 0.;
  CK(cudaMemcpyAsync(c->d_sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  return HARM_OK;
}

// the boundary conditions applied to the input state before the first step
// (init.fishmon.c's bound_prim after init): the adjoint's independent
// variables are the active zones, the ghosts being theirs through this bound
void bound_input(harm_ctx* c)
{
  const StepArgs a = c->args();
  const dim3 b(32, 4);
  k_bound<<<grid2(c->cfg.n1 + 2 * NG, c->cfg.n2 + 2 * NG, b), b, 0, c->stream>>>(a, c->d_p, 1);
  k_poledeath<<<dim3((c->cfg.n1 + 127) / 128, 2), 128, 0, c->stream>>>(a, c->d_p);
}

bool adjoint_supported(const harm_ctx* c)
{
  // the con-to-prim adjoint differentiates the 2D inversion's solution
  return c->cfg.precision == HARM_PREC_FP64 && c->cfg.eom == HARM_EOM_GRMHD && c->cfg.bc == HARM_BC_TORUS &&
         !c->cfg.tryagain;
}

}  // namespace

int harm_run_fixed_dt(harm_ctx* c, const double* dts, int nsteps, double w_mass, double w_em, const double* lam_final,
                      double* J)
{
  if (!c || !dts || nsteps < 1 || !J) return HARM_EINVAL;
  if (!c->geo_ok) return HARM_EGEOMETRY;
  if (!adjoint_supported(c)) return HARM_EINVAL;
  AdjWork w;
  const StepArgs a = c->args();
  w.dts = (double*)w.get((size_t)nsteps * sizeof(double));
  w.La = (double*)w.get((size_t)NPR * c->gr.plane * sizeof(double));
  w.dot = (double*)w.get(dot_blocks(c) * sizeof(double));
  if (!w.ok) return HARM_ENOMEM;
  CK(cudaMemcpyAsync(w.dts, dts, (size_t)nsteps * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  bound_input(c);
  int rc = zero_accumulators(c);
  if (rc) return rc;
  if ((rc = harm_step(c, 0)) != HARM_OK) return rc;  // capture the step graph
  for (int n = 0; n < nsteps; n++) {
    k_set_dt<<<1, 1, 0, c->stream>>>(a, w.dts, n);
    CK(cudaGraphLaunch(c->gexec, c->stream));
  }
  if (lam_final && (rc = host_lambda_to_planes(c, lam_final, w.La)) != HARM_OK) return rc;
  return objective(c, w, w_mass, w_em, lam_final != nullptr, J);
}

int harm_adjoint_run(harm_ctx* c, int nsteps, int checkpoint_every, double w_mass, double w_em,
                     const double* lam_final, double* J, double* grad, double* dts_out, double* ms_out)
{
  if (!c || nsteps < 1 || checkpoint_every < 1 || !J || !grad) return HARM_EINVAL;
  if (!c->geo_ok) return HARM_EGEOMETRY;
  if (!adjoint_supported(c)) return HARM_EINVAL;
  AdjWork w;
  const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  const int nsets = (nck > 1) ? 2 : 1;
  int rc = adj_alloc(c, w, nsteps, std::min(checkpoint_every, nsteps), nsets);
  if (rc) return rc;
  const size_t pl = (size_t)c->gr.plane, P = NPR * pl * sizeof(double);
  std::vector<Saved> ck(nck);
  for (auto& x : ck) x = Saved{(double*)w.get(P), (double*)w.get(pl * sizeof(double))};
  Saved fin{(double*)w.get(P), (double*)w.get(pl * sizeof(double))};
  Saved in0{(double*)w.get(P), (double*)w.get(pl * sizeof(double))};
  if (!w.ok) return HARM_ENOMEM;
  const StepArgs a = c->args();
  cudaStream_t s = c->stream;
  cudaEvent_t e0, e1, e2;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventCreate(&e2));
  save_state(c, in0);
  bound_input(c);
  if ((rc = zero_accumulators(c)) != HARM_OK) return rc;
  if ((rc = harm_step(c, 0)) != HARM_OK) return rc;
  // forward: free dt, recorded; checkpoints every checkpoint_every steps
  CK(cudaEventRecord(e0, s));
  for (int n = 0; n < nsteps; n++) {
    if (n % checkpoint_every == 0) save_state(c, ck[n / checkpoint_every]);
    k_get_dt<<<1, 1, 0, s>>>(a, w.dts, n);
    CK(cudaGraphLaunch(c->gexec, s));
  }
  CK(cudaEventRecord(e1, s));
  if (lam_final) {
    if ((rc = host_lambda_to_planes(c, lam_final, w.La)) != HARM_OK) return rc;
    const dim3 b(32, 4);
    k_mask_ghosts<<<grid2(c->n1m, c->n2m, b), b, 0, s>>>(a, w.La);
  } else {
    CK(cudaMemsetAsync(w.La, 0, P, s));
  }
  if ((rc = objective(c, w, w_mass, w_em, lam_final != nullptr, J)) != HARM_OK) return rc;
  DevScalars hfin;
  CK(cudaMemcpyAsync(&hfin, c->d_sc, sizeof(hfin), cudaMemcpyDeviceToHost, s));
  save_state(c, fin);
  // reverse, segment by segment: recompute the segment from its checkpoint,
  // recording every step, then the steps' adjoints in reverse order (both
  // as per-slot graphs, captured on first use).  The replay of segment sg-1
  // (this context's stream, record set (sg-1) & 1) runs while the adjoint of
  // segment sg (stream sa, set sg & 1) does: they share only the geometry
  // (read) -- the adjoint's steps read their dt from their own scalars.  A
  // set is replayed into only after the adjoint that read it has finished.
  cudaStream_t sa = nullptr;
  cudaEvent_t ev_rec[2] = {nullptr, nullptr}, ev_adj[2] = {nullptr, nullptr}, ev_join = nullptr;
  // released on every return below (after the context's stream has drained
  // what was enqueued on sa, or on an error path)
  struct Release {
    cudaStream_t& sa;
    cudaEvent_t *ev_rec, *ev_adj;
    cudaEvent_t& ev_join;
    ~Release()
    {
      if (sa) cudaStreamSynchronize(sa);
      for (int x = 0; x < 2; x++) {
        if (ev_rec[x]) cudaEventDestroy(ev_rec[x]);
        if (ev_adj[x]) cudaEventDestroy(ev_adj[x]);
      }
      if (ev_join) cudaEventDestroy(ev_join);
      if (sa) cudaStreamDestroy(sa);
    }
  } release{sa, ev_rec, ev_adj, ev_join};
  {
    // the adjoint chain is the critical path (the replay only has to stay one
    // segment ahead of it): its stream takes the device's highest priority,
    // so that its blocks are scheduled first and the replay fills the rest
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CK(cudaStreamCreateWithPriority(&sa, cudaStreamNonBlocking, greatest));
  }
  for (int x = 0; x < 2; x++) {
    CK(cudaEventCreateWithFlags(&ev_rec[x], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_adj[x], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  // the adjoint's context view: its own stream and scalars (a copy of the
  // run's, whose dt each adjoint step sets)
  harm_ctx ca = *c;
  ca.stream = sa;
  ca.d_sc = w.sc_adj;
  const StepArgs aa = ca.args();
  CK(cudaMemcpyAsync(w.sc_adj, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, s));
  for (int x = 0; x < nsets; x++) {
    w.recg[x].assign(w.rec[x].size(), nullptr);
    w.adjg[x].assign(w.rec[x].size(), nullptr);
  }
  auto replay = [&](int sg) -> int {
    const int x = sg & (nsets - 1), n0 = sg * checkpoint_every, len = std::min(checkpoint_every, nsteps - n0);
    load_state(c, ck[sg]);
    for (int m = 0; m < len; m++) {
      if (!w.recg[x][m]) {
        const Rec* r = &w.rec[x][m];
        const int rc2 = capture_graph(c, [r](harm_ctx* t) { return enqueue_step(t, nullptr, r); }, &w.recg[x][m]);
        if (rc2 != HARM_OK) return rc2;
      }
      k_set_dt<<<1, 1, 0, s>>>(a, w.dts, n0 + m);
      CK(cudaGraphLaunch(w.recg[x][m], s));
    }
    // the segment's last state, where its last step's adjoint reads it
    CK(cudaMemcpyAsync(w.pnext[x][len - 1], c->d_p, P, cudaMemcpyDeviceToDevice, s));
    CK(cudaEventRecord(ev_rec[x], s));
    return HARM_OK;
  };
  if ((rc = replay(nck - 1)) != HARM_OK) return rc;
  for (int sg = nck - 1; sg >= 0; sg--) {
    const int x = sg & (nsets - 1), n0 = sg * checkpoint_every, len = std::min(checkpoint_every, nsteps - n0);
    CK(cudaStreamWaitEvent(sa, ev_rec[x], 0));
    if (sg > 0) {
      // set (sg-1) & 1 was read by the adjoint of segment sg+1
      if (sg + 1 < nck) CK(cudaStreamWaitEvent(s, ev_adj[(sg - 1) & (nsets - 1)], 0));
      if ((rc = replay(sg - 1)) != HARM_OK) return rc;
    }
    for (int m = len - 1; m >= 0; m--) {
      if (!w.adjg[x][m]) {
        const Rec* r = &w.rec[x][m];
        const double* po = w.pnext[x][m];
        AdjWork* wp = &w;
        rc = capture_graph(&ca, [=](harm_ctx* t) {
          adjoint_step(t, *wp, *r, po, w_mass, w_em);
          return HARM_OK;
        }, &w.adjg[x][m]);
        if (rc != HARM_OK) return rc;
      }
      k_set_dt<<<1, 1, 0, sa>>>(aa, w.dts, n0 + m);
      CK(cudaGraphLaunch(w.adjg[x][m], sa));
    }
    CK(cudaEventRecord(ev_adj[x], sa));
  }
  // through the input's bound: ghost adjoints onto the active zones
  {
    const dim3 b(32, 4);
    k_adj_poledeath<<<dim3((c->cfg.n1 + 127) / 128, 2), 128, 0, sa>>>(aa, w.La);
    k_adj_ghosts<<<grid2(c->cfg.n1 + 2 * NG, c->cfg.n2 + 2 * NG, b), b, 0, sa>>>(aa, w.La, in0.p);
  }
  CK(cudaEventRecord(ev_join, sa));
  CK(cudaStreamWaitEvent(s, ev_join, 0));
  CK(cudaEventRecord(e2, s));
  // the gradient in the reference layout
  {
    const dim3 b(32, 4);
    k_planes_to_ref<<<grid2(c->n1m, c->n2m, b), b, 0, s>>>(a, w.La, c->d_stage, nullptr);
    CK(cudaMemcpyAsync(grad, c->d_stage, (size_t)c->n1m * c->n2m * NPR * sizeof(double), cudaMemcpyDeviceToHost,
                       s));
  }
  if (dts_out) CK(cudaMemcpyAsync(dts_out, w.dts, (size_t)nsteps * sizeof(double), cudaMemcpyDeviceToHost, s));
  // leave the context at the forward run's end
  load_state(c, fin);
  CK(cudaMemcpyAsync(c->d_sc, &hfin, sizeof(hfin), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  if (ms_out) {
    float f = 0.f, r = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventElapsedTime(&r, e1, e2);
    ms_out[0] = f;
    ms_out[1] = r;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  return HARM_OK;
}

int harm_profile_step(harm_ctx* c, double* ms, int* launches, int nclasses)
{
  if (!c || !ms || !launches || nclasses < KC_COUNT) return HARM_EINVAL;
  if (!c->geo_ok) return HARM_EGEOMETRY;
  Timer T;
  for (int k = 0; k < 64; k++) CK(cudaEventCreate(&T.ev[k]));
  T.on = true;
  CK(cudaEventRecord(T.ev[0], c->stream));
  int rc = enqueue_step(c, &T);
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < nclasses; k++) {
    ms[k] = 0.0;
    launches[k] = 0;
  }
  for (int k = 1; k <= T.n; k++) {
    float t = 0.f;
    cudaEventElapsedTime(&t, T.ev[k - 1], T.ev[k]);
    ms[T.cls[k]] += t;
    launches[T.cls[k]] += T.nk[k];
  }
  for (int k = 0; k < 64; k++) cudaEventDestroy(T.ev[k]);
  return rc;
}

const char* harm_kernel_name(int k) { return (k >= 0 && k < KC_COUNT) ? KC_NAMES[k] : ""; }

int harm_get_horizon(harm_ctx* c, double* out)
{
  if (!c || !out) return HARM_EINVAL;
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->d_sc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 6; k++) out[k] = h.hz[k];
  return HARM_OK;
}

int harm_get_fluxes(harm_ctx* c, double* F1, double* F2)
{
  if (!c || !F1 || !F2) return HARM_EINVAL;
  const int n1 = c->cfg.n1, n2 = c->cfg.n2, n1m = c->n1m, n2m = c->n2m;
  const long long pl = c->gr.plane;
  std::vector<double> h1((size_t)NPR * pl), h2((size_t)NPR * pl), he((size_t)pl);
  if (c->cfg.precision == HARM_PREC_MIXED) {
    std::vector<float> f1((size_t)NPR * pl), f2((size_t)NPR * pl);
    CK(cudaMemcpyAsync(f1.data(), c->d_F1, f1.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(f2.data(), c->d_F2, f2.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < h1.size(); k++) {
      h1[k] = f1[k];
      h2[k] = f2[k];
    }
  } else {
    CK(cudaMemcpyAsync(h1.data(), c->d_F1, h1.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(h2.data(), c->d_F2, h2.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaMemcpyAsync(he.data(), c->d_emf, he.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  auto D = [&](int i, int j) { return c->gr.at(i, j); };
  auto R = [&](int i, int j) { return ((long long)(i + NG) * n2m + (j + NG)) * NPR; };
  for (int ii = 0; ii < n1m; ii++)
    for (int jj = 0; jj < n2m; jj++)
      for (int k = 0; k < NPR; k++) {
        F1[((long long)ii * n2m + jj) * NPR + k] = h1[(size_t)k * pl + D(ii - NG, jj - NG)];
        F2[((long long)ii * n2m + jj) * NPR + k] = h2[(size_t)k * pl + D(ii - NG, jj - NG)];
      }
  // fix_flux's mirrored B2 on the x2 ghost rows (fixup.c:1369-1381)
  for (int i = -1; i < n1; i++) {
    F1[R(i, -1) + B2] = -F1[R(i, 0) + B2];
    F1[R(i, n2) + B2] = -F1[R(i, n2 - 1) + B2];
  }
  // flux-CT rewrite, step_ch.c:1403-1413
  for (int i = 0; i <= n1; i++)
    for (int j = 0; j <= n2 - 1; j++) {
      F1[R(i, j) + B1] = 0.;
      F1[R(i, j) + B2] = 0.5 * (he[D(i, j)] + he[D(i, j + 1)]);
    }
  for (int i = 0; i <= n1 - 1; i++)
    for (int j = 0; j <= n2; j++) {
      F2[R(i, j) + B1] = -0.5 * (he[D(i, j)] + he[D(i + 1, j)]);
      F2[R(i, j) + B2] = 0.;
    }
  return HARM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free step (harm_step_noalloc in include/harm_b200.h).
//
// For callers that cannot call cudaMalloc: the scratch of one step lives in
// this file-scope device array, so the call allocates nothing.  Every device
// that loads the library holds one copy of it until the process exits.
static constexpr long long NOALLOC_MAX_PLANE = 5632;  // pitch * (n2 + 6): 64 x 64 interior zones fit
static constexpr int NOALLOC_MAX_BLOCKS = 256;        // x1/x2 flux blocks (k_flux grid)
static constexpr long long NA_DPLANES = 39;  // pk0 8, F1 8, F2 8, emf, gammacheck, fixbuf 5, ubuf 8
static constexpr long long NA_OFF_BLOCKMIN = NA_DPLANES * NOALLOC_MAX_PLANE;
static constexpr long long NA_OFF_SCALARS = NA_OFF_BLOCKMIN + 2 * NOALLOC_MAX_BLOCKS;
static constexpr long long NA_OFF_WORKLIST = NA_OFF_SCALARS + 32;  // 256 B for DevScalars
static constexpr long long NA_OFF_BYTES = NA_OFF_WORKLIST + NOALLOC_MAX_PLANE / 2;  // one int per zone
static constexpr long long NA_DOUBLES = NA_OFF_BYTES + (4 * NOALLOC_MAX_PLANE) / 8 + 32;  // bsqf, chk x2, fluxf
static_assert(sizeof(DevScalars) <= 32 * sizeof(double), "DevScalars must fit its slot");
static __device__ __align__(256) double g_noalloc_scratch[NA_DOUBLES];

static double* g_noalloc_addr[64];  // per device: address of g_noalloc_scratch
static int g_noalloc_arch[64];      // per device: 1 sm_100, -1 another device (checked once)
static int g_noalloc_grid[64][3];   // per device: n1, n2 and pitch of the last call (the gamma table's layout)

extern "C" int harm_step_noalloc(const harm_config* cfg, const double* d_geo, double* d_prims, int* d_pflag, double* t,
                                 double* dt, int reset_gammacheck, void* stream)
{
  if (!cfg || !d_geo || !d_prims || !d_pflag || !t || !dt) return HARM_EINVAL;
  if (cfg->n1 < 4 || cfg->n2 < 4 || cfg->precision != HARM_PREC_FP64 || cfg->eom != HARM_EOM_GRMHD) return HARM_EINVAL;
  if (cfg->lim != HARM_LIM_MC && cfg->lim != HARM_LIM_PARA) return HARM_EINVAL;
  if (cfg->fluxmethod != HARM_FLUX_HLL && cfg->fluxmethod != HARM_FLUX_LAXF) return HARM_EINVAL;
  if (cfg->bc != HARM_BC_TORUS && cfg->bc != HARM_BC_STAR) return HARM_EINVAL;
  if (cfg->currents) return HARM_EINVAL;  // the diagnostic currents need a context
  if (cfg->tryagain != 0 && cfg->tryagain != 1) return HARM_EINVAL;
  if (cfg->fluxadjust < 0 || cfg->fluxadjust > 3 || (cfg->fluxadjust && !(cfg->gammadamp > 0.0))) return HARM_EINVAL;
  if (!(cfg->tf > *t)) {
    fprintf(stderr, "harm_step_noalloc: end time tf = %g is not after t = %g (a zeroed config has tf = 0)\n", cfg->tf,
            *t);
    return HARM_EINVAL;
  }
  harm_ctx c;
  memset(&c, 0, sizeof(c));
  c.cfg = *cfg;
  c.stream = (cudaStream_t)stream;
  c.n1m = cfg->n1 + 2 * NG;
  c.n2m = cfg->n2 + 2 * NG;
  c.gr.n1 = cfg->n1;
  c.gr.n2 = cfg->n2;
  c.gr.pitch = ((c.n1m + 15) / 16) * 16;
  c.gr.rows = c.n2m;
  c.gr.plane = (long long)c.gr.pitch * c.gr.rows;
  const dim3 b(32, 4);
  c.flux_by = flux_rows(cfg->n1, cfg->n2, false);
  const dim3 gf = flux_grid(cfg->n1, cfg->n2, c.flux_by);
  c.nblocks_flux = gf.x * gf.y;
  c.tile_update = dim3(32, 4);
  c.tile_small = dim3(32, 4);
  if (c.gr.plane > NOALLOC_MAX_PLANE || c.nblocks_flux > NOALLOC_MAX_BLOCKS) {
    fprintf(stderr,
            "harm_step_noalloc: a %d x %d grid needs %lld doubles per plane; the static scratch holds %lld "
            "(at most 64 x 64 active zones)\n",
            cfg->n1, cfg->n2, c.gr.plane, NOALLOC_MAX_PLANE);
    return HARM_EINVAL;
  }
  // set-up, once per device, with that device current: the host-side name of
  // the array is not a device address
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return HARM_ENODEVICE;
  if (!g_noalloc_arch[dev]) {
    // the device check of harm_create (the kernels are built for sm_100a only)
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev));
    g_noalloc_arch[dev] = (prop.major == 10) ? 1 : -1;
  }
  if (g_noalloc_arch[dev] < 0) return HARM_ENODEVICE;
  {
    // the step synchronises with the host to hand t and dt back, which a
    // stream being captured cannot do: refuse instead of breaking the capture
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(c.stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
      fprintf(stderr, "harm_step_noalloc: the stream is being captured; the call must run outside a capture\n");
      return HARM_EINVAL;
    }
  }
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = (double*)p;
  }
  double* s = g_noalloc_addr[dev];
  const long long pl = c.gr.plane;
  c.d_p = d_prims;
  c.d_pflag = d_pflag;
  c.d_geo = const_cast<double*>(d_geo);
  c.d_pk0 = s;
  c.d_F1 = s + 8 * pl;
  c.d_F2 = s + 16 * pl;
  c.d_emf = s + 24 * pl;
  c.d_gammacheck = s + 25 * pl;
  c.d_fixbuf = s + 26 * pl;
  c.d_ubuf = s + 31 * pl;
  c.d_worklist = (int*)(s + NA_OFF_WORKLIST);
  c.d_blockmin = s + NA_OFF_BLOCKMIN;
  c.d_sc = (DevScalars*)(s + NA_OFF_SCALARS);
  c.d_bsqf = (unsigned char*)(s + NA_OFF_BYTES);
  c.d_chk = c.d_bsqf + pl;
  c.d_fluxf = cfg->fluxadjust ? c.d_chk + 2 * pl : nullptr;
  if (!encode_geo_map(&c.geo_map, d_geo, c.gr, c.tile_update) || !encode_prim_map(&c.map_p, d_prims, c.gr, c.flux_by) ||
      !encode_prim_map(&c.map_pk0, c.d_pk0, c.gr, c.flux_by)) {
    fprintf(stderr, "harm_step_noalloc: d_geo and d_prims must be 16-byte aligned (their TMA maps could not be encoded)\n");
    return HARM_EINVAL;
  }
  c.geo_ok = true;
  // the array keeps the last call's contents: the run scalars start from
  // zero on every call, the check-solution gamma table only when asked
  DevScalars h;
  memset(&h, 0, sizeof(h));
  h.t = *t;
  h.dt = *dt;
  h.dt_free = *dt;
  CK(cudaMemcpyAsync(c.d_sc, &h, sizeof(h), cudaMemcpyHostToDevice, c.stream));
  // the gamma table left by the previous call is laid out for that call's
  // grid: on another grid it starts from zero, as on a fresh table
  const bool regrid = g_noalloc_grid[dev][0] != cfg->n1 || g_noalloc_grid[dev][1] != cfg->n2 ||
                      g_noalloc_grid[dev][2] != c.gr.pitch;
  if (reset_gammacheck || regrid) CK(cudaMemsetAsync(c.d_gammacheck, 0, (size_t)pl * sizeof(double), c.stream));
  g_noalloc_grid[dev][0] = cfg->n1;
  g_noalloc_grid[dev][1] = cfg->n2;
  g_noalloc_grid[dev][2] = c.gr.pitch;
  int rc = enqueue_step(&c);
  if (rc != HARM_OK) return rc;
  CK(cudaMemcpyAsync(&h, c.d_sc, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  *t = h.t;
  *dt = h.dt;
  return h.fail_inv ? HARM_EFAIL : HARM_OK;
}
