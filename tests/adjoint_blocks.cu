// Test harness: each adjoint building block of
// harm_ramt_b200/csrc/harm_adjoint.cuh against central finite differences
// of its forward function, on given states and geometry (host code), and the
// update adjoint's two blocks run on the device as one kernel and as two,
// against their host build (tests/test_gpu_adjoint_blocks.py).  Built with
// nvcc (host, and sm_100a device code) by tests/test_adjoint_blocks.py; every
// check returns the relative error
// |lambda . dF/dp v (finite difference) - pbar . v| / max(|.|, |.|).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "../harm_ramt_b200/csrc/harm_adjoint.cuh"

using namespace harm;

namespace {

__host__ __device__ Geo<double> geo_of(const double* gcov16, const double* gcon16, double gdet)
{
  Geo<double> g;
  for (int a = 0; a < 4; a++)
    for (int b = a; b < 4; b++) {
      g.gcov[sym(a, b)] = gcov16[a * 4 + b];
      g.gcon[sym(a, b)] = gcon16[a * 4 + b];
    }
  g.g = gdet;
  return g;
}

// the last check's two directional derivatives (finite difference, adjoint)
double last_fd = 0., last_an = 0.;

double rel(double a, double b)
{
  last_fd = a;
  last_an = b;
  return fabs(a - b) / fmax(fmax(fabs(a), fabs(b)), 1e-300);
}

// forward functions with a scalar output <lambda, F(p)>
double f_flux(const double* p, const Geo<double>& g, int dir, double gam, const double* lam)
{
  State<double> q;
  state_of(p, g, q);
  double F[NPR];
  flux_of<double, false>(p, q, dir, g, gam, F);
  double s = 0.;
  for (int k = 0; k < NPR; k++) s += lam[k] * F[k];
  return s;
}

double f_vchar(const double* p, const Geo<double>& g, int dir, double gam, const double* lam)
{
  State<double> q;
  state_of(p, g, q);
  double vmax, vmin;
  vchar_of(p, q, dir, g, gam, vmax, vmin);
  return lam[0] * vmax + lam[1] * vmin;
}

double f_limit(const double* p, const Geo<double>& g, double gmax, const double* lam)
{
  double pp[NPR];
  memcpy(pp, p, sizeof(pp));
  limit_gamma(gmax, pp, g);
  double s = 0.;
  for (int k = 0; k < NPR; k++) s += lam[k] * pp[k];
  return s;
}

}  // namespace

extern "C" {

void ab_last(double* out)
{
  out[0] = last_fd;
  out[1] = last_an;
}

// which: 0 flux (dir), 1 vchar (dir), 2 limit_gamma (gmax = aux)
double ab_check(int which, const double* p, const double* v, const double* lam, const double* gcov16,
                const double* gcon16, double gdet, int dir, double gam, double aux, double h)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  double pp[NPR], pm[NPR], pb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  for (int k = 0; k < NPR; k++) {
    pp[k] = p[k] + h * v[k];
    pm[k] = p[k] - h * v[k];
  }
  double fd = 0.;
  State<double> q;
  state_of(p, g, q);
  StateAdj qb;
  qb.zero();
  if (which == 0) {
    fd = (f_flux(pp, g, dir, gam, lam) - f_flux(pm, g, dir, gam, lam)) / (2. * h);
    adj_flux(p, q, dir, g, gam, lam, qb, pb);
    adj_state(p, g, q, qb, pb);
  } else if (which == 1) {
    fd = (f_vchar(pp, g, dir, gam, lam) - f_vchar(pm, g, dir, gam, lam)) / (2. * h);
    if (adj_vchar(p, q, dir, g, gam, lam[0], lam[1], qb, pb)) return -1.;
    adj_state(p, g, q, qb, pb);
  } else {
    fd = (f_limit(pp, g, aux, lam) - f_limit(pm, g, aux, lam)) / (2. * h);
    adj_limit_gamma(aux, p, g, lam, pb);
  }
  double an = 0.;
  for (int k = 0; k < NPR; k++) an += pb[k] * v[k];
  return rel(fd, an);
}

// one face: forward through face_flux's arithmetic (in adj_face_flux's own
// forward part) by finite differences of <lambda, F(pl, pr)>
static double face_value(const double* pl, const double* pr, const Geo<double>& g, int dir, double gam,
                         double gmax, int fluxmethod, const double* lam)
{
  double a[NPR], b[NPR];
  memcpy(a, pl, sizeof(a));
  memcpy(b, pr, sizeof(b));
  const int bd = B1 + dir - 1;
  a[bd] = b[bd] = 0.5 * (a[bd] + b[bd]);
  limit_gamma(gmax, a, g);
  limit_gamma(gmax, b, g);
  State<double> ql, qr;
  state_of(a, g, ql);
  state_of(b, g, qr);
  double Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR];
  flux_of<double, false>(a, ql, dir, g, gam, Fl);
  flux_of<double, false>(b, qr, dir, g, gam, Fr);
  flux_of<double, false>(a, ql, 0, g, gam, Ul);
  flux_of<double, false>(b, qr, 0, g, gam, Ur);
  double cxl, cnl, cxr, cnr;
  vchar_of(a, ql, dir, g, gam, cxl, cnl);
  vchar_of(b, qr, dir, g, gam, cxr, cnr);
  double lmin = rmin(cnl, cnr), lmax = rmax(cxl, cxr);
  lmin = fabs(rmax(0., -lmin));
  lmax = fabs(rmax(0., lmax));
  const double cmin = lmin, cmax = lmax, ctop = rmax(lmax, lmin);
  const double hf = (fluxmethod == 1) ? 1.0 : 0.0, lf = (fluxmethod == 1) ? 0.0 : 1.0;
  double s = 0.;
  for (int k = 0; k < NPR; k++) {
    double Fo;
    if (cmax + cmin != 0.0)
      Fo = hf * ((cmax * Fl[k] + cmin * Fr[k] - cmax * cmin * (Ur[k] - Ul[k])) / (cmax + cmin)) +
           lf * (0.5 * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k])));
    else
      Fo = 0.5 * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k]));
    s += lam[k] * Fo;
  }
  return s;
}

double ab_check_face(const double* pl, const double* pr, const double* vl, const double* vr, const double* lam,
                     const double* gcov16, const double* gcon16, double gdet, int dir, double gam, double gmax,
                     int fluxmethod, double h)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  double a[NPR], b[NPR], c[NPR], d[NPR];
  for (int k = 0; k < NPR; k++) {
    a[k] = pl[k] + h * vl[k];
    b[k] = pr[k] + h * vr[k];
    c[k] = pl[k] - h * vl[k];
    d[k] = pr[k] - h * vr[k];
  }
  const double fd = (face_value(a, b, g, dir, gam, gmax, fluxmethod, lam) -
                     face_value(c, d, g, dir, gam, gmax, fluxmethod, lam)) / (2. * h);
  double plb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.}, prb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  if (adj_face_flux(pl, pr, g, dir, gam, gmax, fluxmethod, lam, plb, prb)) return -1.;
  double an = 0.;
  for (int k = 0; k < NPR; k++) an += plb[k] * vl[k] + prb[k] * vr[k];
  return rel(fd, an);
}

// the geometric source block: <lam, dUg(p)> (as k_update forms dUg)
static double source_value(const double* p, const Geo<double>& g, double gam, const double* conn40, const double* lam)
{
  State<double> q;
  state_of(p, g, q);
  double acc[4] = {0., 0., 0., 0.};
  for (int jj = 0; jj < 4; jj++) {
    double row[4];
    mhd_row<double, false>(p, jj, q, gam, row);
    for (int l = 0; l < 4; l++)
      for (int k = 0; k < 4; k++) acc[l] += row[k] * conn40[k * 10 + sym(l, jj)];
  }
  double s = 0.;
  for (int l = 0; l < 4; l++) s += lam[l] * (0. + g.g * acc[l]);
  return s;
}

double ab_check_source(const double* p, const double* v, const double* lam, const double* gcov16, const double* gcon16,
                       double gdet, const double* conn64, double gam, double h)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  double conn40[40];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++)
      for (int j = l; j < 4; j++) conn40[k * 10 + sym(l, j)] = conn64[(k * 4 + l) * 4 + j];
  double pp[NPR], pm[NPR], pb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  for (int k = 0; k < NPR; k++) {
    pp[k] = p[k] + h * v[k];
    pm[k] = p[k] - h * v[k];
  }
  const double fd = (source_value(pp, g, gam, conn40, lam) - source_value(pm, g, gam, conn40, lam)) / (2. * h);
  adj_source(p, g, gam, conn40, lam, pb);
  double an = 0.;
  for (int k = 0; k < NPR; k++) an += pb[k] * v[k];
  return rel(fd, an);
}

// reconstruction rows against finite differences of the forward limiter
double ab_check_recon(int para, const double* y, const double* v, double lam_l, double lam_r, double h)
{
  double cl[5], cr[5];
  recon_rows(para, y, cl, cr);
  double yp[5], ym[5];
  for (int m = 0; m < 5; m++) {
    yp[m] = y[m] + h * v[m];
    ym[m] = y[m] - h * v[m];
  }
  double lp, rp, lm, rm;
  if (para) {
    para4(yp[0], yp[1], yp[2], yp[3], yp[4], lp, rp);
    para4(ym[0], ym[1], ym[2], ym[3], ym[4], lm, rm);
  } else {
    double dq = mc_slope(yp[1], yp[2], yp[3]);
    lp = yp[2] - 0.5 * dq;
    rp = yp[2] + 0.5 * dq;
    dq = mc_slope(ym[1], ym[2], ym[3]);
    lm = ym[2] - 0.5 * dq;
    rm = ym[2] + 0.5 * dq;
  }
  const double fd = (lam_l * (lp - lm) + lam_r * (rp - rm)) / (2. * h);
  double an = 0.;
  for (int m = 0; m < 5; m++) an += (lam_l * cl[m] + lam_r * cr[m]) * v[m];
  return rel(fd, an);
}

// J_U^T x = b through ift_solve, checked as <x, dU/dp v> = <b, v> with
// dU/dp v from finite differences of primtoU
double ab_check_ift(const double* p, const double* v, const double* b, const double* gcov16, const double* gcon16,
                    double gdet, double gam, double h)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  double x[NPR];
  if (ift_solve(p, g, gam, b, x)) return -1.;
  double pp[NPR], pm[NPR], Up[NPR], Um[NPR];
  for (int k = 0; k < NPR; k++) {
    pp[k] = p[k] + h * v[k];
    pm[k] = p[k] - h * v[k];
  }
  State<double> q;
  state_of(pp, g, q);
  flux_of<double, false>(pp, q, 0, g, gam, Up);
  state_of(pm, g, q);
  flux_of<double, false>(pm, q, 0, g, gam, Um);
  double lhs = 0., rhs = 0.;
  for (int k = 0; k < NPR; k++) {
    lhs += x[k] * (Up[k] - Um[k]) / (2. * h);
    rhs += b[k] * v[k];
  }
  return rel(lhs, rhs);
}

// the evolved conserved vector of p and its Jacobian dU/dp (row-major 8x8)
void ab_primtoU(const double* p, const double* gcov16, const double* gcon16, double gdet, double gam, double* U,
                double* J64)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  State<double> q;
  state_of(p, g, q);
  flux_of<double, false>(p, q, 0, g, gam, U);
  if (J64) {
    double J[5][NPR];
    primtoU_jacobian5(p, g, gam, J);
    for (int r = 0; r < NPR; r++)
      for (int c = 0; c < NPR; c++) J64[r * NPR + c] = (r < 5) ? J[r][c] : ((r == c) ? g.g : 0.);
  }
}

// the geometric source dUg[UU..U3] of p as k_update forms it
void ab_source(const double* p, const double* gcov16, const double* gcon16, double gdet, const double* conn64,
               double gam, double* out4)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  double conn40[40];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++)
      for (int j = l; j < 4; j++) conn40[k * 10 + sym(l, j)] = conn64[(k * 4 + l) * 4 + j];
  for (int l = 0; l < 4; l++) {
    double lam[4] = {0., 0., 0., 0.};
    lam[l] = 1.;
    out4[l] = source_value(p, g, gam, conn40, lam);
  }
}

}  // extern "C"

// ---- the update adjoint's two blocks in one kernel and in two, on the device
// and on the host: x = ift_solve(p1, b) (the con-to-prim step), then the
// geometric source's adjoint at pb with dUg's adjoint c dt x[UU..U3].  The
// arrays hold n zones: p1, pb, b 8 a zone, geo 16 + 16 + 1 (gcov, gcon,
// gdet), conn 64 (Gamma^k_lj, k-major); outputs x and lb 8 a zone (x = 0
// where the solve reports a singular matrix).

namespace {

__host__ __device__ void probe_ift(const double* p1, const double* b, const double* geo, double gam, double* x)
{
  const Geo<double> g = geo_of(geo, geo + 16, geo[32]);
  if (ift_solve(p1, g, gam, b, x))
    for (int k = 0; k < NPR; k++) x[k] = 0.;
}

__host__ __device__ void probe_source(const double* pb, const double* x, const double* geo, const double* conn64,
                                      double gam, double cdt, double* lb)
{
  const Geo<double> g = geo_of(geo, geo + 16, geo[32]);
  double conn40[40];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++)
      for (int j = l; j < 4; j++) conn40[k * 10 + sym(l, j)] = conn64[(k * 4 + l) * 4 + j];
  double dUgb[4];
  for (int l = 0; l < 4; l++) dUgb[l] = cdt * x[UU + l];
  for (int k = 0; k < NPR; k++) lb[k] = 0.;
  adj_source(pb, g, gam, conn40, dUgb, lb);
}

// The con-to-prim step as the first build of the update adjoint formed it:
// the full 8 x 8 Jacobian (one reverse sweep per row) in a local array and
// Gaussian elimination with partial pivoting on its transpose, also local.
// In that build the source adjoint computed after it in the same kernel
// differed from the host's; the mode that runs it here shows whether that
// configuration still does.
__host__ __device__ int legacy_ift(const double* p, const double* geo, double gam, const double* b, double* x)
{
  const Geo<double> g = geo_of(geo, geo + 16, geo[32]);
  double J[NPR][NPR];
  {
    State<double> q;
    state_of(p, g, q);
    for (int r = 0; r < NPR; r++) {
      double Fb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
      Fb[r] = 1.;
      StateAdj qb;
      qb.zero();
      double row[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
      adj_flux(p, q, 0, g, gam, Fb, qb, row);
      adj_state(p, g, q, qb, row);
      for (int c = 0; c < NPR; c++) J[r][c] = row[c];
    }
  }
  double A[NPR][NPR + 1];
  for (int r = 0; r < NPR; r++) {
    for (int c = 0; c < NPR; c++) A[r][c] = J[c][r];
    A[r][NPR] = b[r];
  }
  for (int col = 0; col < NPR; col++) {
    int piv = col;
    for (int r = col + 1; r < NPR; r++)
      if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
    if (A[piv][col] == 0.0) return 1;
    if (piv != col)
      for (int c = 0; c <= NPR; c++) {
        const double t = A[col][c];
        A[col][c] = A[piv][c];
        A[piv][c] = t;
      }
    for (int r = col + 1; r < NPR; r++) {
      const double f = A[r][col] / A[col][col];
      for (int c = col; c <= NPR; c++) A[r][c] -= f * A[col][c];
    }
  }
  for (int r = NPR - 1; r >= 0; r--) {
    double s = A[r][NPR];
    for (int c = r + 1; c < NPR; c++) s -= A[r][c] * x[c];
    x[r] = s / A[r][r];
  }
  return 0;
}

__global__ void k_probe_legacy(int n, const double* p1, const double* pb, const double* b, const double* geo,
                               const double* conn, double gam, double cdt, double* x, double* lb)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  double xz[NPR], lz[NPR];
  if (legacy_ift(p1 + 8 * z, geo + 33 * z, gam, b + 8 * z, xz))
    for (int k = 0; k < NPR; k++) xz[k] = 0.;
  probe_source(pb + 8 * z, xz, geo + 33 * z, conn + 64 * z, gam, cdt, lz);
  for (int k = 0; k < NPR; k++) {
    x[8 * z + k] = xz[k];
    lb[8 * z + k] = lz[k];
  }
}

__global__ void k_probe_fused(int n, const double* p1, const double* pb, const double* b, const double* geo,
                              const double* conn, double gam, double cdt, double* x, double* lb)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  double xz[NPR], lz[NPR];
  probe_ift(p1 + 8 * z, b + 8 * z, geo + 33 * z, gam, xz);
  probe_source(pb + 8 * z, xz, geo + 33 * z, conn + 64 * z, gam, cdt, lz);
  for (int k = 0; k < NPR; k++) {
    x[8 * z + k] = xz[k];
    lb[8 * z + k] = lz[k];
  }
}

__global__ void k_probe_ift(int n, const double* p1, const double* b, const double* geo, double gam, double* x)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z < n) probe_ift(p1 + 8 * z, b + 8 * z, geo + 33 * z, gam, x + 8 * z);
}

__global__ void k_probe_source(int n, const double* pb, const double* x, const double* geo, const double* conn,
                               double gam, double cdt, double* lb)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z < n) probe_source(pb + 8 * z, x + 8 * z, geo + 33 * z, conn + 64 * z, gam, cdt, lb + 8 * z);
}

}  // namespace

extern "C" {

// legacy = 1: the con-to-prim step of legacy_ift
void ab_probe_host(int legacy, int n, const double* p1, const double* pb, const double* b, const double* geo,
                   const double* conn, double gam, double cdt, double* x, double* lb)
{
  for (int z = 0; z < n; z++) {
    if (legacy) {
      if (legacy_ift(p1 + 8 * z, geo + 33 * z, gam, b + 8 * z, x + 8 * z))
        for (int k = 0; k < NPR; k++) x[8 * z + k] = 0.;
    } else {
      probe_ift(p1 + 8 * z, b + 8 * z, geo + 33 * z, gam, x + 8 * z);
    }
    probe_source(pb + 8 * z, x + 8 * z, geo + 33 * z, conn + 64 * z, gam, cdt, lb + 8 * z);
  }
}

// fused = 1: one kernel (k_probe_fused), 0: two (k_probe_ift, k_probe_source),
// 2: one kernel with the legacy con-to-prim step (k_probe_legacy).
// Returns 0, or the CUDA error code.
int ab_probe_device(int fused, int n, const double* p1, const double* pb, const double* b, const double* geo,
                    const double* conn, double gam, double cdt, double* x, double* lb)
{
  const size_t s8 = sizeof(double) * 8 * n, sg = sizeof(double) * 33 * n, sc = sizeof(double) * 64 * n;
  double *dp1 = nullptr, *dpb = nullptr, *db = nullptr, *dg = nullptr, *dc = nullptr, *dx = nullptr, *dl = nullptr;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&dp1, s8);
  if (e == cudaSuccess) e = cudaMalloc(&dpb, s8);
  if (e == cudaSuccess) e = cudaMalloc(&db, s8);
  if (e == cudaSuccess) e = cudaMalloc(&dg, sg);
  if (e == cudaSuccess) e = cudaMalloc(&dc, sc);
  if (e == cudaSuccess) e = cudaMalloc(&dx, s8);
  if (e == cudaSuccess) e = cudaMalloc(&dl, s8);
  if (e == cudaSuccess) e = cudaMemcpy(dp1, p1, s8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dpb, pb, s8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, b, s8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dg, geo, sg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dc, conn, sc, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int th = 128, bl = (n + th - 1) / th;
    if (fused == 2) {
      k_probe_legacy<<<bl, th>>>(n, dp1, dpb, db, dg, dc, gam, cdt, dx, dl);
    } else if (fused) {
      k_probe_fused<<<bl, th>>>(n, dp1, dpb, db, dg, dc, gam, cdt, dx, dl);
    } else {
      k_probe_ift<<<bl, th>>>(n, dp1, db, dg, gam, dx);
      k_probe_source<<<bl, th>>>(n, dpb, dx, dg, dc, gam, cdt, dl);
    }
    e = cudaDeviceSynchronize();
  }
  if (e == cudaSuccess) e = cudaMemcpy(x, dx, s8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(lb, dl, s8, cudaMemcpyDeviceToHost);
  cudaFree(dp1);
  cudaFree(dpb);
  cudaFree(db);
  cudaFree(dg);
  cudaFree(dc);
  cudaFree(dx);
  cudaFree(dl);
  return (int)e;
}

}  // extern "C"
