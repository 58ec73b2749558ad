// Reverse-mode (adjoint) building blocks of the FP64 GRMHD step.
//
// Each adj_* function takes the forward inputs of the matching forward
// function in harm_device.cuh, recomputes what it needs, and adds the
// vector-Jacobian product of a given output adjoint to the input adjoints
// (+=).  Branches (limiters, clamps, min/max selections) are taken as the
// forward evaluation takes them: the derivative is that of the active
// piece.  The piecewise-linear reconstructions are differentiated in
// forward mode with the Tan<N> type below (their Jacobian rows are exact).
// Host-and-device so that tests can compare each block with finite
// differences of its forward function on the CPU.
#pragma once
#include "harm_device.cuh"

namespace harm {

// ------------------------------------------------------------ tangents
template <int N>
struct Tan {
  double v;
  double d[N];
  HD_INLINE Tan() {}
  HD_INLINE Tan(double x) : v(x)
  {
    for (int k = 0; k < N; k++) d[k] = 0.;
  }
};
template <int N>
HD_INLINE Tan<N> operator+(const Tan<N>& a, const Tan<N>& b)
{
  Tan<N> r;
  r.v = a.v + b.v;
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N>
HD_INLINE Tan<N> operator-(const Tan<N>& a, const Tan<N>& b)
{
  Tan<N> r;
  r.v = a.v - b.v;
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N>
HD_INLINE Tan<N> operator-(const Tan<N>& a)
{
  Tan<N> r;
  r.v = -a.v;
  for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
  return r;
}
template <int N>
HD_INLINE Tan<N> operator*(const Tan<N>& a, const Tan<N>& b)
{
  Tan<N> r;
  r.v = a.v * b.v;
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N>
HD_INLINE Tan<N> operator/(const Tan<N>& a, const Tan<N>& b)
{
  Tan<N> r;
  r.v = a.v / b.v;
  for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
template <int N>
HD_INLINE bool operator<(const Tan<N>& a, const Tan<N>& b) { return a.v < b.v; }
template <int N>
HD_INLINE bool operator>(const Tan<N>& a, const Tan<N>& b) { return a.v > b.v; }
template <int N>
HD_INLINE bool operator<=(const Tan<N>& a, const Tan<N>& b) { return a.v <= b.v; }
using ::fabs;  // keep fabs(double), sqrt(double) visible next to the overloads below
using ::sqrt;
template <int N>
HD_INLINE Tan<N> fabs(const Tan<N>& a) { return (a.v < 0.) ? -a : a; }
template <int N>
HD_INLINE Tan<N> sqrt(const Tan<N>& a)
{
  Tan<N> r;
  r.v = sqrt(a.v);
  for (int k = 0; k < N; k++) r.d[k] = (r.v > 0.) ? a.d[k] / (2. * r.v) : 0.;
  return r;
}
template <int N>
HD_INLINE bool operator>=(const Tan<N>& a, const Tan<N>& b) { return a.v >= b.v; }

// ------------------------------------------------------------ state
struct StateAdj {
  double ucon[4], ucov[4], bcon[4], bcov[4];
  HD_INLINE void zero()
  {
    for (int k = 0; k < 4; k++) ucon[k] = ucov[k] = bcon[k] = bcov[k] = 0.;
  }
};

// gamma_of: gamma = sqrt(1 + g_ij u^i u^j)
HD_INLINE void adj_gamma(const double* pr, const Geo<double>& g, double gb, double* prb)
{
  const double* c = g.gcov;
  const double gamma = gamma_of(pr, g);
  const double qb = gb / (2. * gamma);
  const double u1 = pr[U1], u2 = pr[U2], u3 = pr[U3];
  prb[U1] += qb * (2. * c[4] * u1 + 2. * c[5] * u2 + 2. * c[6] * u3);
  prb[U2] += qb * (2. * c[7] * u2 + 2. * c[5] * u1 + 2. * c[8] * u3);
  prb[U3] += qb * (2. * c[9] * u3 + 2. * c[6] * u1 + 2. * c[8] * u2);
}

// ucon_of: u^0 = gamma/alpha, u^i = u~^i - gamma beta^i/alpha
HD_INLINE void adj_ucon(const double* pr, const Geo<double>& g, const double* uconb, double* prb)
{
  const double alpha = 1. / sqrt(-g.gcon[0]);
  const double b1 = g.gcon[1] * alpha * alpha, b2 = g.gcon[2] * alpha * alpha, b3 = g.gcon[3] * alpha * alpha;
  const double gb = uconb[0] / alpha - (uconb[1] * b1 + uconb[2] * b2 + uconb[3] * b3) / alpha;
  prb[U1] += uconb[1];
  prb[U2] += uconb[2];
  prb[U3] += uconb[3];
  adj_gamma(pr, g, gb, prb);
}

// w = G v with the symmetric packed metric: vb += G wb
HD_INLINE void adj_lower(const double* c, const double* wb, double* vb)
{
  for (int m = 0; m < 4; m++) {
    double s = 0.;
    for (int n = 0; n < 4; n++) s += c[sym(m, n)] * wb[n];
    vb[m] += s;
  }
}

// state_of: consumes qb (the output adjoints), adds to prb
HD_INLINE void adj_state(const double* pr, const Geo<double>& g, const State<double>& q, const StateAdj& qb,
                         double* prb)
{
  double bconb[4], uconb[4], ucovb[4];
  for (int m = 0; m < 4; m++) {
    bconb[m] = qb.bcon[m];
    uconb[m] = qb.ucon[m];
    ucovb[m] = qb.ucov[m];
  }
  adj_lower(g.gcov, qb.bcov, bconb);
  // b^j = (B^j + b^0 u^j) / u^0, j = 1..3
  double bcon0b = bconb[0];
  const double u0 = q.ucon[0];
  for (int j = 1; j <= 3; j++) {
    const double tb = bconb[j] / u0;
    uconb[0] -= bconb[j] * q.bcon[j] / u0;
    prb[B1 - 1 + j] += tb;
    bcon0b += tb * q.ucon[j];
    uconb[j] += tb * q.bcon[0];
  }
  // b^0 = B^i u_i
  for (int i = 1; i <= 3; i++) {
    prb[B1 - 1 + i] += bcon0b * q.ucov[i];
    ucovb[i] += bcon0b * pr[B1 - 1 + i];
  }
  adj_lower(g.gcov, ucovb, uconb);
  adj_ucon(pr, g, uconb, prb);
}

// mhd_row (GRMHD): mhdb -> qb, prb
HD_INLINE void adj_mhd_row(const double* pr, int dir, const State<double>& q, double gam, const double* mhdb,
                           StateAdj& qb, double* prb)
{
  const double r = pr[RHO], u = pr[UU];
  const double P = (gam - 1.) * u;
  const double w = P + r + u;
  const double bsq = dot4(q.bcon, q.bcov);
  const double eta = w + bsq;
  double etab = 0., ptotb = mhdb[dir], bsqb;
  for (int j = 0; j < 4; j++) {
    etab += mhdb[j] * q.ucon[dir] * q.ucov[j];
    qb.ucon[dir] += mhdb[j] * eta * q.ucov[j];
    qb.ucov[j] += mhdb[j] * eta * q.ucon[dir];
    qb.bcon[dir] -= mhdb[j] * q.bcov[j];
    qb.bcov[j] -= mhdb[j] * q.bcon[dir];
  }
  bsqb = etab + 0.5 * ptotb;
  const double wb = etab, Pb = wb + ptotb;
  prb[RHO] += wb;
  prb[UU] += wb + (gam - 1.) * Pb;
  for (int k = 0; k < 4; k++) {
    qb.bcon[k] += bsqb * q.bcov[k];
    qb.bcov[k] += bsqb * q.bcon[k];
  }
}

// flux_of (GRMHD, with sqrt(-g) and the rest mass in UU): Fb -> qb, prb
HD_INLINE void adj_flux(const double* pr, const State<double>& q, int dir, const Geo<double>& g, double gam,
                        const double* Fb, StateAdj& qb, double* prb)
{
  double finb[NPR];
  for (int k = 0; k < NPR; k++) finb[k] = Fb[k] * g.g;
  finb[RHO] += finb[UU];
  if (dir > 0) {
    const int bd = B1 + dir - 1;
    const double u0 = q.ucon[0];
    for (int k = 1; k <= 3; k++) {
      const int kk = B1 + k - 1;
      const double fin = (pr[kk] * q.ucon[dir] - pr[bd] * q.ucon[k]) / u0;
      const double nb = finb[kk] / u0;
      qb.ucon[0] -= finb[kk] * fin / u0;
      prb[kk] += nb * q.ucon[dir];
      qb.ucon[dir] += nb * pr[kk];
      prb[bd] -= nb * q.ucon[k];
      qb.ucon[k] -= nb * pr[bd];
    }
  } else {
    for (int kk = B1; kk <= B3; kk++) prb[kk] += finb[kk];
  }
  adj_mhd_row(pr, dir, q, gam, &finb[UU], qb, prb);
  prb[RHO] += finb[RHO] * q.ucon[dir];
  qb.ucon[dir] += finb[RHO] * pr[RHO];
}

// vchar_of (FP64): (vmaxb, vminb) -> qb, prb.  Returns the forward fail code
// (no adjoint is added when it is nonzero).
HD_INLINE int adj_vchar(const double* pr, const State<double>& q, int dir, const Geo<double>& g, double gam,
                        double vmaxb, double vminb, StateAdj& qb, double* prb)
{
  const double eps100 = DBL_EPS_REF * 100.0;
  const double bsq = dot4(q.bcon, q.bcov);
  const double rho = pr[RHO], u = pr[UU];
  double WW = rho + gam * u, cs2, EF, va2;
  const bool wwpos = WW > 0.0;
  if (wwpos) cs2 = gam * (gam - 1.) * u / WW;
  else WW = cs2 = 0.0;
  EF = bsq + WW;
  const bool efpos = EF > 0.0;
  if (efpos) va2 = bsq / EF;
  else EF = va2 = 0.0;
  double cms2 = cs2 + va2 - cs2 * va2;
  bool clamped = false;
  if (cms2 < 0.0) {
    if (cms2 / (cs2 + va2) > -eps100) {
      cms2 = 0.0;
      clamped = true;
    } else return FAIL_COEFF_NEG;
  }
  if (cms2 > 1.) {
    if (cms2 < 1.0 + eps100) {
      cms2 = 1.0;
      clamped = true;
    } else return FAIL_COEFF_SUP;
  }
  const double Asq = g.gcon[sym(dir, dir)], Bsq = g.gcon[0], AB = g.gcon[sym(0, dir)];
  const double Au = q.ucon[dir], Bu = q.ucon[0];
  const double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  const double A = Bu2 - (Bsq + Bu2) * cms2;
  const double B = 2. * (AuBu - (AB + AuBu) * cms2);
  const double C = Au2 - (Asq + Au2) * cms2;
  double discr = B * B - 4. * A * C;
  bool dclamped = false;
  if ((discr < 0.0) && (discr > -1E-10)) {
    discr = 0.0;
    dclamped = true;
  } else if (discr < -1E-10) return FAIL_VCHAR_DISCR;
  const double d = sqrt(discr);
  const double vm = -(-B + d) / (2. * A);
  const double vp = -(-B - d) / (2. * A);
  double vmb, vpb;
  if (vp < vm) {
    vmb = vmaxb;
    vpb = vminb;
  } else {
    vpb = vmaxb;
    vmb = vminb;
  }
  double Bb = (vmb + vpb) / (2. * A);
  const double db = (vpb - vmb) / (2. * A);
  double Ab = -(vmb * vm + vpb * vp) / A;
  double Cb = 0.;
  if (!dclamped && d > 0.) {
    const double discrb = db / (2. * d);
    Bb += 2. * B * discrb;
    Ab += -4. * C * discrb;
    Cb = -4. * A * discrb;
  }
  const double Bu2b = Ab * (1. - cms2);
  double cms2b = -Ab * (Bsq + Bu2);
  const double AuBub = 2. * Bb * (1. - cms2);
  cms2b += -2. * Bb * (AB + AuBu);
  const double Au2b = Cb * (1. - cms2);
  cms2b += -Cb * (Asq + Au2);
  qb.ucon[dir] += 2. * Au * Au2b + AuBub * Bu;
  qb.ucon[0] += 2. * Bu * Bu2b + AuBub * Au;
  if (clamped) cms2b = 0.;
  const double cs2b = cms2b * (1. - va2), va2b = cms2b * (1. - cs2);
  double bsqb = 0., WWb = 0.;
  if (efpos) {
    bsqb += va2b / EF;
    const double EFb = -va2b * va2 / EF;
    bsqb += EFb;
    WWb += EFb;
  }
  if (wwpos) {
    prb[UU] += cs2b * gam * (gam - 1.) / WW;
    WWb += -cs2b * cs2 / WW;
    prb[RHO] += WWb;
    prb[UU] += gam * WWb;
  }
  for (int k = 0; k < 4; k++) {
    qb.bcon[k] += bsqb * q.bcov[k];
    qb.bcov[k] += bsqb * q.bcon[k];
  }
  return 0;
}

// limit_gamma: pin -> pout (u~ scaled when gamma > gammamax); poutb -> pinb
// (pinb += ...; the non-velocity components pass straight through)
HD_INLINE void adj_limit_gamma(double gammamax, const double* pin, const Geo<double>& g, const double* poutb,
                               double* pinb)
{
  for (int k = 0; k < NPR; k++)
    if (k < U1 || k > U3) pinb[k] += poutb[k];
  double gamma = (gammamax > 1.0) ? gamma_of(pin, g) : 1.0;
  if (gammamax > 1.0 && gamma > gammamax && gamma != 1.0) {
    const double pref = (gammamax * gammamax - 1.) / (gamma * gamma - 1.);
    const double f = sqrt(pref);
    double fb = 0.;
    for (int k = U1; k <= U3; k++) {
      pinb[k] += poutb[k] * f;
      fb += poutb[k] * pin[k];
    }
    const double prefb = fb / (2. * f);
    const double gammab = -prefb * pref * 2. * gamma / (gamma * gamma - 1.);
    adj_gamma(pin, g, gammab, pinb);
  } else {
    for (int k = U1; k <= U3; k++) pinb[k] += poutb[k];
  }
}

// ------------------------------------------------------------ faces
// The flux through one face from its two interface states (face_flux in
// harm_step_impl.cuh: B^dir continuity, limit_gamma on both states, states,
// fluxes and conserved vectors, wavespeeds, HLL/LAXF).  pl, pr are the
// reconstructed states before the B^dir averaging; Fob the adjoint of the
// face flux.  Adds to plb, prb.  Returns the forward fail code.
HD_INLINE int adj_face_flux(const double* pl_in, const double* pr_in, const Geo<double>& g, int dir, double gam,
                            double gammamax, int fluxmethod, const double* Fob, double* plb, double* prb)
{
  double pa[NPR], pb_[NPR], la[NPR], lb[NPR];
  const int bd = B1 + dir - 1;
  for (int k = 0; k < NPR; k++) {
    pa[k] = pl_in[k];
    pb_[k] = pr_in[k];
  }
  pa[bd] = pb_[bd] = 0.5 * (pl_in[bd] + pr_in[bd]);
  for (int k = 0; k < NPR; k++) {
    la[k] = pa[k];
    lb[k] = pb_[k];
  }
  int rc = limit_gamma(gammamax, la, g);
  if (!rc) rc = limit_gamma(gammamax, lb, g);
  if (rc) return rc;
  State<double> ql, qr;
  state_of(la, g, ql);
  state_of(lb, g, qr);
  double Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR];
  flux_of<double, false>(la, ql, dir, g, gam, Fl);
  flux_of<double, false>(lb, qr, dir, g, gam, Fr);
  flux_of<double, false>(la, ql, 0, g, gam, Ul);
  flux_of<double, false>(lb, qr, 0, g, gam, Ur);
  double cmax_l, cmin_l, cmax_r, cmin_r;
  rc = vchar_of(la, ql, dir, g, gam, cmax_l, cmin_l);
  if (!rc) rc = vchar_of(lb, qr, dir, g, gam, cmax_r, cmin_r);
  if (rc) return rc;
  // cminmax_calc
  const double lmin0 = rmin(cmin_l, cmin_r), lmax0 = rmax(cmax_l, cmax_r);
  const double lmin = fabs(rmax(0., -lmin0)), lmax = fabs(rmax(0., lmax0));
  const double cmin = lmin, cmax = lmax;
  const double ctop = rmax(lmax, lmin);
  const double hllfrac = (fluxmethod == 1) ? 1.0 : 0.0, laxffrac = (fluxmethod == 1) ? 0.0 : 1.0;
  double Flb[NPR], Frb[NPR], Ulb[NPR], Urb[NPR];
  double cmaxb = 0., cminb = 0., ctopb = 0.;
  const double S = cmax + cmin;
  const bool hllform = (S != 0.0);
  for (int k = 0; k < NPR; k++) {
    const double dU = Ur[k] - Ul[k];
    double dUb = 0.;
    Flb[k] = Frb[k] = 0.;
    if (hllform) {
      const double Hb = hllfrac * Fob[k];
      const double H = (cmax * Fl[k] + cmin * Fr[k] - cmax * cmin * dU) / S;
      Flb[k] += Hb * cmax / S;
      Frb[k] += Hb * cmin / S;
      dUb += -Hb * cmax * cmin / S;
      cmaxb += Hb * (Fl[k] - cmin * dU) / S - Hb * H / S;
      cminb += Hb * (Fr[k] - cmax * dU) / S - Hb * H / S;
      const double Lb = laxffrac * Fob[k];
      Flb[k] += 0.5 * Lb;
      Frb[k] += 0.5 * Lb;
      dUb += -0.5 * Lb * ctop;
      ctopb += -0.5 * Lb * dU;
    } else {
      const double Lb = Fob[k];
      Flb[k] += 0.5 * Lb;
      Frb[k] += 0.5 * Lb;
      dUb += -0.5 * Lb * ctop;
      ctopb += -0.5 * Lb * dU;
    }
    Urb[k] = dUb;
    Ulb[k] = -dUb;
  }
  // ctop = rmax(lmax, lmin): (lmax > lmin) ? lmax : lmin
  double lmaxb = cmaxb, lminb = cminb;
  if (lmax > lmin) lmaxb += ctopb;
  else lminb += ctopb;
  // lmax = |max(0, lmax0)|, lmin = |max(0, -lmin0)|
  const double lmax0b = (lmax0 > 0.) ? lmaxb : 0.;
  const double lmin0b = (-lmin0 > 0.) ? -lminb : 0.;
  // lmax0 = rmax(cmax_l, cmax_r), lmin0 = rmin(cmin_l, cmin_r)
  double cmaxlb = 0., cmaxrb = 0., cminlb = 0., cminrb = 0.;
  if (cmax_l > cmax_r) cmaxlb = lmax0b;
  else cmaxrb = lmax0b;
  if (cmin_l > cmin_r) cminrb = lmin0b;
  else cminlb = lmin0b;
  double lab[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.}, lbb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  StateAdj qlb, qrb;
  qlb.zero();
  qrb.zero();
  adj_vchar(la, ql, dir, g, gam, cmaxlb, cminlb, qlb, lab);
  adj_vchar(lb, qr, dir, g, gam, cmaxrb, cminrb, qrb, lbb);
  adj_flux(la, ql, dir, g, gam, Flb, qlb, lab);
  adj_flux(lb, qr, dir, g, gam, Frb, qrb, lbb);
  adj_flux(la, ql, 0, g, gam, Ulb, qlb, lab);
  adj_flux(lb, qr, 0, g, gam, Urb, qrb, lbb);
  adj_state(la, g, ql, qlb, lab);
  adj_state(lb, g, qr, qrb, lbb);
  double pab[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.}, pbb[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
  adj_limit_gamma(gammamax, pa, g, lab, pab);
  adj_limit_gamma(gammamax, pb_, g, lbb, pbb);
  const double tb = pab[bd] + pbb[bd];
  pab[bd] = 0.5 * tb;
  pbb[bd] = 0.5 * tb;
  for (int k = 0; k < NPR; k++) {
    plb[k] += pab[k];
    prb[k] += pbb[k];
  }
  return 0;
}

// The face flux itself (the forward part of adj_face_flux), for the faces
// where fix_flux clamps a component on its sign.  Returns the fail code.
HD_INLINE int face_flux_primal(const double* pl_in, const double* pr_in, const Geo<double>& g, int dir, double gam,
                               double gammamax, int fluxmethod, double* Fo)
{
  double la[NPR], lb[NPR];
  const int bd = B1 + dir - 1;
  for (int k = 0; k < NPR; k++) {
    la[k] = pl_in[k];
    lb[k] = pr_in[k];
  }
  la[bd] = lb[bd] = 0.5 * (pl_in[bd] + pr_in[bd]);
  int rc = limit_gamma(gammamax, la, g);
  if (!rc) rc = limit_gamma(gammamax, lb, g);
  if (rc) return rc;
  State<double> ql, qr;
  state_of(la, g, ql);
  state_of(lb, g, qr);
  double Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR];
  flux_of<double, false>(la, ql, dir, g, gam, Fl);
  flux_of<double, false>(lb, qr, dir, g, gam, Fr);
  flux_of<double, false>(la, ql, 0, g, gam, Ul);
  flux_of<double, false>(lb, qr, 0, g, gam, Ur);
  double cxl, cnl, cxr, cnr;
  rc = vchar_of(la, ql, dir, g, gam, cxl, cnl);
  if (!rc) rc = vchar_of(lb, qr, dir, g, gam, cxr, cnr);
  if (rc) return rc;
  double lmin = rmin(cnl, cnr), lmax = rmax(cxl, cxr);
  lmin = fabs(rmax(0., -lmin));
  lmax = fabs(rmax(0., lmax));
  const double cmin = lmin, cmax = lmax, ctop = rmax(lmax, lmin);
  const double hf = (fluxmethod == 1) ? 1.0 : 0.0, lf = (fluxmethod == 1) ? 0.0 : 1.0;
  for (int k = 0; k < NPR; k++) {
    if (cmax + cmin != 0.0)
      Fo[k] = hf * ((cmax * Fl[k] + cmin * Fr[k] - cmax * cmin * (Ur[k] - Ul[k])) / (cmax + cmin)) +
              lf * (0.5 * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k])));
    else
      Fo[k] = 0.5 * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k]));
  }
  return 0;
}

// Jacobian rows of a zone's two interface states along a direction with
// respect to its stencil (one primitive): PARA4 uses y[-2..2], MC y[-1..1].
// cl[m], cr[m] = d(left state)/d y[m-2], d(right state)/d y[m-2].
HD_INLINE void recon_rows(int para, const double* y, double* cl, double* cr)
{
  if (para) {
    Tan<5> t[5];
    for (int m = 0; m < 5; m++) {
      t[m] = Tan<5>(y[m]);
      t[m].d[m] = 1.;
    }
    Tan<5> l, r;
    para4(t[0], t[1], t[2], t[3], t[4], l, r);
    for (int m = 0; m < 5; m++) {
      cl[m] = l.d[m];
      cr[m] = r.d[m];
    }
  } else {
    Tan<3> t[3];
    for (int m = 0; m < 3; m++) {
      t[m] = Tan<3>(y[m + 1]);
      t[m].d[m] = 1.;
    }
    const Tan<3> dq = mc_slope(t[0], t[1], t[2]);
    const Tan<3> l = t[1] - Tan<3>(0.5) * dq, r = t[1] + Tan<3>(0.5) * dq;
    cl[0] = cr[0] = cl[4] = cr[4] = 0.;
    for (int m = 0; m < 3; m++) {
      cl[m + 1] = l.d[m];
      cr[m + 1] = r.d[m];
    }
  }
}

// ------------------------------------------------------------ ghost zones
// The velocity part of an x1 ghost zone's boundary fill (bounds.fishmon.c:
// inflow_check_rel4vel's fix, fixup.c:1784-1829, then limit_gamma) on u~
// alone, templated for tangents; dofix is decided by the caller on the
// values.  Returns nonzero where the forward map fails.
template <typename T>
HD_INLINE T gamma_T(const T* u, const double* c)
{
  const T q = T(c[4]) * u[0] * u[0] + T(c[7]) * u[1] * u[1] + T(c[9]) * u[2] * u[2] +
              T(2.) * (T(c[5]) * u[0] * u[1] + T(c[6]) * u[0] * u[2] + T(c[8]) * u[1] * u[2]);
  return sqrt(T(1.) + q);
}
template <typename T>
HD_INLINE int x1_velocity_map(T* u, const Geo<double>& g, double gammamax, bool dofix)
{
  if (dofix) {
    T gamma = gamma_T(u, g.gcov);
    for (int k = 0; k < 3; k++) u[k] = u[k] / gamma;
    const double alpha = 1. / sqrt(-g.gcon[0]);
    const double betacon = g.gcon[1] * alpha * alpha;
    u[0] = T(betacon / alpha);
    T vsq = T(0.);
    for (int jj = 1; jj < 4; jj++)
      for (int kk = 1; kk < 4; kk++) vsq = vsq + T(g.gcov[sym(jj, kk)]) * u[jj - 1] * u[kk - 1];
    if (vsq < T(0.0)) {
      if (vsq > T(-DBL_EPS_REF * 100.0)) vsq = T(0.0);
      else return FAIL_VSQ_NEG;
    }
    if (vsq >= T(1.0)) vsq = T(1.0 - 1.0 / (gammamax * gammamax));
    gamma = T(1.) / sqrt(T(1.) - vsq);
    for (int k = 0; k < 3; k++) u[k] = u[k] * gamma;
  }
  if (gammamax > 1.0) {
    const T gamma = gamma_T(u, g.gcov);
    if (gamma > T(gammamax) && gamma.v != 1.0) {
      const T pref = (T(gammamax) * T(gammamax) - T(1.)) / (gamma * gamma - T(1.));
      if (pref < T(0.0)) return FAIL_UTCALC_DISCR;
      const T f = sqrt(pref);
      for (int k = 0; k < 3; k++) u[k] = u[k] * f;
    }
  }
  return 0;
}

// ------------------------------------------------------------ source
// The geometric source dUg[UU+l] = g sum_j sum_k T^j_k Gamma^k_{l j} of state
// p (conn[conn_index(k, l, j)] = Gamma^k_{l j}, symmetric pair (l, j)
// packed): dUgb (the adjoints of dUg[UU..U3]) -> pb.
HD_INLINE void adj_source(const double* p, const Geo<double>& g, double gam, const double* conn40,
                          const double* dUgb, double* pb)
{
  State<double> q;
  state_of(p, g, q);
  StateAdj qb;
  qb.zero();
  // unrolled: jj indexes the state components as a constant
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    double rowb[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double s = 0.;
#pragma unroll
      for (int l = 0; l < 4; l++) s += dUgb[l] * g.g * conn40[k * 10 + sym(l, jj)];
      rowb[k] = s;
    }
    adj_mhd_row(p, jj, q, gam, rowb, qb, pb);
  }
  adj_state(p, g, q, qb, pb);
}

// ------------------------------------------------------------ con-to-prim
// dU/dp of the evolved conserved vector (primtoU with sqrt(-g) and the rest
// mass in UU) at p, rows 0..4 (rho u^t, T^t_t + rho u^t, T^t_i): J[r][c] =
// dU_r / dp_c, by one reverse sweep per row.  Rows B1..B3 are U_B = g B.
HD_INLINE void primtoU_jacobian5(const double* p, const Geo<double>& g, double gam, double J[5][NPR])
{
  State<double> q;
  state_of(p, g, q);
#pragma unroll
  for (int r = 0; r < 5; r++) {
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

// Solves dU/dp^T x = b at p (the implicit-function-theorem step of the
// con-to-prim adjoint).  dU/dp is block triangular: U_B = g B does not
// depend on rho..u3, so the rho..u3 columns give a 5 x 5 system in x_0..4
// (Gaussian elimination with partial pivoting) and the B columns then give
// x_B = (b_B - sum_r J[r][B] x_r) / g.  Returns nonzero for a singular
// matrix.  The matrices stay in registers: every index is a compile-time
// constant after unrolling, the pivot row swapped in by selects.
HD_INLINE int ift_solve(const double* p, const Geo<double>& g, double gam, const double* b, double* x)
{
  // A = the transposed rho..u3 block with b beside it; JB[r] = dU_r/dB
  double A[5][6], JB[5][3];
  {
    State<double> q;
    state_of(p, g, q);
    // one reverse sweep per row (a loop the compiler keeps rolled: the rows
    // shift in from the end, so that A and JB are indexed by constants)
    for (int r = 0; r < 5; r++) {
      double Fb[NPR];
#pragma unroll
      for (int k = 0; k < NPR; k++) Fb[k] = (k == r) ? 1. : 0.;
      StateAdj qb;
      qb.zero();
      double row[NPR] = {0., 0., 0., 0., 0., 0., 0., 0.};
      adj_flux(p, q, 0, g, gam, Fb, qb, row);
      adj_state(p, g, q, qb, row);
#pragma unroll
      for (int m = 0; m < 4; m++) {
#pragma unroll
        for (int c = 0; c < 5; c++) A[c][m] = A[c][m + 1];
#pragma unroll
        for (int c = 0; c < 3; c++) JB[m][c] = JB[m + 1][c];
      }
#pragma unroll
      for (int c = 0; c < 5; c++) A[c][4] = row[c];
#pragma unroll
      for (int c = 0; c < 3; c++) JB[4][c] = row[B1 + c];
    }
  }
#pragma unroll
  for (int r = 0; r < 5; r++) A[r][5] = b[r];
  // fixed trip counts with the triangular ranges as conditions: nvcc then
  // unrolls every loop and keeps A in registers
#pragma unroll
  for (int col = 0; col < 5; col++) {
    int piv = col;
    double big = fabs(A[col][col]);
#pragma unroll
    for (int r = 1; r < 5; r++)
      if (r > col && fabs(A[r][col]) > big) {
        piv = r;
        big = fabs(A[r][col]);
      }
    if (big == 0.0) return 1;
#pragma unroll
    for (int r = 1; r < 5; r++) {
      if (r <= col) continue;
      const bool sw = (r == piv);
#pragma unroll
      for (int c = 0; c < 6; c++) {
        if (c < col) continue;
        const double t = A[col][c], u = A[r][c];
        A[col][c] = sw ? u : t;
        A[r][c] = sw ? t : u;
      }
    }
#pragma unroll
    for (int r = 1; r < 5; r++) {
      if (r <= col) continue;
      const double f = A[r][col] / A[col][col];
#pragma unroll
      for (int c = 0; c < 6; c++)
        if (c >= col) A[r][c] -= f * A[col][c];
    }
  }
#pragma unroll
  for (int rr = 0; rr < 5; rr++) {
    const int r = 4 - rr;
    double s = A[r][5];
#pragma unroll
    for (int c = 1; c < 5; c++)
      if (c > r) s -= A[r][c] * x[c];
    x[r] = s / A[r][r];
  }
#pragma unroll
  for (int c = B1; c <= B3; c++) {
    double s = b[c];
#pragma unroll
    for (int r = 0; r < 5; r++) s -= JB[r][c - B1] * x[r];
    x[c] = s / g.g;
  }
  return 0;
}

}  // namespace harm
