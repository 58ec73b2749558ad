/*
 * Probe API over the reference HARM code (test infrastructure only).
 *
 * This file is compiled *together with* a patched scratch copy of the
 * reference sources by oracle/build_ref.py; it includes the reference's own
 * defs.h (as main.c does) and reads/writes the reference's globals.  Only tests/, the smoke
 * check and the CPU-baseline leg of bench.py load the resulting library.
 *
 * Exports (all prefixed hr_):
 *   hr_configure()      runtime knobs applied inside the reference's init
 *   hr_init()           reference init() (initbase.c:297) from a work dir
 *   hr_step()           one reference time step: step_ch() + error_check()
 *                       as in the run loop of main.c:32-45
 *   hr_get_/hr_set_...  copies of p, pflag, geometry tables, floors, fluxes
 *   hr_utoprim2d()      one call of Utoprim_2d (utoprim_2d.c:25)
 *   hr_cycle_break_uniform()  the deterministic replacement for rand() in
 *                       the Newton cycle break (utoprim_2d.c:669), shared
 *                       bit-for-bit with the GPU kernel and the C oracle.
 */
#include "defs.h"   /* defines the reference globals, as main.c does */
#include "step_ch.h"
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

/* ------------------------------------------------------------------ */
/* knobs applied by init_grid()/init_global() below                    */
static int hr_lim = MC;
static int hr_flux = HLLFLUX;
static int hr_timeorder = 2;
static double hr_cour = 0.8;
static int hr_rescaletype = 0;
static double hr_tf = 1.0e30;
static long hr_ncyclebreak = 0;

/* the b^2 and Lorentz-factor thresholds of get_bsqflags (initbase.c:213-215
   defaults 20, 100, 5); negative keeps the default */
static double hr_bsqorholimit = -1.0, hr_bsqoulimit = -1.0, hr_gammadamp = -1.0;
void hr_set_limits(double bsqorholimit_, double bsqoulimit_, double gammadamp_)
{
  hr_bsqorholimit = bsqorholimit_;
  hr_bsqoulimit = bsqoulimit_;
  hr_gammadamp = gammadamp_;
}

void hr_configure(int lim_, int flux_, int timeorder_, double cour_, int rescale_, double tf_)
{
  hr_lim = lim_;
  hr_flux = flux_;
  hr_timeorder = timeorder_;
  hr_cour = cour_;
  hr_rescaletype = rescale_;
  hr_tf = tf_;
}

extern int hr_orig_init_grid(void);
extern int hr_orig_init_global(void);

#ifndef HR_PROBLEM_DIPOLE
/* init.fishmon.c:35 with the benchmark's coordinates: plain MKS (defcoord 0),
   R0 = 0, Rout = 40, hslope = 0.3, Rin = 0.98 r_h (initbase.c:103-114). */
int init_grid(void)
{
  hr_orig_init_grid();
  defcoord = 0;
  R0 = 0.0;
  Rout = 40.0;
  hslope = 0.3;
  Rhor = rhor_calc(0);
  Rin = 0.98 * Rhor;
  return 0;
}
#else
/* init.ns.c:62 turned into the force-free aligned rotator: flat space in
   spherical polar coordinates (MCOORD SPCMINKMETRIC), log-r and uniform
   theta (defcoord 6, coord.c:283-286), r in [1, 100] stellar radii. */
static double hr_omegastar = 0.2;
void hr_set_omegastar(double w) { hr_omegastar = w; }
double hr_get_omegastar(void) { return Omegastar; }
int init_grid(void)
{
  hr_orig_init_grid();
  a = 0.0;
  defcoord = 6;
  R0 = 0.0;
  Rin = 1.0;
  Rout = 100.0;
  Rhor = rhor_calc(0);
  return 0;
}
#endif

static void hr_env_knobs(void);

/* init.fishmon.c:61 / init.ns.c:105 (ranc(7) seed, gamma, boundary types)
   plus the algorithm knobs of the benchmark.  Output cadences are pushed
   out of range; dumps are disabled below. */
int init_global(void)
{
  hr_orig_init_global();
  lim = hr_lim;
  TIMEORDER = hr_timeorder;
  fluxmethod = hr_flux;
  FLUXB = FLUXCTTOTH;
  UTOPRIMVERSION = UTOPRIM2D;
  cour = hr_cour;
  rescaletype = hr_rescaletype;
  debugfail = 0;
  tf = hr_tf;
  DTd = DTavg = DTener = DTi = DTdebug = 1.0e30;
  if (hr_bsqorholimit >= 0.0) BSQORHOLIMIT = hr_bsqorholimit;
  if (hr_bsqoulimit >= 0.0) BSQOULIMIT = hr_bsqoulimit;
  if (hr_gammadamp >= 0.0) GAMMADAMP = hr_gammadamp;
  DTr = 1000000000L;
#ifdef HR_PROBLEM_DIPOLE
  Omegastar = hr_omegastar; /* stellar surface rotation (bounds.ns.c:107) */
#endif
  hr_env_knobs();
  return 0;
}

/* When the reference's own main() drives the run (the drop-in test builds
   it with main.c, once with its step_ch() and once with the B200 shim in
   its place), the environment sets what hr_configure() sets for the
   library builds: HR_LIM and HR_FLUX (the knobs), HR_TF (the end time), and
   HR_FINAL_STATE, a file that receives at exit the final p and pflag (the
   reference's layouts) followed by t, dt and realnstep. */
static void hr_write_final_state(void)
{
  const char *path = getenv("HR_FINAL_STATE");
  FILE *f;
  double tail[3];
  if (!path || !(f = fopen(path, "wb"))) return;
  tail[0] = t;
  tail[1] = dt;
  tail[2] = (double)realnstep;
  fwrite(&a_p[0][0][0], sizeof(a_p), 1, f);
  fwrite(&a_pflag[0][0][0], sizeof(a_pflag), 1, f);
  fwrite(tail, sizeof(tail), 1, f);
  fclose(f);
}

static void hr_env_knobs(void)
{
  static int registered = 0;
  const char *v;
  if ((v = getenv("HR_LIM"))) lim = atoi(v);
  if ((v = getenv("HR_FLUX"))) fluxmethod = atoi(v);
  if ((v = getenv("HR_TF"))) tf = atof(v);
  if (getenv("HR_FINAL_STATE") && !registered) {
    atexit(hr_write_final_state);
    registered = 1;
  }
}

/* patch 12: the first fatal check of a step, as fail() (fail.c:4-57)
   reports it: the code and the zone of the last get_geometry() call
   (icurr, jcurr, set with JONCHECKS 1, phys.c:757) */
extern int hr_orig_fail(int fail_type);
static int hr_fail_code = 0, hr_fail_i = 0, hr_fail_j = 0;
int fail(int fail_type)
{
  if (whocalleducon != 1 && hr_fail_code == 0) {
    hr_fail_code = fail_type;
    hr_fail_i = icurr;
    hr_fail_j = jcurr;
  }
  return hr_orig_fail(fail_type);
}
void hr_get_fail(int *out) { out[0] = hr_fail_code; out[1] = hr_fail_i; out[2] = hr_fail_j; }
void hr_clear_fail(void) { hr_fail_code = hr_fail_i = hr_fail_j = 0; failed = 0; }

/* patch 12: no dump files from the oracle */
int dump(long dump_cnt) { (void)dump_cnt; return 0; }

/* patch 8 shims; freespace.c (system() calls) is not built, dump files are off */
int isenoughfreespace(unsigned long long need) { (void)need; return 1; }
int init_postfield(FTYPE pr[][N2M][NPR]) { (void)pr; return 0; }
FTYPE cot(FTYPE arg) { return 1.0 / tan(arg); }

#ifndef HR_TRYAGAIN
/* patch 7 stubs: only reachable through the disabled UTOPRIMTRYAGAIN chain */
static int hr_unreachable(const char *who)
{
  fprintf(stderr, "oracle build: %s is not part of this build\n", who);
  failed = 1;
  return 1;
}
int Utoprim_1d_final(FTYPE U[NPR], struct of_geom *g, FTYPE prim[NPR]) { (void)U; (void)g; (void)prim; return hr_unreachable("Utoprim_1d_final"); }
int Utoprim_2d_final(FTYPE U[NPR], struct of_geom *g, FTYPE prim[NPR]) { (void)U; (void)g; (void)prim; return hr_unreachable("Utoprim_2d_final"); }
int Utoprim_5d2_final(FTYPE U[NPR], struct of_geom *g, FTYPE prim[NPR]) { (void)U; (void)g; (void)prim; return hr_unreachable("Utoprim_5d2_final"); }
int dudp_calc_gen(int w, FTYPE *pr, struct of_state *q, struct of_geom *g, FTYPE **alpha) { (void)w; (void)pr; (void)q; (void)g; (void)alpha; return hr_unreachable("dudp_calc_gen"); }
FTYPE contract(FTYPE *a1, FTYPE *a2) { return a1[0]*a2[0] + a1[1]*a2[1] + a1[2]*a2[2] + a1[3]*a2[3]; }
FTYPE covtract(FTYPE *a1, FTYPE *a2) { return a1[0]*a2[0] + a1[1]*a2[1] + a1[2]*a2[2] + a1[3]*a2[3]; }
#endif

/* ------------------------------------------------------------------ */
/* patch 11: deterministic cycle-break factor in [0,1).
   splitmix64 finaliser (Steele, Lea & Flood 2014) of the iterate's bit
   patterns and the iteration count; the top 53 bits scaled by 2^-53. */
static uint64_t hr_mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

FTYPE hr_cycle_break_uniform(FTYPE x0, FTYPE x1, int n_iter)
{
  uint64_t a, b;
  double d0 = (double)x0, d1 = (double)x1;
  memcpy(&a, &d0, 8);
  memcpy(&b, &d1, 8);
  hr_ncyclebreak++;
  uint64_t h = hr_mix64(a ^ hr_mix64(b ^ (uint64_t)(uint32_t)n_iter));
  return (FTYPE)((double)(h >> 11) * (1.0 / 9007199254740992.0));
}

long hr_get_ncyclebreak(void) { return hr_ncyclebreak; }

/* ------------------------------------------------------------------ */
int hr_n1(void) { return N1; }
int hr_n2(void) { return N2; }
int hr_nbnd(void) { return N1BND; }
int hr_npr(void) { return NPR; }
int hr_eomtype(void) { return EOMTYPE; }

int hr_init(const char *workdir)
{
  char cwd[4096];
  char *argv[2] = {"harmref", NULL};
  int ret;
  if (getcwd(cwd, sizeof(cwd)) == NULL) return -1;
  if (chdir(workdir) != 0) return -2;
  ret = init(1, argv);
  if (chdir(cwd) != 0) return -3;
  return ret;
}

/* scalars: t, dt, a, gam, Rin, Rout, hslope, R0, startx1, startx2, dx1, dx2,
   cour, Rhor, RHOMIN, UUMIN, GAMMAMAX, GAMMAFAIL, BSQORHOLIMIT, BSQOULIMIT,
   SAFE, defcon, realnstep, dx3, rescaletype, lim, fluxmethod, TIMEORDER,
   GAMMADAMP, FLUXADJUST */
int hr_get_scalars(double *s)
{
  s[0] = t; s[1] = dt; s[2] = a; s[3] = gam; s[4] = Rin; s[5] = Rout;
  s[6] = hslope; s[7] = R0; s[8] = startx[1]; s[9] = startx[2];
  s[10] = dx[1]; s[11] = dx[2]; s[12] = cour; s[13] = Rhor;
  s[14] = RHOMIN; s[15] = UUMIN; s[16] = GAMMAMAX; s[17] = GAMMAFAIL;
  s[18] = BSQORHOLIMIT; s[19] = BSQOULIMIT; s[20] = SAFE; s[21] = defcon;
  s[22] = (double)realnstep; s[23] = dx[3]; s[24] = rescaletype; s[25] = lim;
  s[26] = fluxmethod; s[27] = TIMEORDER;
  s[28] = GAMMADAMP; s[29] = FLUXADJUST;
  return 30;
}

void hr_set_time(double t_, double dt_) { t = t_; dt = dt_; }

/* full arrays including ghost zones, reference layout [N1M][N2M][...] */
void hr_get_prims(double *out) { memcpy(out, &a_p[0][0][0], sizeof(a_p)); }
void hr_set_prims(const double *in) { memcpy(&a_p[0][0][0], in, sizeof(a_p)); }
void hr_get_pflag(int *out) { memcpy(out, &a_pflag[0][0][0], sizeof(a_pflag)); }
void hr_set_pflag(const int *in) { memcpy(&a_pflag[0][0][0], in, sizeof(a_pflag)); }
void hr_get_fluxes(double *f1, double *f2)
{
  memcpy(f1, &a_F1[0][0][0], sizeof(a_F1));
  memcpy(f2, &a_F2[0][0][0], sizeof(a_F2));
}

/* the reference's own text dump file <workdir>/dumps/dump%04ld
   (dump.c:24-46) of the current state */
extern int hr_orig_dump(long dump_cnt);
int hr_dump(const char *workdir, long cnt)
{
  char cwd[4096];
  int rc;
  if (!getcwd(cwd, sizeof(cwd))) return -1;
  if (chdir(workdir) != 0) return -2;
  mkdir("dumps", 0755);
  rc = hr_orig_dump(cnt);
  if (chdir(cwd) != 0) return -3;
  return rc;
}
int hr_get_defcoord(void) { return defcoord; }

/* the reference's own restart file <workdir>/dumps/rdump-%01ld
   (restart_write, restart.c:182-222) of the current state */
int hr_restart_write(const char *workdir, long cnt)
{
  char cwd[4096];
  int rc;
  if (!getcwd(cwd, sizeof(cwd))) return -1;
  if (chdir(workdir) != 0) return -2;
  mkdir("dumps", 0755);
  rc = restart_write(cnt);
  if (chdir(cwd) != 0) return -3;
  return rc;
}

/* X1, X2, r, th at zone centres (coord() and bl_coord()), [N1M][N2M][4] */
void hr_get_coords(double *out)
{
  int i, j;
  FTYPE X[NDIM], r, th;
  for (i = -N1BND; i < N1 + N1BND; i++)
    for (j = -N2BND; j < N2 + N2BND; j++) {
      double *o = out + ((size_t)(i + N1BND) * N2M + (j + N2BND)) * 4;
      coord(i, j, CENT, X);
      bl_coord(X, &r, &th);
      o[0] = X[1];
      o[1] = X[2];
      o[2] = r;
      o[3] = th;
    }
}

/* diagnostic currents (phys.c:1124-1455): jcon [N1M][N2M][4], fcon
   [N1M][N2M][6], cfaraday [N1M][N2M][5][3] */
void hr_get_currents(double *jcon_, double *fcon_, double *cfaraday_)
{
  memcpy(jcon_, &a_jcon[0][0][0], sizeof(a_jcon));
  memcpy(fcon_, &a_fcon[0][0][0], sizeof(a_fcon));
  memcpy(cfaraday_, &a_cfaraday[0][0][0][0], sizeof(a_cfaraday));
}

/* gcov/gcon [N1M][N2M][4 loc][4][4], gdet [N1M][N2M][4], conn [N1M][N2M][4][4][4] */
void hr_get_geometry(double *gcov_, double *gcon_, double *gdet_, double *conn_)
{
  memcpy(gcov_, &a_gcov[0][0][0][0][0], sizeof(a_gcov));
  memcpy(gcon_, &a_gcon[0][0][0][0][0], sizeof(a_gcon));
  memcpy(gdet_, &a_gdet[0][0][0], sizeof(a_gdet));
  memcpy(conn_, &a_conn[0][0][0][0][0], sizeof(a_conn));
}

/* per-zone density floors at CENT as fixup1zone uses them (fixup.c:295-307):
   set_density_floors() then clamped below by RHOMINLIMIT / UUMINLIMIT.
   out [N1M][N2M][2]. */
void hr_get_floors(double *out)
{
  int i, j;
  struct of_geom geom;
  FTYPE prfloor[NPR];
  FULLLOOP {
    get_geometry(i, j, CENT, &geom);
    set_density_floors(&geom, p[i][j], prfloor);
    if (prfloor[RHO] < RHOMINLIMIT) prfloor[RHO] = RHOMINLIMIT;
    if (prfloor[UU] < UUMINLIMIT) prfloor[UU] = UUMINLIMIT;
    out[((i + N1BND) * N2M + (j + N2BND)) * 2 + 0] = prfloor[RHO];
    out[((i + N1BND) * N2M + (j + N2BND)) * 2 + 1] = prfloor[UU];
  }
}

/* horizon accounting of diag_flux() (diag.c:576-833), global region, inner
   x1 face: pdot[X1DN][RHO], pdot[X1DN][UU], pdotterms[X1DN][3][UU],
   pdotterms[X1DN][6][UU] of the last step, pcum[X1DN][RHO], pcum[X1DN][UU] */
void hr_get_horizon(double *out)
{
  out[0] = pdotreg[GLOBALENERREGION][X1DN][RHO];
  out[1] = pdotreg[GLOBALENERREGION][X1DN][UU];
  out[2] = pdottermsreg[GLOBALENERREGION][X1DN][3][UU];
  out[3] = pdottermsreg[GLOBALENERREGION][X1DN][6][UU];
  out[4] = pcumreg[GLOBALENERREGION][X1DN][RHO];
  out[5] = pcumreg[GLOBALENERREGION][X1DN][UU];
}

/* one step of the run loop (main.c:35-45 without diagnostics/postdt) */
int hr_step(int nsteps)
{
  int s;
  for (s = 0; s < nsteps; s++) {
    nstroke = 0;
    if (step_ch() != 0) return 1;
    if (error_check(2)) return 2;
    if (failed) return 3;
    nstep++;
  }
  return 0;
}

/* one inversion: U in the evolved form (UEVOLVE, with sqrt(-g)), guess in/out */
int hr_utoprimgen(int i, int j, const double *U, double *pr, int *pfl)
{
  struct of_geom geom;
  FTYPE Uc[NPR], pc[NPR];
  int k;
  get_geometry(i, j, CENT, &geom);
  for (k = 0; k < NPR; k++) { Uc[k] = U[k]; pc[k] = pr[k]; }
  Utoprimgen(EVOLVEUTOPRIM, UEVOLVE, Uc, &geom, pc);
  for (k = 0; k < NPR; k++) pr[k] = pc[k];
  *pfl = pflag[i][j][FLAGUTOPRIMFAIL];
  return 0;
}

/* one inversion by the chosen method (Utoprimgen_pick, step_ch.c:583-600,
   `which` = UTOPRIM5D1 ... UTOPRIM5D2 of step_ch.h:39-53) of U in the
   evolved form, as Utoprimgen feeds it (UtoU to the geometry-free form
   first); pflag is cleared before the call */
int hr_utoprim_pick(int which, int i, int j, const double *U, double *pr, int *pfl)
{
  extern void UtoU(int inputtype, int returntype, struct of_geom *ptrgeom, FTYPE *Uin, FTYPE *Uout);
  extern int Utoprimgen_pick(int which, int parameter, FTYPE *Ugeomfree, struct of_geom *ptrgeom, FTYPE *pr);
  struct of_geom geom;
  FTYPE Uc[NPR], Ug[NPR], pc[NPR];
  int k;
  get_geometry(i, j, CENT, &geom);
  for (k = 0; k < NPR; k++) { Uc[k] = U[k]; pc[k] = pr[k]; }
  UtoU(UEVOLVE, UNOTHING, &geom, Uc, Ug);
  pflag[i][j][FLAGUTOPRIMFAIL] = 0;
  Utoprimgen_pick(which, EVOLVENOENTROPY, Ug, &geom, pc);
  for (k = 0; k < NPR; k++) pr[k] = pc[k];
  *pfl = pflag[i][j][FLAGUTOPRIMFAIL];
  return 0;
}

int hr_tryagain(void) { return UTOPRIMTRYAGAIN; }
