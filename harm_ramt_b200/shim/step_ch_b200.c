/*
 * step_ch_b200.c -- the reference-side binding of the B200 step: a drop-in
 * replacement for the reference's  int step_ch(void)  (step_ch.c:16,
 * declared global.h:1383), compiled into the reference's own build in place
 * of that function and linked against libharm_b200.so (include/harm_b200.h).
 *
 * main.c, init(), diag(), dump() and the restart files stay as they are.
 * The first call creates the device context from the reference's run-time
 * knobs (initbase.c:119-243 and the problem's init_global) and its
 * compile-time grid (global.h:126-127), uploads the geometry tables of
 * set_grid() and the per-zone floors once, and the state p/pflag with t,
 * dt and realnstep.  Every call then advances the device-resident state by
 * one step and copies p and pflag back, because the reference's
 * diagnostics read them after every step; a host that only needs them at
 * dump times can move that copy there.  A fatal check on the device is
 * reported through the reference's own fail() with the same code and zone
 * (icurr, jcurr) the reference would report.
 *
 * Build: this file in the reference's source list, step_ch.c's step_ch()
 * renamed or removed, -I<repo>/include, and
 * -L<repo>/harm_ramt_b200 -lharm_b200 -Wl,-rpath,<repo>/harm_ramt_b200.
 */
#include "decs.h"
#include "step_ch.h"
#include "harm_b200.h"

static harm_ctx *b200_ctx = NULL;

static int b200_setup(void)
{
  harm_config cfg = {0};
  static FTYPE floors[N1M][N2M][2];
  struct of_geom geom;
  FTYPE prfloor[NPR];
  int i, j, rc;

  cfg.n1 = N1;
  cfg.n2 = N2;
  cfg.lim = lim;
  cfg.fluxmethod = fluxmethod;
#if (EOMTYPE == EOMFFDE)
  cfg.eom = HARM_EOM_FFDE;
#else
  cfg.eom = HARM_EOM_GRMHD;
#endif
  cfg.precision = HARM_PREC_FP64;
  cfg.cour = cour;
  cfg.gam = gam;
  cfg.dx1 = dx[1];
  cfg.dx2 = dx[2];
  cfg.safe = SAFE;
  cfg.defcon = defcon;
  cfg.gammamax = GAMMAMAX;
  cfg.gammafail = GAMMAFAIL;
  cfg.bsqorholimit = BSQORHOLIMIT;
  cfg.bsqoulimit = BSQOULIMIT;
  cfg.tf = tf;
  cfg.bc = (BCtype[X1DN] == NSSURFACE) ? HARM_BC_STAR : HARM_BC_TORUS;
  cfg.omegastar = Omegastar;
  cfg.tryagain = UTOPRIMTRYAGAIN;
  cfg.fluxadjust = FLUXADJUST;
  cfg.gammadamp = GAMMADAMP;
  if ((rc = harm_create(&cfg, NULL, &b200_ctx)) != HARM_OK) return rc;

  /* the floors exactly as fixup1zone() forms them (fixup.c:295-307) */
  FULLLOOP {
    get_geometry(i, j, CENT, &geom);
    set_density_floors(&geom, p[i][j], prfloor);
    floors[i + N1BND][j + N2BND][0] = (prfloor[RHO] < RHOMINLIMIT) ? RHOMINLIMIT : prfloor[RHO];
    floors[i + N1BND][j + N2BND][1] = (prfloor[UU] < UUMINLIMIT) ? UUMINLIMIT : prfloor[UU];
  }
  if ((rc = harm_upload_geometry(b200_ctx, &a_gcov[0][0][0][0][0], &a_gcon[0][0][0][0][0], &a_gdet[0][0][0],
                                 &a_conn[0][0][0][0][0], &floors[0][0][0])) != HARM_OK)
    return rc;
  if ((rc = harm_set_prims(b200_ctx, &a_p[0][0][0], &a_pflag[0][0][0], 1)) != HARM_OK) return rc;
  return harm_set_time(b200_ctx, t, dt, realnstep);
}

int step_ch(void)
{
  harm_status st;
  int rc;
  if (!b200_ctx && (rc = b200_setup()) != HARM_OK) {
    dualfprintf(fail_file, "step_ch_b200: %s\n", harm_error_string(rc));
    return 1;
  }
  if ((rc = harm_step(b200_ctx, 1)) != HARM_OK) return 1;
  rc = harm_sync(b200_ctx, &st);
  t = st.t;
  dt = st.dt;
  realnstep = st.realnstep;
  if (rc == HARM_EFAIL) {
    icurr = st.fail_i; /* the zone the reference's fail() prints */
    jcurr = st.fail_j;
    fail(st.fail_code);
    return 1;
  }
  if (rc != HARM_OK) return 1;
  return harm_get_prims(b200_ctx, &a_p[0][0][0], &a_pflag[0][0][0]) != HARM_OK;
}
