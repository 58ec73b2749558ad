/*
 * harm_setup.h -- host-side problem set-up for standalone runs: the grid
 * geometry and the initial state of the reference's plugin surface (coord.c,
 * metric.c, set_grid.c, initbase.c) for the Fishbone-Moncrief torus
 * (init.fishmon.c) and the force-free aligned rotator (init.ns.c).
 *
 * A drop-in host keeps calling the reference's own set_grid()/init(); these
 * entry points exist so that the library can produce the same inputs without
 * the reference.  All arrays use the reference layout described in
 * harm_b200.h.
 */
#ifndef HARM_SETUP_H
#define HARM_SETUP_H

#include "harm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct harm_torus_params {
  int n1, n2;             /* interior zones */
  int seed;               /* ranc() seed of init_global (init.fishmon.c:64) */
  int reserved;
  double a;               /* black-hole spin (init.fishmon.c:40) */
  double hslope;          /* MKS theta concentration (defcoord 0) */
  double rout;            /* outer radius */
  double rin_over_rhor;   /* Rin = rin_over_rhor * r_horizon */
  double gam;             /* adiabatic index */
  double torus_rin, torus_rmax, kappa, beta, randfact;  /* init.fishmon.c:134-139 */
  double rhomin, uumin;   /* floor coefficients, rho >= rhomin r^-1.5, u >= uumin r^-2.5 */
  double rhominlimit, uuminlimit;
  double gammamax;
} harm_torus_params;

/* The benchmark torus: a = 0.9375, hslope 0.3, Rout 40, Rin = 0.98 r_h,
   rin 6, rmax 12, kappa 1e-3, beta 100, 4% seeded u perturbation (seed 7),
   gamma 4/3, floors 1e-4 r^-1.5 / 1e-6 r^-2.5, GAMMAMAX 25, 128 x 128. */
void harm_torus_default_params(harm_torus_params* p);

/* set_grid() (set_grid.c:6-89) for MKS defcoord 0 on Kerr-Schild: gcov,
   gcon, gdet at the four grid locations, the numerical connection at CENT
   (metric.c:1188-1262) and the per-zone floors.  grid_out (may be NULL)
   receives startx1, startx2, dx1, dx2, Rin, r_horizon. */
int harm_torus_geometry(const harm_torus_params* p, double* gcov, double* gcon, double* gdet, double* conn,
                        double* floors, double* grid_out);

/* init()'s fresh start (initbase.c:297-562) with the torus of
   init.fishmon.c, given the geometry from harm_torus_geometry().  Active
   zones are final; ghost zones still need bound_prim (harm_bound_prims()
   on the device, after harm_set_prims()). */
int harm_torus_init(const harm_torus_params* p, const double* gcov, const double* gcon, const double* gdet,
                    double* prims);

/* harm_torus_init() that also returns the corner vector potential A_phi
   (init_vpot, init.fishmon.c:236-268), [n1+1][n2+1] at corners (i, j) of
   the active grid, and the two field normalisation factors norm[2]
   (normalize_field, init.fishmon.c:310-375, applied twice). */
int harm_torus_init_vpot(const harm_torus_params* p, const double* gcov, const double* gcon, const double* gdet,
                         double* prims, double* A, double* norm);

/* B1, B2 of the active zones from a corner vector potential: vpot2field
   (initbase.c:565-618) then the normalisation by norm[0], norm[1] (the
   factors harm_torus_init_vpot() returned, held fixed).  With the A and
   norm of harm_torus_init_vpot() it reproduces the init's field exactly. */
int harm_torus_vpot_to_field(const harm_torus_params* p, const double* gdet, const double* A, const double* norm,
                             double* prims);

/* The adjoint of harm_torus_vpot_to_field(): grad_A [n1+1][n2+1] from the
   gradient grad_prims [n1m][n2m][8] of an objective with respect to the
   primitives (its B1, B2 entries of the active zones), e.g. the gradient
   harm_adjoint_run() returns with respect to the initial state. */
int harm_torus_vpot_adjoint(const harm_torus_params* p, const double* gdet, const double* grad_prims,
                            const double* norm, double* grad_A);

/* The coordinate columns of the torus grid for harm_write_dump(): the dump
   header's plugin scalars (defcoord 0) and X1, X2, r, th at every zone
   centre, [n1m][n2m][4] (coord.c:920-938, bl_coord coord.c:334-453). */
int harm_torus_dump_coords(const harm_torus_params* p, harm_dump_header* hdr, double* coords);

/* The force-free aligned rotator of init.ns.c + bounds.ns.c (EOMFFDE,
   MCOORD SPCMINKMETRIC): flat space in spherical polar coordinates,
   defcoord 6 (log r, uniform theta), r in [rin, rout] stellar radii, a dipole
   field A_phi = bpole rin^3 sin^2(theta) / (2 r) (init.ns.c:525) and a
   stellar surface rotating at omegastar (bounds.ns.c:108). */
typedef struct harm_dipole_params {
  int n1, n2;             /* interior zones */
  double rin, rout;       /* stellar surface and outer radius (init_grid) */
  double gam;             /* adiabatic index (init_global) */
  double bpole;           /* polar field (pre_init_specific_init, init.ns.c:50) */
  double omegastar;       /* surface angular frequency (HARM_BC_STAR) */
  double rhomin, uumin;   /* floor coefficients (init_global, rescaletype 0) */
  double rhominlimit, uuminlimit;
  double gammamax;
} harm_dipole_params;

/* 512 x 256, rin 1, rout 100, gamma 4/3, bpole 1, omegastar 0.2, floors
   1e-10 r^-1.5 / 1e-11 r^-2.5, GAMMAMAX 25. */
void harm_dipole_default_params(harm_dipole_params* p);

/* set_grid() for defcoord 6 on flat space (the metric inverse by
   Gauss-Jordan, matrix_inverse, metric.c:1146-1162): the tables of
   harm_torus_geometry() for the dipole grid.  grid_out (may be NULL)
   receives startx1, startx2, dx1, dx2, Rin, Rout. */
int harm_dipole_geometry(const harm_dipole_params* p, double* gcov, double* gcon, double* gdet, double* conn,
                         double* floors, double* grid_out);

/* init()'s fresh start (initbase.c:297-562) for EOMFFDE with init.ns.c's
   star without a disk: the zero atmosphere (set_atmosphere, fixup.c:1119-1190)
   round-tripped through the relative 4-velocity, the dipole vector potential
   at every corner and vpot2field over the whole grid (initbase.c:565-618),
   filterffde twice (phys.ffde.c:1957-1980: state, conserved quantities and
   the force-free inversion, densities zeroed), then fixup's Lorentz-factor
   limit on the active zones.  Every zone is set, ghost zones included (the
   star's boundary holds the ghosts' field); the caller still bounds the
   state (harm_bound_prims() on the device). */
int harm_dipole_init(const harm_dipole_params* p, const double* gcov, const double* gcon, const double* gdet,
                     double* prims);

#ifdef __cplusplus
}
#endif
#endif
