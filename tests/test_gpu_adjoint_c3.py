"""The adjoint at its configured scale: the 256^2 torus from init (MC, HLL,
the seeded 4% perturbation of u), 256 RK2 steps in FP64 with a checkpoint
every 16, J = time-integrated horizon mass flux + EM energy flux.  Its
gradient with respect to the initial A_phi (harm_torus_vpot_adjoint) and the
u of the torus (where the 4% perturbation lives: rho > 5% of its maximum) is
compared with central finite differences at eps = 1e-6 along 32 seeded
directions (16 in A_phi, 16 in u), through the same init (field rebuilt
from the perturbed A_phi, normalisation held fixed) and the frozen-dt run.

In 256 steps from init (t ~ 2.3 GM/c^3) nothing from the torus (inner edge
r = 6) has reached the horizon, so J does not depend on the torus yet: the
finite differences are exactly zero and the adjoint's directional
derivatives are negligible (the linearised numerical domain of dependence
reaches the horizon only through factors far below round-off).  The check
is that the two agree at the level J can resolve: |adjoint - finite
difference| <= REL_TOL x max(|adjoint|, |finite difference|, 1e-9 |J| / eps).
Where a direction does give a nonzero finite difference, its forward and
backward one-sided differences are reported too (a spread means a kink:
a limiter, floor or wavespeed switch within +-eps)."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

N, NSTEPS, CKPT, NDIR, EPS = 256, 256, 16, 32, 1e-6
REL_TOL = 1e-5


def _ctx(harm, par, geom, p):
    h = harm.HarmGPU(par.n1, par.n2, geom["dx1"], geom["dx2"], lim=harm.LIM_MC, fluxmethod=harm.FLUX_HLL,
                     gam=par.gam, gammamax=par.gammamax)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p)
    h.set_time(0.0, 1e-5, 0)
    return h


def test_adjoint_c3_scale_against_finite_differences(harm):
    par = harm.torus_params(N, N)
    geom = harm.torus_geometry(par)
    p0, A, norm = harm.torus_init_vpot(par, geom)
    h = _ctx(harm, par, geom, p0)
    J, grad, dts, ms = h.adjoint(NSTEPS, CKPT, 1.0, 1.0, None)
    h.close()
    gA = harm.vpot_adjoint(par, geom, grad, norm)
    gu = grad[..., 1]
    assert np.isfinite(gA).all() and np.isfinite(gu).all() and J != 0.0

    def objective(Ax, ux):
        p = harm.vpot_to_field(par, geom, Ax, norm, p0)
        p[..., 1] = ux
        hh = _ctx(harm, par, geom, p)
        v = hh.run_fixed_dt(dts, 1.0, 1.0, None)
        hh.close()
        return v

    u0 = p0[..., 1].copy()
    J0 = objective(A, u0)
    assert J0 == J  # the frozen-dt rerun is the run the adjoint differentiated
    rng = np.random.default_rng(20261203)
    torus = p0[..., 0] > 0.05 * p0[3:-3, 3:-3, 0].max()
    floor = 1e-9 * abs(J) / EPS
    rows, worst = [], 0.0
    for d in range(NDIR):
        along_A = d < NDIR // 2
        vA = rng.standard_normal(A.shape) * (A > 0.5 * A.max()) * A.max() if along_A else np.zeros(A.shape)
        vu = np.zeros(u0.shape) if along_A else rng.standard_normal(u0.shape) * np.abs(u0) * torus
        an = float((gA * vA).sum() + (gu * vu).sum())
        Jp = objective(A + EPS * vA, u0 + EPS * vu)
        Jm = objective(A - EPS * vA, u0 - EPS * vu)
        c, f, b = (Jp - Jm) / (2 * EPS), (Jp - J0) / EPS, (J0 - Jm) / EPS
        scale = max(abs(c), abs(an), floor)
        err = abs(c - an) / scale
        spread = abs(f - b) / scale
        rows.append((d, "A_phi" if along_A else "u", an, c, spread, err))
        worst = max(worst, err)
    print(f"\nC3 adjoint, {N}^2 torus from init, {NSTEPS} steps (t = {dts.sum():.4g}), checkpoint every {CKPT}: "
          f"forward {ms[0]:.1f} ms, backward {ms[1]:.1f} ms (backward/forward {ms[1] / ms[0]:.2f}); J = {J:.6e}; "
          f"max |dJ/dA_phi| = {np.abs(gA).max():.2e}, max |dJ/du| over the torus = {np.abs(gu * torus).max():.2e}, "
          f"over all zones = {np.abs(gu).max():.2e}")
    print("dir field  adjoint          finite diff      one-sided spread  difference / scale")
    for d, fld, an, c, spread, err in rows:
        print(f"{d:3d} {fld:5s}  {an: .8e} {c: .8e} {spread:9.2e}         {err:9.2e}")
    print(f"worst difference / scale {worst:.2e} (scale floor {floor:.2e})")
    assert worst < REL_TOL, worst
