"""Gradients with respect to the torus's initial vector potential A_phi and
internal energy u (harm_adjoint_run, then harm_torus_vpot_adjoint for A),
against central finite differences through the same init: the field is
rebuilt from the perturbed A (harm_torus_vpot_to_field, normalisation held
fixed), u is perturbed directly, and the frozen-dt run is repeated.

The initial state holds exact ties (floored atmosphere of equal rho and u
along each radius, zero velocity and field outside the torus), where the
step's limiters and wavespeed maxima sit on their kinks.  The directions
therefore stay inside the torus (A_phi perturbed where it exceeds half its
maximum, u where rho > 5% of its maximum).  Along A directions the forward
and backward one-sided differences still part as the run goes on (by ~3e-6
relative after 1 step of this 64^2 grid, ~4e-5 after 6, ~6e-4 after 16,
the same with the data jittered): zeros that a multiplicative jitter
cannot untie (B = 0 outside the field region, u~1 = u~2 = 0) meet the
perturbed field.  Directions along B itself do not show it.  The check
therefore runs 3 steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
# relative finite-difference steps; the one whose forward and backward
# one-sided differences agree best is used (smaller steps drown in the
# objective's round-off: 1e-9 would give ~3e-5 relative noise here)
EPS = (1e-6, 1e-7, 1e-8)


def _setup(harm, n):
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0, A, norm = harm.torus_init_vpot(par, geom)
    return par, geom, p0, A, norm


def _ctx(harm, par, geom, p):
    h = harm.HarmGPU(par.n1, par.n2, geom["dx1"], geom["dx2"], lim=harm.LIM_PARA, fluxmethod=harm.FLUX_HLL,
                     gam=par.gam, gammamax=par.gammamax)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p)
    h.set_time(0.0, 1e-5, 0)  # init_defglobal()'s first dt
    return h


def test_gradient_wrt_vector_potential_and_internal_energy(harm):
    n, nsteps, ckpt = 64, 3, 2  # two checkpoint segments, the second partial
    par, geom, p0, A, norm = _setup(harm, n)
    rng = np.random.default_rng(11)
    torus = p0[..., 0] > 0.05 * p0[3:-3, 3:-3, 0].max()
    lam = rng.standard_normal(p0.shape) * torus[..., None]
    h = _ctx(harm, par, geom, p0)
    J, grad, dts, ms = h.adjoint(nsteps, ckpt, 1.0, 1.0, lam)
    h.close()
    gA = harm.vpot_adjoint(par, geom, grad, norm)
    gu = grad[..., 1]
    assert np.abs(gA).max() > 0 and np.abs(gu).max() > 0

    def objective(Ax, ux):
        p = harm.vpot_to_field(par, geom, Ax, norm, p0)
        p[..., 1] = ux
        return _ctx(harm, par, geom, p).run_fixed_dt(dts, 1.0, 1.0, lam)

    assert objective(A, p0[..., 1]) == J
    worst = 0.0
    for d in range(4):
        vA = rng.standard_normal(A.shape) * (A > 0.5 * A.max()) * A.max()
        vu = rng.standard_normal(gu.shape) * torus * p0[..., 1]
        if d == 0:
            vu = 0 * vu  # the A direction alone
        an = float((gA * vA).sum() + (gu * vu).sum())
        J0 = objective(A, p0[..., 1])
        best = None
        for eps in EPS:
            Jp = objective(A + eps * vA, p0[..., 1] + eps * vu)
            Jm = objective(A - eps * vA, p0[..., 1] - eps * vu)
            c, f, b = (Jp - Jm) / (2 * eps), (Jp - J0) / eps, (J0 - Jm) / eps
            spread = abs(f - b) / max(abs(c), 1e-300)
            if best is None or spread < best[1]:
                best = (c, spread)
        fd = best[0]
        err = abs(fd - an) / max(abs(fd), abs(an), 1e-300)
        print(f"direction {d}: adjoint {an:.6e}, finite difference {fd:.6e} (one-sided spread {best[1]:.1e}), "
              f"relative difference {err:.1e}")
        worst = max(worst, err)
    print(f"d/dA_phi, d/du vs finite differences, {nsteps} steps: worst relative difference {worst:.2e}")
    assert worst < REL_TOL, worst
