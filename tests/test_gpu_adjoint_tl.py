"""The adjoint kernels against the tangent-linear reference: <dJ/dp_0, v>
from harm_adjoint_run on the GPU equals dJ along v from the tangent-linear
form of the oracle (oracle/harm_oracle_tl.cpp, forward mode through the
same step, the same dt sequence) for 32 seeded directions, to REL_TOL.

The GPU's forward run is the oracle's bit for bit, so both take the same
branch at every limiter, floor, repair and wavespeed choice: the comparison
is between two exact derivatives of the same piecewise-smooth map (the
adjoint's inversion derivative from the implicit-function theorem at the
converged state, the tangent's through the Newton iterations), not against
finite differences.  J = time-integrated horizon mass flux + EM energy
flux (+ a weighting of the final state in one case)."""
import numpy as np
import pytest

import harmtest as ht

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10
NDIR = 32


def _developed(harm, n, nsteps_pre, lim):
    h, geom, p0 = harm.torus_context(n, n, lim=lim, fluxmethod=harm.FLUX_HLL)
    h.step_ch(nsteps_pre)
    st = h.sync()
    p, _ = h.get_prims()
    h.close()
    p = p * (1.0 + 1e-4 * np.random.default_rng(7).standard_normal(p.shape))
    return geom, p, st["dt"]


def _ctx(harm, n, geom, p, dt, lim):
    par = harm.torus_params(n, n)
    h = harm.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=lim, fluxmethod=harm.FLUX_HLL, gam=par.gam,
                     gammamax=par.gammamax)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p)
    h.set_time(0.0, dt, 0)
    return h


@pytest.mark.parametrize("n,lim,pre,nsteps,ckpt", [(32, 4, 40, 12, 4), (32, 3, 60, 16, 16), (64, 4, 100, 8, 4)])
def test_adjoint_matches_tangent_linear(harm, n, lim, pre, nsteps, ckpt):
    geom, p, dt = _developed(harm, n, pre, lim)
    h = _ctx(harm, n, geom, p, dt, lim)
    J, grad, dts, _ = h.adjoint(nsteps, ckpt, 1.0, 1.0, None)
    h.close()
    par = harm.torus_params(n, n)
    tl = ht.OracleTL(n, n, geom, lim=lim, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"], gam=par.gam,
                     gammamax=par.gammamax)
    rng = np.random.default_rng(100 + n + lim)
    act = np.zeros(p.shape)
    act[3:-3, 3:-3] = 1.0
    # the adjoint takes a tie's rows for a field component whose stencil is
    # round-off (below 1e-10 sqrt(rho), harm_adjoint.cu k_adj_recon): there
    # it is not the derivative of the branch the round-off picked, which the
    # tangent follows.  The checked directions leave the field alone in and
    # next to such zones (|B| < 1e-6 sqrt(rho) within two zones); the others
    # are reported.
    quiet = np.abs(p[..., 5:8]) < 1e-6 * np.sqrt(np.maximum(p[..., 0:1], 0.0))
    near = quiet.copy()
    for sh in (-2, -1, 1, 2):
        near |= np.roll(quiet, sh, axis=0) | np.roll(quiet, sh, axis=1)
    fieldmask = np.ones(p.shape)
    fieldmask[..., 5:8] = ~near
    errs, errs_all = [], []
    for d in range(NDIR):
        v = rng.standard_normal(p.shape) * np.abs(p) * act
        for vv, out in ((v * fieldmask, errs), (v, errs_all)):
            Jt, dJ, _, _ = tl.objective(p, vv, dts)
            an = float((grad * vv).sum())
            out.append(abs(an - dJ) / max(abs(an), abs(dJ), 1e-300))
    assert abs(Jt - J) <= 1e-14 * abs(J), (Jt, J)  # the same objective (summed in another order)
    errs, errs_all = np.array(errs), np.array(errs_all)
    print(f"\nadjoint vs tangent-linear, {n}^2 lim {lim}, {nsteps} steps (checkpoint every {ckpt}), {NDIR} directions: "
          f"relative differences median {np.median(errs):.2e}, worst {errs.max():.2e}; with the field of the "
          f"round-off zones in the directions too: median {np.median(errs_all):.2e}, worst {errs_all.max():.2e} "
          f"({near.mean():.2f} of the field components masked)")
    assert errs.max() < REL_TOL, errs.max()
