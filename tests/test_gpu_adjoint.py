"""Adjoint of the FP64 torus step (harm_adjoint_run) against central finite
differences of the same objective with the same dt sequence
(harm_run_fixed_dt), and wrapped in a torch.autograd.Function.

Objective: J = w_mass sum dt mdot + w_em sum dt edot + <lam, p_N> (horizon
mass flux, horizon EM energy flux, a random weighting of the final state).
Directional derivatives along seeded random directions must agree to the
tolerance written here."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5  # |<grad, v> - (J(+eps v) - J(-eps v)) / 2 eps| / |.|
EPS = (1e-7, 1e-8, 1e-9)  # relative finite-difference steps, largest first


def _developed(harm, n, nsteps_pre):
    """A torus a few steps after init (so the flow and the repairs are
    live), as a full reference-layout array with its dt.

    The step is piecewise smooth, and a developed state sits exactly on some
    of its kinks.  Floored zones of one radius hold identical rho and u (the
    floors depend on r only), so the x2 limiters see exact ties there.  A
    finite difference that moves one of those zones alone straddles the
    kink, and there the directional derivative is not linear in the
    direction.  A seeded 1e-4 relative perturbation of every zone takes the
    base state off those ties.  Ghost zones are refilled from the active
    zones by the boundary conditions before the first step (harm_adjoint_run
    and harm_run_fixed_dt both do it), so their copies stay tied to their
    sources under any perturbation."""
    h, geom, p0 = harm.torus_context(n, n, lim=harm.LIM_PARA, fluxmethod=harm.FLUX_HLL)
    h.step_ch(nsteps_pre)
    st = h.sync()
    p, _ = h.get_prims()
    h.close()
    p = p * (1.0 + 1e-4 * np.random.default_rng(7).standard_normal(p.shape))
    return geom, p, st["dt"]


def _fd(harm, n, geom, p, dt, dts, wm, we, lam, v):
    """Central difference of the objective along v.  The first step in EPS
    whose forward and backward one-sided differences agree to REL_TOL / 10
    is used, so that no limiter, floor or wavespeed switch lies within
    +-eps (a switch makes the two one-sided differences differ)."""
    J0 = _ctx(harm, n, geom, p, dt).run_fixed_dt(dts, wm, we, lam)
    best = None
    for eps in EPS:
        Jp = _ctx(harm, n, geom, p + eps * v, dt).run_fixed_dt(dts, wm, we, lam)
        Jm = _ctx(harm, n, geom, p - eps * v, dt).run_fixed_dt(dts, wm, we, lam)
        c, f, b = (Jp - Jm) / (2 * eps), (Jp - J0) / eps, (J0 - Jm) / eps
        spread = abs(f - b) / max(abs(c), 1e-300)
        if best is None or spread < best[1]:
            best = (c, spread)
        if spread < REL_TOL / 10:
            break
    return best[0]


def _ctx(harm, n, geom, p, dt):
    par = harm.torus_params(n, n)
    h = harm.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=harm.LIM_PARA, fluxmethod=harm.FLUX_HLL, gam=par.gam,
                     gammamax=par.gammamax)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p)
    h.set_time(0.0, dt, 0)
    return h


def _check(harm, n, geom, p, dt, nsteps, ckpt, wm, we, lam, ndir, seed):
    h = _ctx(harm, n, geom, p, dt)
    J, grad, dts, ms = h.adjoint(nsteps, ckpt, wm, we, lam)
    h.close()
    assert np.isfinite(grad).all() and np.abs(grad).max() > 0
    assert np.abs(grad[:3]).max() == 0 and np.abs(grad[-3:]).max() == 0  # ghost entries
    assert np.abs(grad[:, :3]).max() == 0 and np.abs(grad[:, -3:]).max() == 0
    rng = np.random.default_rng(seed)
    act = np.zeros(p.shape)
    act[3:-3, 3:-3] = 1.0
    worst = 0.0
    for _ in range(ndir):
        v = rng.standard_normal(p.shape) * np.abs(p) * act
        fd = _fd(harm, n, geom, p, dt, dts, wm, we, lam, v)
        an = float((grad * v).sum())
        worst = max(worst, abs(fd - an) / max(abs(fd), abs(an), 1e-300))
    J0 = _ctx(harm, n, geom, p, dt).run_fixed_dt(dts, wm, we, lam)
    assert J0 == J  # the frozen-dt rerun is the same run
    return worst, ms


@pytest.mark.parametrize("nsteps,ckpt", [(1, 1), (6, 4)])
def test_adjoint_matches_finite_differences_final_state(harm, nsteps, ckpt):
    n = 32
    geom, p, dt = _developed(harm, n, 40)
    lam = np.random.default_rng(1).standard_normal(p.shape)
    worst, _ = _check(harm, n, geom, p, dt, nsteps, ckpt, 0.0, 0.0, lam, 6, 2)
    print(f"adjoint vs finite differences, <lam, p_N>, {nsteps} steps: worst relative difference {worst:.2e}")
    assert worst < REL_TOL, worst


def test_adjoint_matches_finite_differences_horizon_fluxes(harm):
    n = 32
    geom, p, dt = _developed(harm, n, 40)
    worst, ms = _check(harm, n, geom, p, dt, 12, 4, 1.0, 1.0, None, 6, 3)
    print(f"adjoint vs finite differences, horizon mass + EM flux, 12 steps: worst {worst:.2e}; "
          f"forward {ms[0]:.2f} ms, backward {ms[1]:.2f} ms")
    assert worst < REL_TOL, worst


def test_torch_autograd_wrapper(harm):
    """The adjoint as the backward of a torch.autograd.Function (test
    harness only): gradcheck-style comparison of one directional
    derivative."""
    torch = pytest.importorskip("torch")
    n = 32
    geom, p, dt = _developed(harm, n, 40)

    class Steps(torch.autograd.Function):
        @staticmethod
        def forward(ctx, p0):
            h = _ctx(harm, n, geom, p0.detach().cpu().numpy(), dt)
            J, grad, dts, _ = h.adjoint(4, 2, 1.0, 1.0, None)
            h.close()
            ctx.save_for_backward(torch.from_numpy(grad))
            ctx.dts = dts
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad

    x = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    J = Steps.apply(x)
    J.backward()
    act = np.zeros(p.shape)
    act[3:-3, 3:-3] = 1.0
    v = np.random.default_rng(5).standard_normal(p.shape) * np.abs(p) * act
    h = _ctx(harm, n, geom, p, dt)
    _, _, dts, _ = h.adjoint(4, 2, 1.0, 1.0, None)
    h.close()
    fd = _fd(harm, n, geom, p, dt, dts, 1.0, 1.0, None, v)
    an = float((x.grad * torch.from_numpy(v)).sum())
    assert abs(fd - an) <= REL_TOL * max(abs(fd), abs(an))
