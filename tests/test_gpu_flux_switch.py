"""The per-zone HLL/LAXF switch (FLUXADJUST, harm_config.fluxadjust) on the
GPU against the oracle and the reference built with FLUXADJUST
FLUXBSQORHOANDU ("torusfa"): primitives, inversion flags, the flux choice
of every zone (pflag[..][FLAGREALFLUX] over the range get_bsqflags sets),
fluxes, t and dt equal after every step.

Lowered b^2 / Lorentz-factor thresholds make the switch pick LAXF in a large
share of the zones from the first step on; the reference's own thresholds
are run too (the switch then acts in a few zones of the developing flow).
"""
import numpy as np
import pytest

import harmtest as ht
from test_oracle_vs_reference import FLUXADJUST_LIMITS

pytestmark = pytest.mark.gpu

LIMITS = dict(zip(("bsqorholimit", "bsqoulimit", "gammadamp"), FLUXADJUST_LIMITS))


def _setup(harm, n, lim, flux, limits, precision=0):
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    kw = dict(limits or {})
    o = ht.Oracle(n, n, geom, lim=lim, fluxmethod=flux, dx1=geom["dx1"], dx2=geom["dx2"], fluxadjust=3, **kw)
    po = o.bound(p0)
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    h = harm.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=lim, fluxmethod=flux, fluxadjust=3, precision=precision,
                     **kw)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p0)
    h.bound_prims()
    h.set_time(0.0, 1e-5, 0)
    return h, o, po, fo


def _check(h, po, fo, what):
    pg, fg = h.get_prims()
    if not np.array_equal(pg, po):
        bad = np.argwhere(pg != po)
        raise AssertionError(f"{what}: {len(bad)} values differ, first {bad[:4].tolist()}")
    assert np.array_equal(fg[3:-3, 3:-3, 0], fo[3:-3, 3:-3, 0]), f"{what}: inversion flags differ"
    assert np.array_equal(fg[2:-2, 2:-2, 4], fo[2:-2, 2:-2, 4]), f"{what}: flux choices differ"
    return int((fg[2:-2, 2:-2, 4] == 0).sum())


@pytest.mark.parametrize("n,lim,flux,nsteps,limits", [(32, 4, 1, 150, LIMITS), (32, 3, 1, 100, LIMITS),
                                                     (32, 4, 1, 400, None), (64, 4, 1, 60, LIMITS)])
def test_gpu_flux_switch_matches_oracle(harm, n, lim, flux, nsteps, limits):
    h, o, po, fo = _setup(harm, n, lim, flux, limits)
    t, dt = 0.0, 1e-5
    nlaxf = 0
    for s in range(1, nsteps + 1):
        rc, t, dt = o.step(po, fo, t, dt)
        assert rc == 0
        h.step_ch(1)
        st = h.sync()
        nlaxf += _check(h, po, fo, f"step {s}")
        assert (st["t"], st["dt"]) == (t, dt)
    f1g, f2g = h.get_fluxes()
    f1o, f2o = o.fluxes()
    assert np.array_equal(f1g[3:-3, 3:-3], f1o[3:-3, 3:-3]) and np.array_equal(f2g[3:-3, 3:-3], f2o[3:-3, 3:-3])
    assert nlaxf > 0
    print(f"\n{n}^2 lim {lim}: {nlaxf} zone-steps with LAXF hydro fluxes over {nsteps} steps")
    h.close()


def test_gpu_flux_switch_matches_reference(harm):
    lim, flux, n, nsteps = 3, 1, 32, 100
    r = ht.ref_run(n, n, lim=lim, flux=flux, nsteps=nsteps, problem="torusfa", limits=FLUXADJUST_LIMITS)
    if r is None:
        pytest.skip("reference build (oracle/_ref) with FLUXADJUST not present")
    cfg = ht.ref_config(r)
    h = harm.HarmGPU(n, n, cfg.pop("dx1"), cfg.pop("dx2"), lim=lim, fluxmethod=flux, **cfg)
    g = r["geom"]
    h.upload_geometry(g["gcov"], g["gcon"], g["gdet"], g["conn"], g["floors"])
    h.set_prims(r["prims"][0], r["pflag"][0])
    h.set_time(r["times"][0][0], r["times"][0][1], 0)
    for s in range(1, nsteps + 1):
        h.step_ch(1)
        st = h.sync()
        pg, fg = h.get_prims()
        assert np.array_equal(pg, r["prims"][s]), f"step {s}"
        assert np.array_equal(fg[3:-3, 3:-3, 0], r["pflag"][s][3:-3, 3:-3, 0])
        assert np.array_equal(fg[2:-2, 2:-2, 4], r["pflag"][s][2:-2, 2:-2, 4])
        assert (st["t"], st["dt"]) == tuple(r["times"][s])
    h.close()


@pytest.mark.slow
def test_gpu_flux_switch_torus512(harm):
    """The benchmark size: 3 steps against the oracle, 1 against the reference."""
    h, o, po, fo = _setup(harm, 512, 4, 1, LIMITS)
    t, dt = 0.0, 1e-5
    for s in range(1, 4):
        rc, t, dt = o.step(po, fo, t, dt)
        h.step_ch(1)
        st = h.sync()
        nl = _check(h, po, fo, f"512^2 step {s}")
        assert (st["t"], st["dt"]) == (t, dt) and nl > 0
    h.close()
    r = ht.ref_run(512, 512, lim=4, flux=1, nsteps=1, problem="torusfa", limits=FLUXADJUST_LIMITS)
    if r is None:
        pytest.skip("reference build (oracle/_ref) of the 512^2 torus with FLUXADJUST not present")
    cfg = ht.ref_config(r)
    h = harm.HarmGPU(512, 512, cfg.pop("dx1"), cfg.pop("dx2"), lim=4, fluxmethod=1, **cfg)
    g = r["geom"]
    h.upload_geometry(g["gcov"], g["gcon"], g["gdet"], g["conn"], g["floors"])
    h.set_prims(r["prims"][0], r["pflag"][0])
    h.set_time(r["times"][0][0], r["times"][0][1], 0)
    h.step_ch(1)
    st = h.sync()
    pg, fg = h.get_prims()
    assert np.array_equal(pg, r["prims"][1]) and (st["t"], st["dt"]) == tuple(r["times"][1])
    assert np.array_equal(fg[2:-2, 2:-2, 4], r["pflag"][1][2:-2, 2:-2, 4])
    h.close()


def test_gpu_flux_switch_mixed_precision_runs(harm):
    """The mixed form with the switch: same choices as FP64 where the
    FP64 state decides them (the flags come from the FP64 state), results
    within the mixed form's tolerance of FP64 after 30 steps."""
    out = {}
    for prec in (0, 1):
        h, o, po, fo = _setup(harm, 64, 4, 1, LIMITS, precision=prec)
        h.step_ch(30)
        h.sync()
        out[prec] = h.get_prims()[0][3:-3, 3:-3]
        h.close()
    d = np.abs(out[1][..., 0] - out[0][..., 0]).sum() / np.abs(out[0][..., 0]).sum()
    assert 0 < d < 1e-5, d
