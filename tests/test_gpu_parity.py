"""GPU step vs the oracle (C restatement) and the compiled reference.

The bar is bit-for-bit equality of every primitive in every active zone, of
the inversion-failure flags, and of t and dt, after each step: the FP64
kernels keep the reference's evaluation order and are built without
multiply-add contraction.  Ghost zones are compared for the primitives too.
"""
import numpy as np
import pytest

import harmtest as ht

pytestmark = pytest.mark.gpu

I = ht.interior


def _gpu_from(hb, n, geom, p0, pflag0, t0, dt0, lim, flux, cfg=None):
    cfg = cfg or {}
    h = hb.HarmGPU(n, n, cfg.get("dx1", geom.get("dx1")), cfg.get("dx2", geom.get("dx2")), lim=lim, fluxmethod=flux,
                   **{k: v for k, v in cfg.items() if k not in ("dx1", "dx2")})
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p0, pflag0)
    h.set_time(t0, dt0, 0)
    return h


def _assert_same(pg, fg, po, fo, what):
    same = np.array_equal(pg, po)
    if not same:
        bad = np.argwhere(pg != po)
        d = np.abs(pg - po).max()
        raise AssertionError(f"{what}: {len(bad)} primitive values differ (max abs {d:.3e}), first {bad[:4].tolist()}")
    assert np.array_equal(I(fg)[..., 0], I(fo)[..., 0]), f"{what}: inversion flags differ"


@pytest.mark.parametrize("lim,flux,nsteps", [(3, 1, 40), (4, 0, 30), (4, 1, 30)])
def test_gpu_matches_oracle_torus32(harm, lim, flux, nsteps):
    n = 32
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=lim, fluxmethod=flux, dx1=geom["dx1"], dx2=geom["dx2"])
    po = o.bound(p0)
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    h = _gpu_from(harm, n, geom, p0, None, 0.0, 1e-5, lim, flux)
    h.bound_prims()
    pg, fg = h.get_prims()
    _assert_same(pg, fg, po, fo, "after bound")
    t, dt = 0.0, 1e-5
    for s in range(nsteps):
        rc, t, dt = o.step(po, fo, t, dt)
        assert rc == 0
        h.step_ch(1)
        st = h.sync()
        pg, fg = h.get_prims()
        _assert_same(pg, fg, po, fo, f"step {s + 1}")
        assert st["t"] == t and st["dt"] == dt, (st, t, dt)
        assert list(h.get_horizon().values()) == list(o.horizon()), f"step {s + 1}: horizon accounting"
    f1g, f2g = h.get_fluxes()
    f1o, f2o = o.fluxes()
    assert np.array_equal(f1g[3:-3, 3:-3], f1o[3:-3, 3:-3]) and np.array_equal(f2g[3:-3, 3:-3], f2o[3:-3, 3:-3])


def test_end_time_clamp_matches_oracle(harm):
    """The run stops exactly on a moved end time and continues from it as
    the oracle does (the last step clamped onto each end time)."""
    n = 32
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    po = o.bound(p0)
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    h = _gpu_from(harm, n, geom, p0, None, 0.0, 1e-5, 4, 1)
    h.bound_prims()
    t, dt, nstep = 0.0, 1e-5, 0
    for tf in (0.05, 0.2):
        dt = o.set_end_time(tf, t, dt)
        while t < tf:
            rc, t, dt = o.step(po, fo, t, dt)
            assert rc == 0
            nstep += 1
        st = h.run_to(tf)
        assert st["t"] == t == tf and st["dt"] == dt == 0.0 and st["realnstep"] == nstep
        pg, fg = h.get_prims()
        _assert_same(pg, fg, po, fo, f"at t={tf}")


def test_gpu_matches_reference_torus32(harm):
    r = ht.ref_run(32, 32, lim=3, flux=1, nsteps=25)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    cfg = ht.ref_config(r)
    cfg["currents"] = True
    h = _gpu_from(harm, 32, r["geom"], r["prims"][0], r["pflag"][0], r["times"][0][0], r["times"][0][1], 3, 1, cfg)
    assert all(np.array_equal(x, y) for x, y in zip(h.get_currents(), r["currents"][0])), "t=0 currents"
    for s in range(1, 26):
        h.step_ch(1)
        st = h.sync()
        pg, fg = h.get_prims()
        _assert_same(I(pg), fg, I(r["prims"][s]), r["pflag"][s], f"step {s}")
        assert (st["t"], st["dt"]) == tuple(r["times"][s])
        assert list(h.get_horizon().values()) == list(r["horizon"][s]), f"step {s}: horizon accounting"
        jc, fc, cf = h.get_currents()
        rj, rf, rc = r["currents"][s]
        assert np.array_equal(jc, rj) and np.array_equal(fc, rf) and np.array_equal(cf, rc), f"step {s}: currents"


@pytest.mark.slow
def test_gpu_matches_oracle_torus512_one_step(harm):
    """Full benchmark size: one step against the oracle, bit for bit."""
    n = 512
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    po = o.bound(p0)
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    h = _gpu_from(harm, n, geom, p0, None, 0.0, 1e-5, 4, 1)
    h.bound_prims()
    rc, t, dt = o.step(po, fo, 0.0, 1e-5)
    h.step_ch(1)
    st = h.sync()
    pg, fg = h.get_prims()
    _assert_same(pg, fg, po, fo, "512^2 step 1")
    assert st["t"] == t and st["dt"] == dt
