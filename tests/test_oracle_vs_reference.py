"""The C restatement (oracle) against the reference compiled from its own
sources (oracle/_ref): identical initial state and geometry, bit-for-bit
equal primitives, inversion flags, t and dt after every step.  Skipped where
the reference build is absent (it is built from the reference tree)."""
import numpy as np
import pytest

import harmtest as ht

CASES = [(16, 3, 1, 120), (32, 4, 0, 60), (32, 4, 1, 60), (64, 3, 1, 25)]


@pytest.mark.parametrize("n,lim,flux,nsteps", CASES)
def test_oracle_matches_reference(n, lim, flux, nsteps):
    r = ht.ref_run(n, n, lim=lim, flux=flux, nsteps=nsteps)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    o = ht.Oracle(n, n, r["geom"], lim=lim, fluxmethod=flux, **ht.ref_config(r))
    p = r["prims"][0].copy()
    f = r["pflag"][0].copy()
    t, dt = r["times"][0]
    o.init_currents(p, dt)
    assert all(np.array_equal(x, y) for x, y in zip(o.currents(), r["currents"][0])), "t=0 currents differ"
    nfixed = 0
    for s in range(1, nsteps + 1):
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
        assert np.array_equal(p, r["prims"][s]), f"step {s}: primitives differ"
        assert np.array_equal(f[3:-3, 3:-3, 0], r["pflag"][s][3:-3, 3:-3, 0]), f"step {s}: flags differ"
        assert (t, dt) == tuple(r["times"][s]), f"step {s}: t/dt differ"
        assert np.array_equal(o.horizon(), r["horizon"][s]), f"step {s}: horizon accounting differs"
        assert all(np.array_equal(x, y) for x, y in zip(o.currents(), r["currents"][s])), f"step {s}: currents"
        nfixed += int((f[3:-3, 3:-3, 0] == -1).sum())
    f1, f2 = o.fluxes()
    I = ht.interior
    assert np.array_equal(I(f1), I(r["F1"])) and np.array_equal(I(f2), I(r["F2"]))
    # the run exercised the Newton cycle break (the reference's count is
    # cumulative from init, the oracle's from this run)
    assert r["ncyclebreak"] >= o.ncyclebreak()


# force-free aligned rotator (phys.ffde.c, bounds.ns.c): n1 x n2 grid,
# limiter, flux, steps
DIPOLE_CASES = [(32, 16, 3, 0, 300), (32, 16, 4, 1, 150), (64, 32, 3, 1, 40)]


@pytest.mark.parametrize("n1,n2,lim,flux,nsteps", DIPOLE_CASES)
def test_oracle_matches_reference_dipole_ffde(n1, n2, lim, flux, nsteps):
    r = ht.ref_run(n1, n2, lim=lim, flux=flux, nsteps=nsteps, problem="dipole")
    if r is None:
        pytest.skip("reference build (oracle/_ref) of the dipole problem not present")
    assert r["eomtype"] == 1
    o = ht.Oracle(n1, n2, r["geom"], lim=lim, fluxmethod=flux, eom=1, bc=1, omegastar=r["omegastar"],
                  **ht.ref_config(r))
    p = r["prims"][0].copy()
    f = r["pflag"][0].copy()
    t, dt = r["times"][0]
    o.init_currents(p, dt)
    for s in range(1, nsteps + 1):
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
        assert np.array_equal(p, r["prims"][s]), f"step {s}: primitives differ"
        assert all(np.array_equal(x, y) for x, y in zip(o.currents(), r["currents"][s])), f"step {s}: currents"
        assert np.array_equal(f[..., 0], r["pflag"][s][..., 0]), f"step {s}: flags differ"
        assert (t, dt) == tuple(r["times"][s]), f"step {s}: t/dt differ"
        assert np.array_equal(o.horizon(), r["horizon"][s]), f"step {s}: surface accounting differs"
    f1, f2 = o.fluxes()
    I = ht.interior
    assert np.array_equal(I(f1), I(r["F1"])) and np.array_equal(I(f2), I(r["F2"]))
    # force-free state: no matter, field held fixed inside the star's surface
    assert not p[..., 0:2].any()
    assert np.array_equal(p[:3, 3:-3, 5:8], r["prims"][0][:3, 3:-3, 5:8])


# the torus with the per-zone HLL/LAXF switch (FLUXADJUST FLUXBSQORHOANDU,
# build "torusfa"): n, limiter, flux, steps, (BSQORHOLIMIT, BSQOULIMIT,
# GAMMADAMP) or None for the reference's defaults.  With the defaults the
# switch picks LAXF in a few zones only over these steps; the lowered
# thresholds make it pick LAXF in 12-58% of the zones (and exercise the
# check-solution votes of the b^2 flags much more)
FLUXADJUST_LIMITS = (0.05, 0.02, 0.52)
FLUXADJUST_CASES = [(32, 4, 1, 120, FLUXADJUST_LIMITS), (32, 3, 1, 100, FLUXADJUST_LIMITS), (32, 4, 1, 400, None)]


@pytest.mark.parametrize("n,lim,flux,nsteps,limits", FLUXADJUST_CASES)
def test_oracle_matches_reference_flux_switch(n, lim, flux, nsteps, limits):
    r = ht.ref_run(n, n, lim=lim, flux=flux, nsteps=nsteps, problem="torusfa", limits=limits)
    if r is None:
        pytest.skip("reference build (oracle/_ref) with FLUXADJUST not present")
    cfg = ht.ref_config(r)
    assert cfg["fluxadjust"] == 3
    if limits is not None:
        assert (cfg["bsqorholimit"], cfg["bsqoulimit"], cfg["gammadamp"]) == limits
    o = ht.Oracle(n, n, r["geom"], lim=lim, fluxmethod=flux, **cfg)
    p = r["prims"][0].copy()
    f = r["pflag"][0].copy()
    t, dt = r["times"][0]
    nlaxf = 0
    for s in range(1, nsteps + 1):
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
        assert np.array_equal(p, r["prims"][s]), f"step {s}: primitives differ"
        # every flag, FLAGREALFLUX included, over the range get_bsqflags sets
        assert np.array_equal(f[2:-2, 2:-2], r["pflag"][s][2:-2, 2:-2]), f"step {s}: flags differ"
        assert (t, dt) == tuple(r["times"][s]), f"step {s}: t/dt differ"
        nlaxf += int((f[2:-2, 2:-2, 4] == 0).sum())
    assert nlaxf > 0, "the switch never picked LAXF"
    print(f"\nflux switch, limits {limits}: {nlaxf} zone-steps with LAXF hydro fluxes")
