"""Force-free electrodynamics (the phys.ffde.c variant of the step) on the
GPU: the aligned rotator (dipole field, stellar surface rotating at
omegastar, bounds.ns.c) in flat space, spherical polar log-r coordinates.

FP64 is compared bit for bit with the reference compiled from its own sources
(geometry and initial state from its init()) and with the oracle over longer
runs; the mixed form (FP32 face fluxes) is compared with FP64 under the
tolerances written here."""
import numpy as np
import pytest

import harmtest as ht

pytestmark = pytest.mark.gpu


def _gpu(harm, r, lim, flux, precision=0, currents=False):
    n1, n2 = r["n1"], r["n2"]
    cfg = ht.ref_config(r)
    h = harm.HarmGPU(n1, n2, cfg.pop("dx1"), cfg.pop("dx2"), lim=lim, fluxmethod=flux, eom=harm.EOM_FFDE,
                     bc=harm.BC_STAR, omegastar=r["omegastar"], precision=precision, currents=currents, **cfg)
    g = r["geom"]
    h.upload_geometry(g["gcov"], g["gcon"], g["gdet"], g["conn"], g["floors"])
    h.set_prims(r["prims"][0], r["pflag"][0])
    h.set_time(r["times"][0][0], r["times"][0][1], 0)
    return h


def _ref(n1, n2, lim, flux, nsteps):
    r = ht.ref_run(n1, n2, lim=lim, flux=flux, nsteps=nsteps, problem="dipole")
    if r is None:
        pytest.skip("reference build (oracle/_ref) of the dipole problem not present")
    return r


@pytest.mark.parametrize("lim,flux,nsteps", [(3, 0, 60), (4, 1, 40)])
def test_ffde_gpu_matches_reference_dipole(harm, lim, flux, nsteps):
    r = _ref(32, 16, lim, flux, nsteps)
    h = _gpu(harm, r, lim, flux, currents=True)
    for s in range(1, nsteps + 1):
        h.step_ch(1)
        st = h.sync()
        pg, fg = h.get_prims()
        assert np.array_equal(pg, r["prims"][s]), f"step {s}: {np.count_nonzero(pg != r['prims'][s])} values differ"
        assert np.array_equal(fg[..., 0], r["pflag"][s][..., 0])
        assert (st["t"], st["dt"]) == tuple(r["times"][s])
        assert list(h.get_horizon().values()) == list(r["horizon"][s]), f"step {s}: surface accounting"
        assert all(np.array_equal(x, y) for x, y in zip(h.get_currents(), r["currents"][s])), f"step {s}: currents"
    f1g, f2g = h.get_fluxes()
    I = ht.interior
    assert np.array_equal(I(f1g), I(r["F1"])) and np.array_equal(I(f2g), I(r["F2"]))
    h.close()


def test_ffde_gpu_matches_oracle_dipole_long(harm):
    n1, n2, lim, flux, nsteps = 64, 32, 3, 0, 600
    r = _ref(n1, n2, lim, flux, 0)
    o = ht.Oracle(n1, n2, r["geom"], lim=lim, fluxmethod=flux, eom=1, bc=1, omegastar=r["omegastar"],
                  **ht.ref_config(r))
    p = r["prims"][0].copy()
    f = r["pflag"][0].copy()
    t, dt = r["times"][0]
    h = _gpu(harm, r, lim, flux)
    for s in range(nsteps):
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
    h.step_ch(nsteps)
    st = h.sync()
    pg, fg = h.get_prims()
    assert np.array_equal(pg, p), f"{np.count_nonzero(pg != p)} values differ after {nsteps} steps"
    assert (st["t"], st["dt"]) == (t, dt) and st["realnstep"] == nsteps
    assert list(h.get_horizon().values()) == list(o.horizon())
    h.close()


# mixed (FP32 face fluxes) against FP64 on the 64 x 32 rotator at t = 5
TOL_MIXED = {"B": 1e-4, "u": 1e-3, "spindown_integrated": 1e-4}


def test_ffde_mixed_precision_vs_fp64(harm):
    n1, n2, lim, flux, tf = 64, 32, 3, 0, 5.0
    r = _ref(n1, n2, lim, flux, 0)
    out = {}
    for prec in (harm.PREC_FP64, harm.PREC_MIXED):
        h = _gpu(harm, r, lim, flux, precision=prec)
        st = h.run_to(tf)
        p, _ = h.get_prims()
        out[prec] = (p[3:-3, 3:-3], h.get_horizon(), st)
        h.close()
    pd, hd, sd = out[harm.PREC_FP64]
    pm, hm, sm = out[harm.PREC_MIXED]
    assert sd["t"] == sm["t"] == tf
    l1 = lambda a, b: float(np.abs(a - b).sum() / np.abs(b).sum())
    gc = r["geom"]["gcov"][3:-3, 3:-3, 3, 1:4, 1:4]  # CENT spatial metric

    def capped(p):
        # drift Lorentz factor at the cap GAMMAMAX: zones where B^2 - E^2 > 0
        # had to be enforced (AVOIDUTINF 2, phys.ffde.c:230-236)
        u = p[..., 2:5]
        gamma = np.sqrt(1.0 + np.einsum("...i,...ij,...j->...", u, gc, u))
        return float((gamma > 25.0 * (1 - 1e-9)).mean())

    err = {"B": l1(pm[..., 5:8], pd[..., 5:8]), "u": l1(pm[..., 2:5], pd[..., 2:5]),
           "spindown_integrated": abs(hm["pcum_uu"] - hd["pcum_uu"]) / abs(hd["pcum_uu"])}
    print("ffde mixed vs fp64 at t=%g:" % tf, err, "zones at the gamma cap: fp64 %.4f mixed %.4f"
          % (capped(pd), capped(pm)))
    for k, v in err.items():
        assert v < TOL_MIXED[k], (k, v)
    assert not pm[..., 0:2].any() and not pd[..., 0:2].any()
    assert np.isfinite(pm).all() and not np.array_equal(pm, pd)


@pytest.mark.parametrize("n1,n2,nsteps", [(32, 16, 30), (512, 256, 2)])
def test_ffde_host_setup_runs_as_reference(harm, n1, n2, nsteps):
    """The dipole built by the library's own set-up (harm_dipole_geometry,
    harm_dipole_init; no reference code in the loop) and bounded on the
    device equals the reference's init in every zone, ghosts included, and
    steps exactly as the reference does (MC + LAXF)."""
    r = _ref(n1, n2, 3, 0, nsteps)
    h, _, _ = harm.dipole_context(n1, n2, lim=3, fluxmethod=0, omegastar=float(r["omegastar"]))
    pg, _ = h.get_prims()
    assert np.array_equal(pg, r["prims"][0]), f"{np.count_nonzero(pg != r['prims'][0])} values differ after the bound"
    for s in range(1, nsteps + 1):
        h.step_ch(1)
        st = h.sync()
        pg, _ = h.get_prims()
        assert np.array_equal(pg, r["prims"][s]), f"step {s}: {np.count_nonzero(pg != r['prims'][s])} values differ"
        assert (st["t"], st["dt"]) == tuple(r["times"][s])
    h.close()
