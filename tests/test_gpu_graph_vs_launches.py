"""The graph-launched step against the same step launched kernel by kernel
(harm_profile_step), bit for bit, from the torus's initial state through its
start-up transient, where fixup_checksolution flags zones next to later
candidates so that its parallel sweep needs more than one round (counted in
harm_status.chk_multi; the runs here must contain such sweeps)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(harm, n, lim, flux):
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    hs = []
    for _ in range(2):
        h = harm.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=lim, fluxmethod=flux, gam=par.gam,
                         gammamax=par.gammamax)
        h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
        h.set_prims(p0)
        h.bound_prims()
        h.set_time(0.0, 1.0e-5, 0)
        hs.append(h)
    return hs


@pytest.mark.parametrize("n,lim,flux,nsteps", [(64, 4, 1, 300), (128, 3, 1, 200)])
def test_graph_step_matches_unconditional_launches(harm, n, lim, flux, nsteps):
    hg, hp = _pair(harm, n, lim, flux)
    for s in range(1, nsteps + 1):
        hg.step_ch(1)
        hp.profile_step()
        if s % 10 == 0 or s == nsteps:
            sg, sp = hg.sync(), hp.sync()
            pg, fg = hg.get_prims()
            pp, fp = hp.get_prims()
            assert np.array_equal(pg, pp) and np.array_equal(fg, fp), f"{n}^2 step {s}: graph and launches differ"
            assert (sg["t"], sg["dt"], sg["chk_multi"]) == (sp["t"], sp["dt"], sp["chk_multi"])
    print(f"{n}^2: {sg['chk_multi']} substeps ran more than one check-solution round")
    TEST_COUNTS[(n, lim)] = sg["chk_multi"]
    hg.close()
    hp.close()


TEST_COUNTS = {}


def test_multi_round_sweeps_were_exercised():
    if len(TEST_COUNTS) < 2:
        pytest.skip("the comparison runs did not complete")
    assert sum(TEST_COUNTS.values()) > 0, f"no multi-round sweep in the runs: {TEST_COUNTS}"
