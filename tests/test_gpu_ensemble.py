"""Batched form: an ensemble of uneven tori advanced by one CUDA graph launch
per step (harm_ensemble_*) gives every member exactly the state it reaches
when stepped on its own; tile shapes (set by hand or by the autotuner) do
not change results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [dict(n1=64, n2=96, a=0.3, beta=50.0, torus_rmax=11.0), dict(n1=96, n2=64, a=0.9, beta=500.0, torus_rmax=15.0),
         dict(n1=128, n2=128, a=0.0, beta=20.0, torus_rmax=13.0)]


def _members(harm, lim=4, flux=1, precision=0):
    from harm_ramt_b200 import ensemble
    return [h for h, _ in ensemble.build(harm, SPECS, lim=lim, fluxmethod=flux, precision=precision)]


@pytest.mark.parametrize("per_launch", [1, 5])
def test_ensemble_matches_members_stepped_alone(harm, per_launch):
    nsteps = 20
    ens_members = _members(harm)
    alone = _members(harm)
    e = harm.Ensemble(ens_members, steps_per_launch=per_launch)
    e.step(nsteps)
    st = e.sync()
    for h in alone:
        h.step_ch(nsteps)
    for k, (a, b) in enumerate(zip(ens_members, alone)):
        sb = b.sync()
        pa, fa = a.get_prims()
        pb, fb = b.get_prims()
        assert np.array_equal(pa, pb) and np.array_equal(fa, fb), f"member {k}"
        assert (st[k]["t"], st[k]["dt"], st[k]["realnstep"]) == (sb["t"], sb["dt"], sb["realnstep"]) == (
            sb["t"], sb["dt"], nsteps)
    e.close()


def test_tile_shapes_do_not_change_results(harm):
    h0, h1, h2 = (_members(harm)[1] for _ in range(3))
    h1.set_tiles((64, 2), (128, 2))
    h2.set_tiles((128, 1), (32, 8))
    assert h1.get_tiles() == ((64, 2), (128, 2))
    for h in (h0, h1, h2):
        h.step_ch(25)
    p0, _ = h0.get_prims()
    for h in (h1, h2):
        p, _ = h.get_prims()
        assert np.array_equal(p, p0)
    with pytest.raises(harm.HarmError):
        h0.set_tiles((256, 1), (32, 4))  # k_update takes at most 128 threads


def test_autotune_sets_a_candidate(harm):
    from harm_ramt_b200 import autotune
    h = _members(harm)[2]
    up, sm, table = autotune.tune(h, reps=1, key=("test", 128, 128))
    assert up in autotune.UPDATE_CANDIDATES and sm in autotune.SMALL_CANDIDATES
    assert h.get_tiles() == (up, sm) and len(table) == len(autotune.UPDATE_CANDIDATES) + len(autotune.SMALL_CANDIDATES)
    assert all(v > 0 for v in table.values())
