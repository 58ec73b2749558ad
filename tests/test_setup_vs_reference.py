"""Host-side set-up (geometry and torus init) against the reference's own
set_grid()/init() at several sizes (skipped without the reference build)."""
import numpy as np
import pytest

import harmtest as ht


@pytest.mark.parametrize("n", [32, 64])
def test_setup_matches_reference(harm, n):
    r = ht.ref_run(n, n, nsteps=0)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    g = harm.torus_geometry(harm.torus_params(n, n))
    for k in ("gcov", "gcon", "gdet", "conn", "floors"):
        assert np.array_equal(g[k], r["geom"][k]), k
    s = r["scalars"]
    assert (g["dx1"], g["dx2"], g["startx1"]) == (s[10], s[11], s[8])
    p = harm.torus_init(harm.torus_params(n, n), g)
    I = ht.interior
    assert np.array_equal(I(p)[..., :7], I(r["prims"][0])[..., :7])


def test_torus_dump_coords_match_reference(harm):
    r = ht.ref_run(32, 32, lim=3, flux=1, nsteps=0, dump=True)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    hdr, co = harm.torus_dump_coords(harm.torus_params(32, 32))
    assert np.array_equal(co, r["coords"])
    s = r["scalars"]
    ref = dict(startx1=s[8], startx2=s[9], a=s[2], R0=s[7], Rin=s[4], Rout=s[5], hslope=s[6], defcoord=r["defcoord"])
    assert all(hdr[k] == ref[k] for k in ref), (hdr, ref)


@pytest.mark.parametrize("n1,n2", [(32, 16), (64, 32)])
def test_dipole_setup_matches_reference(harm, n1, n2):
    """The force-free aligned rotator: the defcoord 6 flat-space tables, and
    the init (dipole potential, vpot2field, filterffde twice, fixup) on the
    active zones and on the star's inner ghost zones, whose field the
    surface boundary holds (it sets only their velocity)."""
    r = ht.ref_run(n1, n2, lim=3, flux=0, nsteps=0, problem="dipole")
    if r is None:
        pytest.skip("reference build (oracle/_ref) of the dipole problem not present")
    par = harm.dipole_params(n1, n2, omegastar=float(r["omegastar"]))
    g = harm.dipole_geometry(par)
    for k in ("gcov", "gcon", "gdet", "conn", "floors"):
        assert np.array_equal(g[k], r["geom"][k]), k
    s = r["scalars"]
    assert (g["dx1"], g["dx2"], g["startx1"]) == (s[10], s[11], s[8])
    cfg = ht.ref_config(r)
    assert (par.gam, par.gammamax) == (cfg["gam"], cfg["gammamax"])
    p = harm.dipole_init(par, g)
    ref = r["prims"][0]
    I = ht.interior
    assert np.array_equal(I(p), I(ref))
    inner = (slice(0, 3), slice(3, n2 + 3))
    for k in (0, 1, 2, 3, 5, 6, 7):
        assert np.array_equal(p[inner][..., k], ref[inner][..., k]), k
