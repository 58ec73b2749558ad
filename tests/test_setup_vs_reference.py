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
