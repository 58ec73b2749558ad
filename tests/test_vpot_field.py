"""The torus's initial field from its vector potential (vpot2field and the
two normalisations of the reference's init) and the map's adjoint, on the
CPU: the field built from the returned A_phi reproduces the init's field
bit for bit, and <grad_A, v> = <grad, dB/dA v> for random vectors."""
import numpy as np


def test_field_from_vpot_reproduces_init(harm):
    par = harm.torus_params(48, 40)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    p1, A, norm = harm.torus_init_vpot(par, geom)
    assert np.array_equal(p0, p1)
    assert A.shape == (49, 41) and A.max() > 0 and A.min() >= 0
    assert np.array_equal(harm.vpot_to_field(par, geom, A, norm, p1), p1)


def test_vpot_adjoint_identity(harm):
    par = harm.torus_params(48, 40)
    geom = harm.torus_geometry(par)
    p1, A, norm = harm.torus_init_vpot(par, geom)
    rng = np.random.default_rng(3)
    for _ in range(4):
        g = rng.standard_normal(p1.shape)
        v = rng.standard_normal(A.shape)
        gA = harm.vpot_adjoint(par, geom, g, norm)
        z = np.zeros_like(p1)
        dB = harm.vpot_to_field(par, geom, v, norm, z)  # linear in A
        lhs, rhs = float((gA * v).sum()), float((g * dB).sum())
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)
