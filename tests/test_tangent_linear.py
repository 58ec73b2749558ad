"""The tangent-linear form of the oracle (oracle/harm_oracle_tl.cpp: the same
C restatement compiled with a dual-number type), the reference gradient the
adjoint kernels are checked against on the GPU (tests/test_gpu_adjoint_tl.py).

Its values are the oracle's own, bit for bit, and its tangents agree with
central differences of the oracle's objective along seeded directions."""
import numpy as np
import pytest

import harmtest as ht

EPS = (1e-6, 1e-7, 1e-8)


def _state(n, nsteps):
    import harm_ramt_b200 as hb
    par = hb.torus_params(n, n)
    geom = hb.torus_geometry(par)
    p0 = hb.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    p = o.bound(p0)
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    t, dt = 0.0, 1e-5
    for _ in range(nsteps):
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
    # off the exact ties of the floored atmosphere (see tests/test_gpu_adjoint.py)
    p = p * (1.0 + 1e-4 * np.random.default_rng(7).standard_normal(p.shape))
    return geom, p, dt


def _objective(o, geom, p0, dts):
    p = o.bound(p0)
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    J, t = 0.0, 0.0
    for dt in dts:
        d = float(dt)
        rc, _, _ = o.step(p, f, t, d)
        assert rc == 0
        t += d
        hz = o.horizon()
        J += d * (hz[0] + (hz[2] + hz[3]))
    return J, p


def test_tangent_linear_values_equal_the_oracle():
    n = 32
    geom, p, dt = _state(n, 30)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    tl = ht.OracleTL(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    dts = [dt * (1.0 + 0.01 * k) for k in range(8)]
    v = np.random.default_rng(3).standard_normal(p.shape) * np.abs(p)
    v[:3] = v[-3:] = 0.0
    v[:, :3] = v[:, -3:] = 0.0
    J, dJ, pt, _ = tl.objective(p, v, dts)
    Jo, po = _objective(o, geom, p, dts)
    assert np.array_equal(pt, po), "the dual-number run's values differ from the oracle's"
    assert J == Jo and dJ != 0.0


def test_tangent_linear_matches_finite_differences():
    n = 32
    geom, p, dt = _state(n, 30)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    tl = ht.OracleTL(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    dts = [dt] * 6
    rng = np.random.default_rng(11)
    worst = 0.0
    for d in range(4):
        v = rng.standard_normal(p.shape) * np.abs(p)
        v[:3] = v[-3:] = 0.0
        v[:, :3] = v[:, -3:] = 0.0
        J0, dJ, _, _ = tl.objective(p, v, dts)
        best = None
        for eps in EPS:
            Jp, _ = _objective(o, geom, p + eps * v, dts)
            Jm, _ = _objective(o, geom, p - eps * v, dts)
            c, f, b = (Jp - Jm) / (2 * eps), (Jp - J0) / eps, (J0 - Jm) / eps
            spread = abs(f - b) / max(abs(c), 1e-300)
            if best is None or spread < best[1]:
                best = (c, spread)
        err = abs(best[0] - dJ) / max(abs(dJ), 1e-300)
        worst = max(worst, err)
    print(f"tangent-linear vs finite differences, 6 steps of the 32^2 torus: worst relative difference {worst:.2e}")
    assert worst < 1e-5, worst
