"""Mixed-precision form (FP32 reconstruction/wavespeeds/face fluxes, FP64
inversion, update, source, EMF, dt) against the FP64 path from the same
initial torus: relative L1 errors in rho, u, B and the time-integrated
horizon mass flux, with the tolerances written here."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"rho": 1e-4, "u": 1e-4, "B": 1e-3, "mdot": 1e-4}


def _run(harm, n, precision, tf):
    h, geom, p0 = harm.torus_context(n, n, lim=harm.LIM_PARA, fluxmethod=harm.FLUX_HLL, precision=precision, tf=tf)
    st = h.run_to(tf)
    p, f = h.get_prims()
    hz = h.get_horizon()
    h.close()
    return p, hz, st


def l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def test_mixed_precision_error_vs_fp64(harm):
    n, tf = 64, 20.0
    pd, hzd, std = _run(harm, n, harm.PREC_FP64, tf)
    pm, hzm, stm = _run(harm, n, harm.PREC_MIXED, tf)
    assert std["t"] == tf and stm["t"] == tf
    I = (slice(3, -3), slice(3, -3))
    err = {"rho": l1(pm[I][..., 0], pd[I][..., 0]), "u": l1(pm[I][..., 1], pd[I][..., 1]),
           "B": l1(pm[I][..., 5:8], pd[I][..., 5:8]),
           "mdot": abs(hzm["pcum_rho"] - hzd["pcum_rho"]) / abs(hzd["pcum_rho"])}
    print("mixed vs fp64 at t=%g:" % tf, err)
    for k, v in err.items():
        assert v < TOL[k], (k, v)
    assert not np.array_equal(pm, pd)  # the FP32 faces are really in use
