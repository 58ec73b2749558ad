"""Fatal checks of the device step, made by uploading a state with corrupted
zones (the failure is made on the host; nothing faults on the device).

The step must return HARM_EFAIL through harm_sync with the fail() code and
zone that the oracle and the reference report for the same state
(tests/test_failures.py pins those): the device keeps the first report in
the reference's order, so the answer does not depend on which thread got
there first.  Repeated runs give the same answer, and the context steps on
normally once a good state is uploaded again.
"""
import numpy as np
import pytest

from test_failures import FAIL_CASES, corrupted_torus

pytestmark = pytest.mark.gpu


def _ctx(harm, geom, n, lim=3, flux=1):
    h = harm.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=lim, fluxmethod=flux)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    return h


@pytest.mark.parametrize("zones,expect", FAIL_CASES)
def test_gpu_reports_the_references_fail_code_and_zone(harm, zones, expect):
    n = 32
    geom, p, o = corrupted_torus(n, zones)
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    rc, _, _ = o.step(p.copy(), f, 0.0, 1e-5)
    assert o.fail() == expect
    h = _ctx(harm, geom, n)
    for rep in range(3):
        h.set_prims(p)
        h.set_time(0.0, 1e-5, 0)
        h.step_ch(1)
        with pytest.raises(harm.HarmError) as e:
            h.sync()
        assert e.value.code == 6  # HARM_EFAIL
        st = h.sync(raise_on_fail=False)
        assert (st["fail_code"], st["fail_i"], st["fail_j"]) == expect, (rep, st)
        assert st["fail_step"] == 0
    h.close()


def test_gpu_context_usable_after_failure(harm):
    n = 32
    geom, bad, o = corrupted_torus(n, [(12, 14)])
    _, good, _ = corrupted_torus(n, [])
    h = _ctx(harm, geom, n)
    h.set_prims(bad)
    h.set_time(0.0, 1e-5, 0)
    h.step_ch(1)
    assert h.sync(raise_on_fail=False)["fail_code"] == 5
    h.set_prims(good)
    h.set_time(0.0, 1e-5, 0)
    h.step_ch(3)
    st = h.sync()
    assert st["fail_code"] == 0 and st["realnstep"] == 3 and st["fail_step"] == -1
    po = good.copy()
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    t, dt = 0.0, 1e-5
    for _ in range(3):
        rc, t, dt = o.step(po, fo, t, dt)
        assert rc == 0
    pg, _ = h.get_prims()
    assert np.array_equal(pg, po)
    h.close()


def test_gpu_failure_in_a_later_step_names_that_step(harm):
    """The corrupted zone is uploaded after two good steps: the report names
    the third step (realnstep 2 at its start)."""
    n = 32
    geom, good, o = corrupted_torus(n, [])
    h = _ctx(harm, geom, n)
    h.set_prims(good)
    h.set_time(0.0, 1e-5, 0)
    h.step_ch(2)
    st = h.sync()
    p, f = h.get_prims()
    p[12 + 3, 14 + 3, 0] = -1.2 * p[12 + 3, 14 + 3, 1]
    h.set_prims(p, f, reset_gammacheck=False)
    h.step_ch(1)
    st = h.sync(raise_on_fail=False)
    assert (st["fail_code"], st["fail_i"], st["fail_j"], st["fail_step"]) == (5, 12, 14, 2), st
    h.close()
