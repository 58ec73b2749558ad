"""The UTOPRIMTRYAGAIN retry chain on the GPU: each inversion method and the
whole Utoprimgen through harm_invert_zones against the reference's outputs
(tests/golden/tryagain32.npz), and full steps of the 32^2 torus with the
chain on (harm_config.tryagain = 1) against the reference built with the
chain on (UTOPRIMTRYAGAIN 1), bit for bit."""
import os

import numpy as np
import pytest

import harmtest as ht

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "tryagain32.npz")
N = 32
I = ht.interior


@pytest.fixture(scope="module")
def fix():
    return dict(np.load(FIX))


@pytest.fixture(scope="module")
def ctx(harm):
    par = harm.torus_params(N, N)
    geom = harm.torus_geometry(par)
    h = harm.HarmGPU(N, N, geom["dx1"], geom["dx2"], lim=harm.LIM_MC, fluxmethod=harm.FLUX_HLL, tryagain=True)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    yield h
    h.close()


@pytest.mark.parametrize("method", [0, 2, 3, 4, 5, 6, 7])
def test_device_method_matches_reference(fix, ctx, method):
    pr, code = ctx.invert_zones(method, fix["ij"], fix["U"], fix["guess"])
    bad = np.flatnonzero((code != fix[f"code_{method}"]) |
                         ~np.all((pr == fix[f"pr_{method}"]) | (np.isnan(pr) & np.isnan(fix[f"pr_{method}"])), axis=1))
    assert bad.size == 0, f"method {method}: {bad.size} of {len(code)} cases differ, first {bad[:5].tolist()}"


def test_device_chain_matches_reference(fix, ctx, harm):
    pr, code = ctx.invert_zones(harm.INV_CHAIN, fix["ij"], fix["U"], fix["guess"])
    bad = np.flatnonzero((code != fix["chain_code"]) |
                         ~np.all((pr == fix["chain_pr"]) | (np.isnan(pr) & np.isnan(fix["chain_pr"])), axis=1))
    assert bad.size == 0, f"{bad.size} chain results differ, first {bad[:5].tolist()}"


def test_steps_match_reference_with_chain(harm):
    """25 steps of the 32^2 torus from init (MC + HLL), the chain rescuing the
    inversions the start-up transient fails, against the reference built
    with UTOPRIMTRYAGAIN 1; the same steps without the chain differ."""
    r = ht.ref_run(32, 32, lim=3, flux=1, nsteps=25, problem="torusta")
    if r is None:
        pytest.skip("reference build with the retry chain (oracle/_ref) not present")
    cfg = ht.ref_config(r)
    geom = r["geom"]

    def ctx_from(tryagain):
        h = harm.HarmGPU(32, 32, cfg["dx1"], cfg["dx2"], lim=3, fluxmethod=1, tryagain=tryagain,
                         **{k: v for k, v in cfg.items() if k not in ("dx1", "dx2")})
        h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
        h.set_prims(r["prims"][0], r["pflag"][0])
        h.set_time(r["times"][0][0], r["times"][0][1], 0)
        return h

    h, h0 = ctx_from(True), ctx_from(False)
    differs = False
    for s in range(1, 26):
        h.step_ch(1)
        h0.step_ch(1)
        st = h.sync()
        h0.sync()
        pg, fg = h.get_prims()
        p0, _ = h0.get_prims()
        assert np.array_equal(I(pg), I(r["prims"][s])), f"step {s}: primitives differ from the reference"
        assert np.array_equal(I(fg)[..., 0], I(r["pflag"][s])[..., 0]), f"step {s}: inversion flags differ"
        assert (st["t"], st["dt"]) == tuple(r["times"][s])
        differs |= not np.array_equal(I(pg), I(p0))
    h.close()
    h0.close()
    assert differs, "the chain changed nothing: the test does not exercise it"
