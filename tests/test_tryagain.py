"""The UTOPRIMTRYAGAIN retry chain (step_ch.c:608-626) on the CPU: each
inversion method of harm_ramt_b200/csrc/harm_tryagain.cuh compiled for the
host against the reference's own outputs on the same inputs
(tests/golden/tryagain32.npz, made by tests/golden/make_golden_tryagain.py
from the reference built with the chain on), bit for bit: the primitives
and the pflag code of 5D1, 1D, 1D_OPT, 1D_FINAL, 2D_FINAL and 5D2_FINAL,
and the whole chain after the primary 2D inversion.  The cases are the
failed inversions of the torus's first steps (which 5D1 rescues) and
perturbed states on which every method fails in some way."""
import ctypes
import os

import numpy as np
import pytest

import harmtest as ht

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "tryagain32.npz")
N = 32
GAM, GAMMAFAIL = 4.0 / 3.0, 2500.0
P = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def fix():
    return dict(np.load(FIX))


@pytest.fixture(scope="module")
def geom(harm):
    return harm.torus_geometry(harm.torus_params(N, N))


@pytest.fixture(scope="module")
def host():
    lib = ht.tryagain_host_lib()
    if lib is None:
        pytest.skip("nvcc not available")
    return lib


def _p(a):
    return a.ctypes.data_as(P)


def test_fixture_covers_every_outcome(fix):
    """the torus's own failures come first (all rescued by 5D1); the
    perturbed cases make every method fail in some way"""
    nt = int(fix["ntorus"])
    assert nt > 20 and np.all(fix["code_2"][:nt] == 101) and np.all(fix["code_0"][:nt] == 0)
    for m in (0, 3, 4, 5, 6, 7):
        assert np.any(fix[f"code_{m}"] != 0), f"method {m} never fails in the fixture"
    codes = set(np.concatenate([fix[f"code_{m}"] for m in (0, 2, 3, 4, 5, 6, 7)]).tolist())
    assert {0, 1, 2, 4, 6, 101} <= codes
    assert np.any(fix["chain_code"] == 0) and np.any(fix["chain_code"] != 0)


@pytest.mark.parametrize("method", [0, 3, 4, 5, 6, 7])
def test_method_matches_reference(fix, geom, host, method):
    bad = []
    for c, (i, j) in enumerate(fix["ij"]):
        gc, gn, gd = ht.cent_geometry(geom, int(i), int(j))
        x = fix["guess"][c].copy()
        code = host.ta_pick(method, _p(gc), _p(gn), gd, GAM, GAMMAFAIL, _p(np.ascontiguousarray(fix["U"][c])), _p(x))
        if code != fix[f"code_{method}"][c] or not np.array_equal(x, fix[f"pr_{method}"][c], equal_nan=True):
            bad.append(c)
    assert not bad, f"method {method}: {len(bad)} of {len(fix['ij'])} cases differ, first {bad[:5]}"


def test_oracle_2d_matches_reference(fix, geom):
    """the primary inversion the chain starts from (the oracle's 2D is the
    kernels' 2D bit for bit)"""
    o = ht.Oracle(N, N, geom, lim=3, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    lib = ht.oracle_lib()
    lib.ho_utoprim.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, P, P]
    for c, (i, j) in enumerate(fix["ij"]):
        x = fix["guess"][c].copy()
        code = lib.ho_utoprim(o.h, int(i), int(j), _p(np.ascontiguousarray(fix["U"][c])), _p(x))
        assert code == fix["code_2"][c] and np.array_equal(x, fix["pr_2"][c], equal_nan=True), f"case {c}"


def test_chain_matches_reference(fix, geom, host):
    bad = []
    for c, (i, j) in enumerate(fix["ij"]):
        gc, gn, gd = ht.cent_geometry(geom, int(i), int(j))
        x = fix["pr_2"][c].copy()
        code = host.ta_chain(_p(gc), _p(gn), gd, GAM, GAMMAFAIL, _p(np.ascontiguousarray(fix["U"][c])),
                             _p(np.ascontiguousarray(fix["guess"][c])), _p(x), int(fix["code_2"][c]))
        if code != fix["chain_code"][c] or not np.array_equal(x, fix["chain_pr"][c], equal_nan=True):
            bad.append(c)
    assert not bad, f"{len(bad)} chain results differ, first {bad[:5]}"


def test_fixture_is_the_reference(fix):
    """the fixture against the reference itself, where its build is present"""
    ref = ht.ref_utoprim_pick(N, N, (0, 2, 3, 4, 5, 6, 7), fix["ij"], fix["U"], fix["guess"])
    if ref is None:
        pytest.skip("reference build with the retry chain (oracle/_ref) not present")
    for m in (0, 2, 3, 4, 5, 6, 7):
        assert np.array_equal(ref[m][1], fix[f"code_{m}"]) and np.array_equal(ref[m][0], fix[f"pr_{m}"], equal_nan=True)
    assert np.array_equal(ref["chain"][1], fix["chain_code"])
    assert np.array_equal(ref["chain"][0], fix["chain_pr"], equal_nan=True)


@pytest.mark.parametrize("seed", [11, 47])
def test_methods_match_reference_on_fresh_cases(geom, host, seed):
    """the same comparison on cases drawn afresh (another seed of the fixture
    generator's perturbations), against the reference run now"""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden_tryagain as mg
    ij, U, pr, _ = mg.cases(seed=seed, nsynth=200)
    ref = ht.ref_utoprim_pick(N, N, (0, 2, 3, 4, 5, 6, 7), ij, U, pr)
    if ref is None:
        pytest.skip("reference build with the retry chain (oracle/_ref) not present")
    for m in (0, 3, 4, 5, 6, 7):
        rpr, rcode = ref[m]
        for c, (i, j) in enumerate(ij):
            gc, gn, gd = ht.cent_geometry(geom, int(i), int(j))
            x = pr[c].copy()
            code = host.ta_pick(m, _p(gc), _p(gn), gd, GAM, GAMMAFAIL, _p(np.ascontiguousarray(U[c])), _p(x))
            assert code == rcode[c] and np.array_equal(x, rpr[c], equal_nan=True), f"seed {seed} method {m} case {c}"
    rpr, rcode = ref["chain"]
    for c, (i, j) in enumerate(ij):
        gc, gn, gd = ht.cent_geometry(geom, int(i), int(j))
        x = ref[2][0][c].copy()
        code = host.ta_chain(_p(gc), _p(gn), gd, GAM, GAMMAFAIL, _p(np.ascontiguousarray(U[c])),
                             _p(np.ascontiguousarray(pr[c])), _p(x), int(ref[2][1][c]))
        assert code == rcode[c] and np.array_equal(x, rpr[c], equal_nan=True), f"seed {seed} chain case {c}"

