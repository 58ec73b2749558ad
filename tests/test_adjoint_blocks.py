"""The adjoint's building blocks (harm_ramt_b200/csrc/harm_adjoint.cuh)
against central finite differences of their forward functions, on the CPU:
states, fluxes and conserved vectors in every direction, wavespeeds, the
Lorentz-factor limit, a whole face (HLL and LAXF), the MC and PARA4
reconstruction rows, and the con-to-prim inverse-Jacobian solve.  States
are taken from the developed benchmark torus (its own metric at those
zones), perturbed in random directions."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "adjoint_blocks.cu")
LIB = os.path.join(HERE, "_build", "libadjoint_blocks.so")
HDRS = [os.path.join(HERE, "..", "harm_ramt_b200", "csrc", f) for f in ("harm_adjoint.cuh", "harm_device.cuh")]


def _lib():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    deps = [SRC] + HDRS
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run([nvcc, "-O2", "--fmad=false", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC", "-shared", "-o", LIB + ".tmp", SRC], check=True)
        os.replace(LIB + ".tmp", LIB)
    lib = ctypes.CDLL(LIB)
    d, i = ctypes.c_double, ctypes.c_int
    P = ctypes.POINTER(ctypes.c_double)
    lib.ab_check.restype = d
    lib.ab_check.argtypes = [i, P, P, P, P, P, d, i, d, d, d]
    lib.ab_check_face.restype = d
    lib.ab_check_face.argtypes = [P, P, P, P, P, P, P, d, i, d, d, i, d]
    lib.ab_check_recon.restype = d
    lib.ab_check_recon.argtypes = [i, P, P, d, d, d]
    lib.ab_check_source.restype = d
    lib.ab_check_source.argtypes = [P, P, P, P, P, d, P, d, d]
    lib.ab_check_ift.restype = d
    lib.ab_check_ift.argtypes = [P, P, P, P, P, d, d, d]
    lib.ab_probe_host.argtypes = [i, i, P, P, P, P, P, d, d, P, P]
    lib.ab_probe_device.restype = i
    lib.ab_probe_device.argtypes = [i, i, P, P, P, P, P, d, d, P, P]
    return lib


def _p(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.fixture(scope="module")
def torus_zones(harm):
    """Developed-torus states with their metric, from the oracle (CPU)."""
    import harmtest as ht
    n = 64
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    p = o.bound(p0)
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    t, dt = 0.0, 1e-5
    for _ in range(60):
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
    rng = np.random.default_rng(3)
    zones = [(int(rng.integers(3, n + 3)), int(rng.integers(3, n + 3))) for _ in range(24)]
    return p, geom, zones


def _zone(p, geom, i, j, loc=3):
    return p[i, j].copy(), geom["gcov"][i, j, loc].copy(), geom["gcon"][i, j, loc].copy(), geom["gdet"][i, j, loc]


# finite-difference steps: each check takes the best of these (truncation
# error grows with h, round-off as 1/h); a wrong derivative fails at all
HS = (1e-5, 1e-6, 1e-7)
TOL = 1e-6


@pytest.mark.parametrize("which,dirs", [(0, (0, 1, 2)), (1, (1, 2))])
def test_state_flux_and_wavespeed_adjoints(torus_zones, which, dirs):
    lib = _lib()
    p, geom, zones = torus_zones
    rng = np.random.default_rng(11 + which)
    worst = 0.0
    for (i, j) in zones:
        for d in dirs:
            pz, gc, gn, gd = _zone(p, geom, i, j)
            v = rng.standard_normal(8) * np.abs(pz) + 1e-3 * rng.standard_normal(8) * np.abs(pz).max()
            lam = rng.standard_normal(8)
            args = [_p(x) for x in (pz, v, lam, gc, gn)]
            err = min(lib.ab_check(which, args[0][1], args[1][1], args[2][1], args[3][1], args[4][1], gd, d,
                                   4.0 / 3.0, 0.0, h) for h in HS)
            assert err >= 0.0
            worst = max(worst, err)
    assert worst < TOL, worst


def test_limit_gamma_adjoint(torus_zones):
    lib = _lib()
    p, geom, zones = torus_zones
    rng = np.random.default_rng(5)
    for (i, j) in zones[:8]:
        pz, gc, gn, gd = _zone(p, geom, i, j)
        pz[2:5] *= 30.0  # fast enough that the limit is active at gammamax 5
        for gmax in (5.0, 1e6):
            v = rng.standard_normal(8) * np.abs(pz)
            lam = rng.standard_normal(8)
            args = [_p(x) for x in (pz, v, lam, gc, gn)]
            err = min(lib.ab_check(2, args[0][1], args[1][1], args[2][1], args[3][1], args[4][1], gd, 1, 4.0 / 3.0,
                                   gmax, h) for h in HS)
            assert err < TOL, (gmax, err)


@pytest.mark.parametrize("fluxmethod", [0, 1])
def test_face_flux_adjoint(torus_zones, fluxmethod):
    lib = _lib()
    p, geom, zones = torus_zones
    rng = np.random.default_rng(7 + fluxmethod)
    worst = 0.0
    for (i, j) in zones:
        for d in (1, 2):
            loc = 0 if d == 1 else 1
            pl = p[i - (d == 1), j - (d == 2)].copy()
            pr = p[i, j].copy()
            gc, gn, gd = geom["gcov"][i, j, loc], geom["gcon"][i, j, loc], geom["gdet"][i, j, loc]
            vl = rng.standard_normal(8) * np.abs(pl)
            vr = rng.standard_normal(8) * np.abs(pr)
            lam = rng.standard_normal(8)
            a = [_p(x) for x in (pl, pr, vl, vr, lam, gc, gn)]
            err = min(lib.ab_check_face(a[0][1], a[1][1], a[2][1], a[3][1], a[4][1], a[5][1], a[6][1], gd, d,
                                        4.0 / 3.0, 25.0, fluxmethod, h) for h in HS)
            assert err >= 0.0
            worst = max(worst, err)
    assert worst < TOL, worst


@pytest.mark.parametrize("para", [0, 1])
def test_reconstruction_rows(para):
    lib = _lib()
    rng = np.random.default_rng(13 + para)
    worst = 0.0
    for _ in range(400):
        y = rng.standard_normal(5).cumsum() * rng.uniform(0.1, 2.0)
        v = rng.standard_normal(5)
        a = [_p(x) for x in (y, v)]
        ll, lr = rng.standard_normal(), rng.standard_normal()
        err = min(lib.ab_check_recon(para, a[0][1], a[1][1], ll, lr, h) for h in HS)
        worst = max(worst, err)
    assert worst < 1e-6, worst


def test_geometric_source_adjoint(torus_zones):
    lib = _lib()
    p, geom, zones = torus_zones
    rng = np.random.default_rng(19)
    worst = 0.0
    for (i, j) in zones + [(3, 5), (3, 30), (4, 3), (40, 3)]:
        pz, gc, gn, gd = _zone(p, geom, i, j)
        conn = geom["conn"][i, j].copy()
        v = rng.standard_normal(8) * np.abs(pz)
        lam = rng.standard_normal(4)
        a = [_p(x) for x in (pz, v, lam, gc, gn, conn)]
        err = min(lib.ab_check_source(a[0][1], a[1][1], a[2][1], a[3][1], a[4][1], gd, a[5][1], 4.0 / 3.0, h)
                  for h in HS)
        worst = max(worst, err)
    assert worst < TOL, worst


def test_inverse_jacobian_solve(torus_zones):
    lib = _lib()
    p, geom, zones = torus_zones
    rng = np.random.default_rng(17)
    worst = 0.0
    for (i, j) in zones:
        pz, gc, gn, gd = _zone(p, geom, i, j)
        v = rng.standard_normal(8) * np.abs(pz)
        b = rng.standard_normal(8)
        a = [_p(x) for x in (pz, v, b, gc, gn)]
        err = min(lib.ab_check_ift(a[0][1], a[1][1], a[2][1], a[3][1], a[4][1], gd, 4.0 / 3.0, h) for h in HS)
        assert err >= 0.0
        worst = max(worst, err)
    assert worst < TOL, worst
