"""Generates tests/golden/tryagain32.npz: inputs and the reference's own
outputs for the UTOPRIMTRYAGAIN retry chain (step_ch.c:608-626) on the 32^2
torus (MC + HLL).

Cases: (1) every inversion the torus's own first 5 steps from init fail
(2D code 101), recorded by the oracle with their U and guess; (2) seeded
perturbations of developed states (step 40): U's internal energy moved by up
to 150%, momentum scaled up to 30x, guesses with velocities scaled by 3e3
or 1e5, densities scaled down to 1% or made negative, so that every method
fails in some of them.  Outputs: each method of Utoprimgen_pick (5D1, 2D,
1D, 1D_OPT, 1D_FINAL, 2D_FINAL, 5D2_FINAL) and the whole Utoprimgen of the
reference built with the chain on (oracle/build_ref.py --problem torusta).

Run from the repository root after building that reference:
    python oracle/build_ref.py --problem torusta --sizes 32x32
    python tests/golden/make_golden_tryagain.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, ".."))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
import harmtest as ht  # noqa: E402
import harm_ramt_b200 as hb  # noqa: E402

N = 32
METHODS = (0, 2, 3, 4, 5, 6, 7)
OUT = os.path.join(HERE, "tryagain32.npz")


def cases(seed=20261203, nsynth=240):
    par = hb.torus_params(N, N)
    geom = hb.torus_geometry(par)
    p0 = hb.torus_init(par, geom)
    o = ht.Oracle(N, N, geom, lim=hb.LIM_MC, fluxmethod=hb.FLUX_HLL, dx1=geom["dx1"], dx2=geom["dx2"])
    o.record_failures(1000)
    po = o.bound(p0)
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    t, dt = 0.0, 1e-5
    for _ in range(5):
        rc, t, dt = o.step(po, fo, t, dt)
        assert rc == 0
    ij0, U0, pr0 = o.failures()
    for _ in range(35):
        rc, t, dt = o.step(po, fo, t, dt)
        assert rc == 0
    lib = ht.tryagain_host_lib()
    P = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(seed)
    ij, U, pr = [], [], []
    for c in range(nsynth):
        i, j = int(rng.integers(0, N)), int(rng.integers(0, N))
        p = po[i + ht.NG, j + ht.NG].copy()
        gc, gn, gd = ht.cent_geometry(geom, i, j)
        Uev = np.zeros(8)
        lib.ta_primtoU(gc.ctypes.data_as(P), gn.ctypes.data_as(P), gd, par.gam, p.ctypes.data_as(P),
                       Uev.ctypes.data_as(P))
        guess = p * (1 + 0.05 * rng.standard_normal(8))
        kind = c % 5
        if kind == 1:
            Uev[1] = Uev[0] + (Uev[1] - Uev[0]) * (1 + rng.uniform(-1.5, 1.5))
        elif kind == 2:
            Uev[2:5] *= rng.uniform(1.5, 30.0)
        elif kind == 3:
            guess[2:5] *= (1e5 if c % 2 else 3e3)
        elif kind == 4:
            Uev[0] *= (rng.uniform(0.01, 3.0) if c % 3 else -rng.uniform(0.1, 2.0))
        ij.append((i, j))
        U.append(Uev)
        pr.append(guess)
    ij = np.concatenate([ij0, np.array(ij, dtype=np.int32)])
    U = np.concatenate([U0, np.array(U)])
    pr = np.concatenate([pr0, np.array(pr)])
    return ij, U, pr, len(ij0)


def main():
    ij, U, pr, ntorus = cases()
    ref = ht.ref_utoprim_pick(N, N, METHODS, ij, U, pr)
    if ref is None:
        raise SystemExit("reference build oracle/_ref/libharmref_torusta_32x32.so not found")
    out = dict(ij=ij, U=U, guess=pr, ntorus=ntorus, chain_pr=ref["chain"][0], chain_code=ref["chain"][1])
    for m in METHODS:
        out[f"pr_{m}"] = ref[m][0]
        out[f"code_{m}"] = ref[m][1]
    np.savez_compressed(OUT, **out)
    print(OUT, len(ij), "cases;", "chain codes", dict(zip(*np.unique(ref["chain"][1], return_counts=True))))


if __name__ == "__main__":
    main()
