#!/usr/bin/env python3
"""Generates the golden fixtures in this directory from the reference itself
(compiled from its own sources into oracle/_ref by oracle/build_ref.py).

  python tests/golden/make_golden.py

Fixtures (compressed .npz, a few hundred kB in all):
  torus16_<lim>_<flux>.npz  16x16 torus: the reference's initial state, its
      state and inversion flags after steps 1, 2, 3, 5, 10, 20 and 30, t and
      dt at those steps, and SHA-256 digests of its geometry tables (gcov, gcon,
      gdet, conn, floors) that pin the library's host-side set-up.
  cycle_break.npz  known answers of the deterministic Newton cycle-break
      factor computed by the reference build's hr_cycle_break_uniform().
"""
import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import harmtest as ht  # noqa: E402

NSTEPS = 30
KEEP = [0, 1, 2, 3, 5, 10, 20, 30]  # stored snapshots (step numbers)
CASES = [(3, 1), (4, 0), (4, 1)]  # (lim, flux): MC/HLL, PARA/LAXF, PARA/HLL


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def main():
    if ht.ref_lib_path(16, 16) is None:
        raise SystemExit("oracle/_ref/libharmref_torus_16x16.so missing: run oracle/build_ref.py first")
    names = {3: "mc", 4: "para", 0: "laxf", 1: "hll"}
    for lim, flux in CASES:
        r = ht.ref_run(16, 16, lim=lim, flux=flux, nsteps=NSTEPS)
        g = r["geom"]
        out = os.path.join(HERE, f"torus16_{names[lim]}_{names[flux]}.npz")
        np.savez_compressed(out, steps=np.array(KEEP), prims=np.stack([r["prims"][k] for k in KEEP]),
                            pflag=np.stack([r["pflag"][k] for k in KEEP])[..., 0],
                            times=np.array([r["times"][k] for k in KEEP]), scalars=r["scalars"],
                            geom_sha=np.array([digest(g[k]) for k in ("gcov", "gcon", "gdet", "conn", "floors")]))
        print(out)
    lib = ctypes.CDLL(ht.ref_lib_path(16, 16))
    lib.hr_cycle_break_uniform.restype = ctypes.c_double
    lib.hr_cycle_break_uniform.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int]
    rng = np.random.default_rng(7)
    x0 = rng.uniform(1e-8, 1e3, 64)
    x1 = rng.uniform(0, 1, 64)
    it = rng.integers(0, 200, 64)
    u = np.array([lib.hr_cycle_break_uniform(a, b, int(c)) for a, b, c in zip(x0, x1, it)])
    np.savez_compressed(os.path.join(HERE, "cycle_break.npz"), x0=x0, x1=x1, it=it, u=u)


if __name__ == "__main__":
    main()
