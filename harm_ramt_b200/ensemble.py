"""Batched ensembles of tori of uneven size.

``sample_tori`` draws the ensemble of the batched form: grids N1, N2 uniform
in {64, 96, ..., 384}, spin a ~ U[0, 0.99], minimum plasma beta
log-uniform in [10, 1000], pressure-maximum radius rmax ~ U[10, 16]; every
other parameter is the benchmark torus's.  ``build`` sets the tori up on the
host (threads: the set-up is C code that releases the interpreter lock) and
returns one context per torus; ``Ensemble`` (harm_ramt_b200) advances them
with one CUDA graph launch per step.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np

SIZES = tuple(range(64, 385, 32))


def sample_tori(n, seed=0):
    """n parameter sets (dicts of n1, n2, a, beta, torus_rmax)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(dict(n1=int(rng.choice(SIZES)), n2=int(rng.choice(SIZES)), a=float(rng.uniform(0.0, 0.99)),
                        beta=float(10.0 ** rng.uniform(1.0, 3.0)), torus_rmax=float(rng.uniform(10.0, 16.0))))
    return out


def _setup(hb, spec):
    par = hb.torus_params(spec["n1"], spec["n2"], a=spec["a"], beta=spec["beta"], torus_rmax=spec["torus_rmax"])
    geom = hb.torus_geometry(par)
    p0 = hb.torus_init(par, geom)
    return par, geom, p0


def build(hb, specs, *, lim, fluxmethod, precision=0, stream=None, threads=16, fluxadjust=0):
    """One context per spec, uploaded, bounded and at t = 0 (dt = 1e-5), with
    (params, geometry, initial prims) kept for restarting."""
    with ThreadPoolExecutor(max_workers=threads) as ex:
        made = list(ex.map(lambda s: _setup(hb, s), specs))
    members = []
    for spec, (par, geom, p0) in zip(specs, made):
        h = hb.HarmGPU(spec["n1"], spec["n2"], geom["dx1"], geom["dx2"], lim=lim, fluxmethod=fluxmethod, gam=par.gam,
                       gammamax=par.gammamax, precision=precision, stream=stream, fluxadjust=fluxadjust)
        h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
        h.set_prims(p0)
        h.bound_prims()
        h.set_time(0.0, 1.0e-5, 0)
        members.append((h, p0))
    return members


def reset(h, p0):
    """Back to the initial state of a member (after tuning or a warm-up)."""
    h.set_prims(p0)
    h.bound_prims()
    h.set_time(0.0, 1.0e-5, 0)
