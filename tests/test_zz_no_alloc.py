"""The allocation-free step, harm_step_noalloc(), against harm_step().

harm_step_noalloc() serves callers that cannot call cudaMalloc -- a host code
that owns all device memory through its own pool, or one that runs where
allocation is not allowed -- by keeping the step's scratch in a static array
inside the library.  Here the caller's buffers come from torch; the entry
point is called through the C ABI twice in a row and each result must equal,
bit for bit (the tolerance of every parity test here), what the context-based
harm_step() produces from the same state: on grids up to the array's limit,
with the retry chain of inversions, and with a call on another grid between
two calls on the same one.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NG = 3


def _sym(a, b):
    a, b = min(a, b), max(a, b)
    return [[0, 1, 2, 3], [None, 4, 5, 6], [None, None, 7, 8], [None, None, None, 9]][a][b]


def _pitch(n1):
    return ((n1 + 2 * NG + 15) // 16) * 16


def _to_planes(a, n1):
    """[n1m, n2m, k] reference layout -> [k, n2m, pitch] planes (i fastest)."""
    n1m, n2m, k = a.shape
    out = np.zeros((k, n2m, _pitch(n1)), dtype=a.dtype)
    out[:, :, :n1m] = np.transpose(a, (2, 1, 0))
    return out


def _from_planes(pl, n1m):
    return np.ascontiguousarray(np.transpose(pl[:, :, :n1m], (2, 1, 0)))


def _geo_planes(geom, n1):
    n1m, n2m = geom["gdet"].shape[:2]
    cols = []
    for loc in range(4):
        for a in range(4):
            for b in range(a, 4):
                cols.append(geom["gcov"][:, :, loc, a, b])
        for a in range(4):
            for b in range(a, 4):
                cols.append(geom["gcon"][:, :, loc, a, b])
        cols.append(geom["gdet"][:, :, loc])
    for k in range(4):
        for l in range(4):
            for j in range(l, 4):
                cols.append(geom["conn"][:, :, k, l, j])
    cols.append(geom["floors"][:, :, 0])
    cols.append(geom["floors"][:, :, 1])
    stack = np.stack(cols, axis=-1)
    assert stack.shape[-1] == 126
    return _to_planes(stack, n1)


def _fn(harm):
    lib = harm.load_library()
    fn = lib.harm_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p]
    return fn


def _torus(harm, n1, n2):
    par = harm.torus_params(n1, n2)
    geom = harm.torus_geometry(par)
    return par, geom, harm.torus_init(par, geom)


def _context_steps(harm, par, geom, p0, nsteps, tryagain, pflag0=None, t0=0.0, dt0=1e-5):
    """(prims, flags, t, dt) after each of nsteps harm_step() calls from p0"""
    n1, n2 = par.n1, par.n2
    h = harm.HarmGPU(n1, n2, geom["dx1"], geom["dx2"], lim=harm.LIM_PARA, fluxmethod=harm.FLUX_HLL,
                     tryagain=tryagain)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p0, pflag0, reset_gammacheck=True)
    if pflag0 is None:
        h.bound_prims()
    h.set_time(t0, dt0, 0)
    pb, fb = h.get_prims()
    out = []
    for _ in range(nsteps):
        h.step_ch(1)
        st = h.sync()
        p, f = h.get_prims()
        out.append((p, f, st["t"], st["dt"]))
    h.close()
    return pb, fb, out


def _noalloc_call(harm, fn, cfg, d_geo, d_p, d_f, t, dt, reset, n1):
    rc = fn(ctypes.byref(cfg), d_geo.data_ptr(), d_p.data_ptr(), d_f.data_ptr(), ctypes.byref(t), ctypes.byref(dt),
            reset, None)
    assert rc == 0, harm.HarmError(rc, "harm_step_noalloc")
    import torch
    torch.cuda.synchronize()
    p = _from_planes(d_p.cpu().numpy(), n1 + 2 * NG)
    f = _from_planes(d_f.cpu().numpy(), n1 + 2 * NG)[:, :, 0]
    return p, f


def _device_state(harm, par, geom, pb, fb):
    import torch
    dev = torch.device("cuda:0")
    n1 = par.n1
    d_geo = torch.from_numpy(_geo_planes(geom, n1)).to(dev)
    d_p = torch.from_numpy(_to_planes(pb, n1)).to(dev)
    d_f = torch.from_numpy(_to_planes(fb[:, :, :1].astype(np.int32), n1)).to(dev)
    torch.cuda.synchronize()
    return d_geo, d_p, d_f


def _cfg(harm, par, geom, tryagain):
    cfg = harm._Config(par.n1, par.n2, harm.LIM_PARA, harm.FLUX_HLL, 0, 0, 0.8, par.gam, geom["dx1"], geom["dx2"], 1.3,
                       1.0, par.gammamax, 2500.0, 20.0, 100.0, 1.0e30)
    cfg.tryagain = int(tryagain)
    return cfg


# 32 x 32; 64 x 64 (pitch 80 x 70 rows = 5600 doubles a plane) and 58 x 82
# (pitch 64 x 88 rows = 5632, exactly the limit): the planes at the end of
# the static array sit where an offset mistake would show; the retry chain
# (tryagain) on the start-up transient, where 2D inversions fail
@pytest.mark.parametrize("n1,n2,tryagain", [(32, 32, 0), (64, 64, 0), (58, 82, 0), (32, 32, 1)])
def test_step_noalloc_matches_step(harm, n1, n2, tryagain):
    par, geom, p0 = _torus(harm, n1, n2)
    pb, fb, expect = _context_steps(harm, par, geom, p0, 2, tryagain)
    fn = _fn(harm)
    cfg = _cfg(harm, par, geom, tryagain)
    d_geo, d_p, d_f = _device_state(harm, par, geom, pb, fb)
    t, dt = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    for call in range(2):
        p, f = _noalloc_call(harm, fn, cfg, d_geo, d_p, d_f, t, dt, 1 if call == 0 else 0, n1)
        ep, ef, et, edt = expect[call]
        assert np.array_equal(p, ep), f"call {call + 1}: primitives differ from harm_step()"
        assert np.array_equal(f[NG:-NG, NG:-NG], ef[NG:-NG, NG:-NG, 0]), f"call {call + 1}: flags differ"
        assert (t.value, dt.value) == (et, edt)


def test_step_noalloc_other_grid_between_calls(harm):
    """A 32 x 32 call, a 48 x 40 call, then the 32 x 32 state again without
    asking for a reset: the shared array holds the 48 x 40 call's contents,
    and the gamma table of the other grid is not carried over (the third
    call equals a context step from the same state with a fresh table)."""
    fn = _fn(harm)
    parA, geomA, p0A = _torus(harm, 32, 32)
    parB, geomB, p0B = _torus(harm, 48, 40)
    pbA, fbA, expA = _context_steps(harm, parA, geomA, p0A, 1, 0)
    pbB, fbB, expB = _context_steps(harm, parB, geomB, p0B, 1, 0)
    cfgA, cfgB = _cfg(harm, parA, geomA, 0), _cfg(harm, parB, geomB, 0)
    dA = _device_state(harm, parA, geomA, pbA, fbA)
    dB = _device_state(harm, parB, geomB, pbB, fbB)
    tA, dtA = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    tB, dtB = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    p, f = _noalloc_call(harm, fn, cfgA, *dA, tA, dtA, 1, 32)
    assert np.array_equal(p, expA[0][0])
    p, f = _noalloc_call(harm, fn, cfgB, *dB, tB, dtB, 0, 48)
    assert np.array_equal(p, expB[0][0]), "a grid change must not read the other grid's gamma table"
    # the A state after its first step, stepped by a fresh context (fresh table)
    _, _, expA2 = _context_steps(harm, parA, geomA, expA[0][0], 1, 0, pflag0=expA[0][1], t0=expA[0][2],
                                 dt0=expA[0][3])
    p, f = _noalloc_call(harm, fn, cfgA, *dA, tA, dtA, 0, 32)
    assert np.array_equal(p, expA2[0][0]) and (tA.value, dtA.value) == expA2[0][2:]


def test_step_noalloc_rejects_end_time_not_after_t(harm):
    """A zeroed tf (or any tf <= t) is refused before any device work."""
    fn = _fn(harm)
    cfg = harm._Config(32, 32, harm.LIM_MC, harm.FLUX_HLL, 0, 0, 0.8, 4.0 / 3.0, 0.01, 0.01, 1.3, 1.0, 25.0, 2500.0,
                       20.0, 100.0, 0.0)
    t, dt = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the argument checks come first
    assert fn(ctypes.byref(cfg), dummy, dummy, dummy, ctypes.byref(t), ctypes.byref(dt), 0, None) == 1


def test_step_noalloc_rejects_large_grid(harm):
    fn = _fn(harm)
    cfg = harm._Config(128, 128, harm.LIM_MC, harm.FLUX_HLL, 0, 0, 0.8, 4.0 / 3.0, 0.01, 0.01, 1.3, 1.0, 25.0, 2500.0,
                       20.0, 100.0, 1.0e30)
    t, dt = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    assert fn(ctypes.byref(cfg), dummy, dummy, dummy, ctypes.byref(t), ctypes.byref(dt), 0, None) == 1
