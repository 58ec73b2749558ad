"""The allocation-free step, harm_step_noalloc(), against harm_step().

harm_step_noalloc() serves callers that cannot call cudaMalloc -- a host code
that owns all device memory through its own pool, or one that runs where
allocation is not allowed -- by keeping the step's scratch in a static array
inside the library.  Here the caller's buffers come from torch; the entry
point is called through the C ABI twice in a row and each result must equal,
bit for bit (the tolerance of every parity test here), what the context-based
harm_step() produces from the same state.
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


def test_step_noalloc_matches_step(harm):
    import torch

    n = 32
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    h = harm.HarmGPU(n, n, geom["dx1"], geom["dx2"], lim=harm.LIM_PARA, fluxmethod=harm.FLUX_HLL)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p0, reset_gammacheck=True)
    h.bound_prims()
    h.set_time(0.0, 1e-5, 0)
    pb, fb = h.get_prims()
    expect = []
    for _ in range(2):
        h.step_ch(1)
        st = h.sync()
        p, f = h.get_prims()
        expect.append((p, f, st["t"], st["dt"]))
    h.close()

    lib = harm.load_library()
    fn = lib.harm_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p]
    cfg = harm._Config(n, n, harm.LIM_PARA, harm.FLUX_HLL, 0, 0, 0.8, par.gam, geom["dx1"], geom["dx2"], 1.3, 1.0,
                       par.gammamax, 2500.0, 20.0, 100.0, 1.0e30)
    dev = torch.device("cuda:0")
    d_geo = torch.from_numpy(_geo_planes(geom, n)).to(dev)
    d_p = torch.from_numpy(_to_planes(pb, n)).to(dev)
    d_f = torch.from_numpy(_to_planes(fb[:, :, :1].astype(np.int32), n)).to(dev)
    torch.cuda.synchronize()
    t, dt = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    n1m = n + 2 * NG
    for call in range(2):
        rc = fn(ctypes.byref(cfg), d_geo.data_ptr(), d_p.data_ptr(), d_f.data_ptr(), ctypes.byref(t), ctypes.byref(dt),
                1 if call == 0 else 0, None)
        assert rc == 0, harm.HarmError(rc, "harm_step_noalloc")
        torch.cuda.synchronize()
        p = _from_planes(d_p.cpu().numpy(), n1m)
        f = _from_planes(d_f.cpu().numpy(), n1m)[:, :, 0]
        ep, ef, et, edt = expect[call]
        assert np.array_equal(p, ep), f"call {call + 1}: primitives differ from harm_step()"
        assert np.array_equal(f[NG:-NG, NG:-NG], ef[NG:-NG, NG:-NG, 0]), f"call {call + 1}: flags differ"
        assert (t.value, dt.value) == (et, edt)


def test_step_noalloc_rejects_large_grid(harm):
    lib = harm.load_library()
    fn = lib.harm_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p]
    cfg = harm._Config(128, 128, harm.LIM_MC, harm.FLUX_HLL, 0, 0, 0.8, 4.0 / 3.0, 0.01, 0.01, 1.3, 1.0, 25.0, 2500.0,
                       20.0, 100.0, 1.0e30)
    t, dt = ctypes.c_double(0.0), ctypes.c_double(1e-5)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    assert fn(ctypes.byref(cfg), dummy, dummy, dummy, ctypes.byref(t), ctypes.byref(dt), 0, None) == 1
