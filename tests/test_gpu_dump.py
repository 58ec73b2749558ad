"""Dump files: the text dump written from the device state
(harm_write_dump) is byte-for-byte the file the reference's own dump()
(dump.c:24-191) writes for the same state: header line, 56 columns per
zone, currents included."""
import os
import tempfile

import numpy as np
import pytest

import harmtest as ht

pytestmark = pytest.mark.gpu


def _header(r):
    s = r["scalars"]
    return dict(startx1=s[8], startx2=s[9], a=s[2], R0=s[7], Rin=s[4], Rout=s[5], hslope=s[6],
                defcoord=r["defcoord"])


def _dump_bytes(h, header, coords):
    fd, path = tempfile.mkstemp(prefix="harm_dump_")
    os.close(fd)
    try:
        h.write_dump(path, header, coords)
        with open(path, "rb") as f:
            return f.read()
    finally:
        os.unlink(path)


def _first_difference(a, b):
    la, lb = a.split(b"\n"), b.split(b"\n")
    for k, (x, y) in enumerate(zip(la, lb)):
        if x != y:
            return k, x[:200], y[:200]
    return len(la), len(la), len(lb)


@pytest.mark.parametrize("problem,n1,n2,lim,flux,nsteps", [("torus", 32, 32, 3, 1, 12), ("dipole", 32, 16, 3, 0, 12)])
def test_dump_file_matches_reference_bytes(harm, problem, n1, n2, lim, flux, nsteps):
    r = ht.ref_run(n1, n2, lim=lim, flux=flux, nsteps=nsteps, problem=problem, dump=True)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    cfg = ht.ref_config(r)
    kw = dict(eom=harm.EOM_FFDE, bc=harm.BC_STAR, omegastar=r["omegastar"]) if problem == "dipole" else {}
    h = harm.HarmGPU(n1, n2, cfg.pop("dx1"), cfg.pop("dx2"), lim=lim, fluxmethod=flux, currents=True, **kw, **cfg)
    g = r["geom"]
    h.upload_geometry(g["gcov"], g["gcon"], g["gdet"], g["conn"], g["floors"])
    h.set_prims(r["prims"][0], r["pflag"][0])
    h.set_time(r["times"][0][0], r["times"][0][1], 0)
    h.step_ch(nsteps)
    h.sync()
    mine = _dump_bytes(h, _header(r), r["coords"])
    assert mine == r["dump"], _first_difference(mine, r["dump"])
    h.close()


def test_restart_on_device_from_reference_rdump(harm):
    """A reference restart file continued on the device: the state read from
    it, uploaded and bounded, steps exactly as the oracle steps it; the
    device state written back out reads in again unchanged (to the file's
    15 digits)."""
    from harm_ramt_b200 import restart as R
    n, lim, flux, nsteps = 32, 4, 1, 20
    r = ht.ref_run(n, n, lim=lim, flux=flux, nsteps=5, dump=True)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    d = tempfile.mkdtemp(prefix="harm_rdump_")
    src = os.path.join(d, "rdump-0")
    with open(src, "wb") as f:
        f.write(r["rdump"])
    rd = R.read_rdump(src)
    p0 = np.zeros((n + 6, n + 6, 8))
    p0[3:-3, 3:-3] = rd["prims"]
    cfg = ht.ref_config(r)
    g = r["geom"]
    h = harm.HarmGPU(n, n, cfg.pop("dx1"), cfg.pop("dx2"), lim=lim, fluxmethod=flux, **cfg)
    h.upload_geometry(g["gcov"], g["gcon"], g["gdet"], g["conn"], g["floors"])
    h.set_prims(p0)
    h.bound_prims()
    hd = rd["header"]
    h.set_time(hd["t"], hd["dt"], hd["realnstep"])
    o = ht.Oracle(n, n, g, lim=lim, fluxmethod=flux, **ht.ref_config(r))
    po = o.bound(p0)
    fo = np.zeros(po.shape[:2] + (5,), dtype=np.int32)
    pg, _ = h.get_prims()
    assert np.array_equal(pg, po)
    t, dt = hd["t"], hd["dt"]
    for _ in range(nsteps):
        rc, t, dt = o.step(po, fo, t, dt)
        assert rc == 0
    h.step_ch(nsteps)
    st = h.sync()
    pg, fg = h.get_prims()
    assert np.array_equal(pg, po) and (st["t"], st["dt"]) == (t, dt)
    assert st["realnstep"] == hd["realnstep"] + nsteps
    out = os.path.join(d, "rdump-1")
    R.write_rdump(out, R.rdump_header_from_context(h, hd), pg, rd["accounting"], rd["rescaletype"], rd["lumvsr"])
    back = R.read_rdump(out)
    assert np.array_equal(back["prims"], np.vectorize(lambda x: float("%.15g" % x))(pg[3:-3, 3:-3]))
    assert back["header"]["realnstep"] == st["realnstep"]
    h.close()
    for fn in (src, out):
        os.unlink(fn)
    os.rmdir(d)
