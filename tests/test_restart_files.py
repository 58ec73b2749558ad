"""Reference restart files (restart.c, text form): the reader recovers the
header and the state the reference wrote (15 significant digits, as the
file holds), and reading then writing reproduces the reference's file byte
for byte (torus and force-free dipole).  Skipped without the reference
build."""
import os
import tempfile

import numpy as np
import pytest

import harmtest as ht
from harm_ramt_b200 import restart as R


@pytest.mark.parametrize("problem,n1,n2,lim,flux", [("torus", 32, 32, 3, 1), ("dipole", 32, 16, 3, 0)])
def test_rdump_read_write_roundtrip(problem, n1, n2, lim, flux):
    r = ht.ref_run(n1, n2, lim=lim, flux=flux, nsteps=7, problem=problem, dump=True)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    d = tempfile.mkdtemp(prefix="harm_rdump_")
    src, dst = os.path.join(d, "rdump-0"), os.path.join(d, "rdump-0.rewritten")
    with open(src, "wb") as f:
        f.write(r["rdump"])
    rd = R.read_rdump(src)
    h = rd["header"]
    assert (h["totalsize1"], h["totalsize2"], h["realnstep"]) == (n1, n2, 7)
    t, dt = r["times"][7]
    assert h["t"] == float("%.15g" % t) and h["dt"] == float("%.15g" % dt)
    p = ht.interior(r["prims"][7])
    assert np.array_equal(rd["prims"], np.vectorize(lambda x: float("%.15g" % x))(p))
    R.write_rdump(dst, h, rd["prims"], rd["accounting"], rd["rescaletype"], rd["lumvsr"])
    with open(dst, "rb") as f:
        assert f.read() == r["rdump"]
    os.unlink(src)
    os.unlink(dst)
    os.rmdir(d)
