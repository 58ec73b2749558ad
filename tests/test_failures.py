"""Fatal checks and bad input files, made on the host (no GPU involved).

A state with a corrupted zone is stepped by the oracle and by the reference
compiled from its own sources: both must stop at the same check, with the
same fail() code (global.h:562-579) at the same zone -- the first zone of
the first pass of the step in the reference's loop order (fail.c:4-57
reports the zone of the last get_geometry() call).  These cases pin what the
device must report through harm_status (tests/test_gpu_failures.py).

Restart files cut short or holding a non-number are rejected with a clear
error instead of producing a state.
"""
import os
import tempfile

import numpy as np
import pytest

import harmtest as ht
from harm_ramt_b200 import restart as R

NG = ht.NG

# (corrupted zones, expected (code, i, j)): a negative density with positive
# internal energy at a zone makes the fast speed superluminal in vchar
# (FAIL_COEFF_SUP = 5, vchar.c:87-92) on the x1 face at the zone's own left
# side, which is the first face of the step to see it; with several such
# zones the first one in the i-outer, j-inner face loop wins
FAIL_CASES = [
    ([(12, 14)], (5, 12, 14)),
    ([(20, 3), (5, 25), (5, 26)], (5, 5, 25)),
    ([(0, 5)], (5, 0, 5)),
    ([(31, 31), (31, 2)], (5, 31, 2)),
]


def corrupted_torus(n, zones, lim=3, flux=1):
    """(geometry, bounded initial torus with negative density at `zones`)"""
    import harm_ramt_b200 as hb
    par = hb.torus_params(n, n)
    geom = hb.torus_geometry(par)
    p0 = hb.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=lim, fluxmethod=flux, dx1=geom["dx1"], dx2=geom["dx2"])
    p = o.bound(p0)
    for i, j in zones:
        p[i + NG, j + NG, 0] = -1.2 * p[i + NG, j + NG, 1]
    return geom, p, o


@pytest.mark.parametrize("zones,expect", FAIL_CASES)
def test_oracle_reports_the_references_fail_code_and_zone(zones, expect):
    n = 32
    geom, p, o = corrupted_torus(n, zones)
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    rc, _, _ = o.step(p.copy(), f, 0.0, 1e-5)
    assert rc == expect[0] and o.fail() == expect
    r = ht.ref_fail(n, n, p)
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    assert r["rc"] != 0 and r["fail"] == expect, r


def test_oracle_clean_step_reports_no_failure():
    geom, p, o = corrupted_torus(32, [])
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    rc, _, _ = o.step(p, f, 0.0, 1e-5)
    assert rc == 0 and o.fail() == (0, 0, 0)


def _rdump_text(n1=8, n2=6):
    h = {name: (0.5 if conv == "g" else 1) for name, conv in R.HEADER_FIELDS}
    h.update(totalsize1=n1, totalsize2=n2)
    rng = np.random.default_rng(3)
    d = tempfile.mkdtemp(prefix="harm_rdump_")
    path = os.path.join(d, "rdump-0")
    R.write_rdump(path, h, rng.random((n1, n2, 8)))
    with open(path) as fh:
        return path, fh.read()


def test_rdump_roundtrip_synthetic():
    path, text = _rdump_text()
    rd = R.read_rdump(path)
    assert rd["prims"].shape == (8, 6, 8) and len(rd["lumvsr"]) == 8
    os.unlink(path)


@pytest.mark.parametrize("cut", ["header", "accounting", "body", "value"])
def test_truncated_or_corrupt_rdump_is_rejected(cut):
    path, text = _rdump_text()
    first, body = text.split("\n", 1)
    if cut == "header":
        bad = " ".join(first.split()[:20]) + "\n" + body
    elif cut == "accounting":
        bad = " ".join(first.split()[:len(R.HEADER_FIELDS) + 10]) + "\n" + body
    elif cut == "body":
        bad = first + "\n" + body[: len(body) // 2]
    else:
        bad = first + "\n" + body.replace(body.split()[7], "nan?", 1)
    with open(path, "w") as fh:
        fh.write(bad)
    with pytest.raises(ValueError, match="rdump"):
        R.read_rdump(path)
    os.unlink(path)
