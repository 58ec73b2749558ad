"""The update adjoint's two blocks on the device against their host build:
the con-to-prim implicit-function solve (ift_solve) and the geometric
source's adjoint (adj_source), run as one kernel (the solve's output feeding
the source adjoint in the same thread, as a fused update adjoint would) and
as two kernels (as harm_adjoint.cu runs them: k_adj_update, k_adj_source).
Both must equal the host build of the same functions bit for bit (IEEE ==),
on every active zone of a developed 64^2 torus with seeded right-hand sides.
The device code is built without contraction, like the host's, so the two
round alike operation by operation."""
import numpy as np
import pytest

from test_adjoint_blocks import _lib, _p

pytestmark = pytest.mark.gpu


def _inputs(harm):
    import harmtest as ht
    n = 64
    par = harm.torus_params(n, n)
    geom = harm.torus_geometry(par)
    p0 = harm.torus_init(par, geom)
    o = ht.Oracle(n, n, geom, lim=4, fluxmethod=1, dx1=geom["dx1"], dx2=geom["dx2"])
    p = o.bound(p0)
    f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
    t, dt = 0.0, 1e-5
    pb = None
    for s in range(60):
        if s == 59:
            pb = p.copy()
        rc, t, dt = o.step(p, f, t, dt)
        assert rc == 0
    act = (slice(3, n + 3), slice(3, n + 3))
    nz = n * n
    p1 = p[act].reshape(nz, 8)
    pbz = pb[act].reshape(nz, 8)
    geo = np.concatenate([geom["gcov"][act][:, :, 3].reshape(nz, 16), geom["gcon"][act][:, :, 3].reshape(nz, 16),
                          geom["gdet"][act][:, :, 3].reshape(nz, 1)], axis=1)
    conn = geom["conn"][act].reshape(nz, 64)
    rng = np.random.default_rng(2026)
    b = rng.standard_normal((nz, 8)) * np.abs(p1).max(axis=1, keepdims=True)
    return nz, p1, pbz, b, geo, conn, par.gam, 0.5 * dt


def test_update_adjoint_blocks_fused_and_split_equal_host(harm):
    lib = _lib()
    nz, p1, pb, b, geo, conn, gam, cdt = _inputs(harm)
    ins = [_p(x) for x in (p1, pb, b, geo, conn)]
    xh, lh = np.zeros((nz, 8)), np.zeros((nz, 8))
    lib.ab_probe_host(0, nz, *[q for _, q in ins], gam, cdt, _p(xh)[1], _p(lh)[1])
    assert np.isfinite(lh).all() and np.count_nonzero(xh) > 0
    for fused in (1, 0):
        xd, ld = np.zeros((nz, 8)), np.zeros((nz, 8))
        rc = lib.ab_probe_device(fused, nz, *[q for _, q in ins], gam, cdt, _p(xd)[1], _p(ld)[1])
        assert rc == 0, rc
        what = "one kernel" if fused else "two kernels"
        assert np.array_equal(xd, xh), f"{what}: ift_solve differs in {np.count_nonzero(xd != xh)} values"
        assert np.array_equal(ld, lh), (f"{what}: source adjoint differs in {np.count_nonzero(ld != lh)} values, "
                                        f"max rel {np.max(np.abs(ld - lh) / np.maximum(np.abs(lh), 1e-300)):.3e}")
    print(f"\nupdate adjoint blocks, {nz} zones: device (one kernel and two) == host, bit for bit")
    # the first build's con-to-prim step (8 x 8 local arrays) with the source
    # adjoint in the same kernel: reported against its own host build
    xl, ll = np.zeros((nz, 8)), np.zeros((nz, 8))
    lib.ab_probe_host(1, nz, *[q for _, q in ins], gam, cdt, _p(xl)[1], _p(ll)[1])
    xd, ld = np.zeros((nz, 8)), np.zeros((nz, 8))
    assert lib.ab_probe_device(2, nz, *[q for _, q in ins], gam, cdt, _p(xd)[1], _p(ld)[1]) == 0
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))
    print(f"legacy 8x8 solve + source adjoint in one kernel: solve differs from the host in "
          f"{np.count_nonzero(xd != xl)} values (max rel {rel(xd, xl):.2e}), source adjoint in "
          f"{np.count_nonzero(ld != ll)} (max rel {rel(ld, ll):.2e}); legacy vs current solve on the host: "
          f"max rel {rel(xl, xh):.2e}")
