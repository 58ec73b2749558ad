"""Test support: the oracle (C restatement, oracle/harm_oracle.c), the
reference compiled from its own sources (oracle/_ref, optional) and helpers
to drive them on the same inputs as the GPU path.

The oracle is test infrastructure only; the product never imports it.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SRC = os.path.join(ORACLE_DIR, "harm_oracle.c")
ORACLE_LIB = os.path.join(ORACLE_DIR, "libharm_oracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")

NG = 3


class OracleConfig(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("lim", ctypes.c_int), ("fluxmethod", ctypes.c_int),
                ("eom", ctypes.c_int), ("cour", ctypes.c_double), ("gam", ctypes.c_double), ("dx1", ctypes.c_double),
                ("dx2", ctypes.c_double), ("safe", ctypes.c_double), ("defcon", ctypes.c_double),
                ("gammamax", ctypes.c_double), ("gammafail", ctypes.c_double), ("bsqorholimit", ctypes.c_double),
                ("bsqoulimit", ctypes.c_double), ("tf", ctypes.c_double), ("bc", ctypes.c_int),
                ("omegastar", ctypes.c_double), ("fluxadjust", ctypes.c_int), ("gammadamp", ctypes.c_double)]


def build_oracle(force=False):
    """Compiles the C restatement with no FP contraction (like the reference)."""
    if (not force and os.path.exists(ORACLE_LIB)
            and os.path.getmtime(ORACLE_LIB) >= os.path.getmtime(ORACLE_SRC)
            and os.path.getmtime(ORACLE_LIB) >= os.path.getmtime(os.path.join(ORACLE_DIR, "harm_oracle.h"))):
        return ORACLE_LIB
    tmp = ORACLE_LIB + ".tmp%d" % os.getpid()
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", tmp, ORACLE_SRC,
                    "-lm"], check=True)
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


ORACLE_TL_SRC = os.path.join(ORACLE_DIR, "harm_oracle_tl.cpp")
ORACLE_TL_LIB = os.path.join(ORACLE_DIR, "libharm_oracle_tl.so")


def build_oracle_tl(force=False):
    """Compiles the tangent-linear form of the oracle (harm_oracle.c with a
    dual-number type, oracle/harm_oracle_tl.cpp), no FP contraction."""
    deps = [ORACLE_TL_SRC, ORACLE_SRC, os.path.join(ORACLE_DIR, "harm_oracle.h")]
    if not force and os.path.exists(ORACLE_TL_LIB) and all(os.path.getmtime(ORACLE_TL_LIB) >= os.path.getmtime(d)
                                                           for d in deps):
        return ORACLE_TL_LIB
    tmp = ORACLE_TL_LIB + ".tmp%d" % os.getpid()
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", tmp,
                    ORACLE_TL_SRC, "-lm"], check=True, cwd=ORACLE_DIR)
    os.replace(tmp, ORACLE_TL_LIB)
    return ORACLE_TL_LIB


class OracleTL:
    """The oracle's step in forward mode: a state and one tangent."""

    def __init__(self, n1, n2, geom, *, lim=3, fluxmethod=1, cour=0.8, gam=4.0 / 3.0, dx1, dx2, safe=1.3,
                 defcon=1.0, gammamax=25.0, gammafail=2500.0, bsqorholimit=20.0, bsqoulimit=100.0, tf=1e30, eom=0,
                 bc=0, omegastar=0.0, fluxadjust=0, gammadamp=5.0):
        lib = ctypes.CDLL(build_oracle_tl())
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        lib.tl_create.restype = vp
        lib.tl_create.argtypes = [ctypes.POINTER(OracleConfig), dp, dp, dp, dp, dp]
        lib.tl_destroy.argtypes = [vp]
        lib.tl_bound.argtypes = [vp, dp, dp]
        lib.tl_step.argtypes = [vp, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.c_double, ctypes.c_double]
        lib.tl_horizon.argtypes = [vp, dp, dp]
        self.lib = lib
        self.cfg = OracleConfig(n1, n2, lim, fluxmethod, eom, cour, gam, dx1, dx2, safe, defcon, gammamax, gammafail,
                                bsqorholimit, bsqoulimit, tf, bc, omegastar, fluxadjust, gammadamp)
        g = {k: np.ascontiguousarray(geom[k], dtype=np.float64) for k in ("gcov", "gcon", "gdet", "conn", "floors")}
        self.h = lib.tl_create(ctypes.byref(self.cfg), _dp(g["gcov"]), _dp(g["gcon"]), _dp(g["gdet"]), _dp(g["conn"]),
                               _dp(g["floors"]))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.tl_destroy(self.h)
            self.h = None

    def bound(self, p, dp):
        self.lib.tl_bound(self.h, _dp(p), _dp(dp))

    def step(self, p, dp, pflag, t, dt):
        return self.lib.tl_step(self.h, _dp(p), _dp(dp), pflag.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), t, dt)

    def horizon(self):
        v, d = np.zeros(6), np.zeros(6)
        self.lib.tl_horizon(self.h, _dp(v), _dp(d))
        return v, d

    def objective(self, p0, v, dts, wm=1.0, we=1.0):
        """J = sum_n dt_n (wm mdot_n + we edot_n) of the run from p0 (ghosts
        refilled by bound_prim) with the dt sequence dts, and its derivative
        along v (active zones)"""
        p = np.ascontiguousarray(p0, dtype=np.float64).copy()
        dp = np.ascontiguousarray(v, dtype=np.float64).copy()
        self.bound(p, dp)
        f = np.zeros(p.shape[:2] + (5,), dtype=np.int32)
        J = dJ = 0.0
        t = 0.0
        for dt in dts:
            rc = self.step(p, dp, f, t, float(dt))
            assert rc == 0, rc
            t += float(dt)
            hv, hd = self.horizon()
            J += float(dt) * (wm * hv[0] + we * (hv[2] + hv[3]))
            dJ += float(dt) * (wm * hd[0] + we * (hd[2] + hd[3]))
        return J, dJ, p, dp


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(build_oracle())
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        lib.ho_create.restype = vp
        lib.ho_create.argtypes = [ctypes.POINTER(OracleConfig), dp, dp, dp, dp, dp]
        lib.ho_destroy.argtypes = [vp]
        lib.ho_step.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int), dp, dp]
        lib.ho_bound.argtypes = [vp, dp]
        lib.ho_set_end_time.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp]
        lib.ho_init_currents.argtypes = [vp, dp, ctypes.c_double]
        lib.ho_init_currents.restype = None
        lib.ho_get_currents.argtypes = [vp, dp, dp, dp]
        lib.ho_get_currents.restype = None
        lib.ho_set_end_time.restype = None
        lib.ho_bsqflags.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int)]
        lib.ho_get_fluxes.argtypes = [vp, dp, dp]
        lib.ho_get_horizon.argtypes = [vp, dp]
        lib.ho_ncyclebreak.argtypes = [vp]
        lib.ho_ncyclebreak.restype = ctypes.c_long
        lib.ho_cycle_break_uniform.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int]
        lib.ho_cycle_break_uniform.restype = ctypes.c_double
        lib.ho_record_failures.argtypes = [vp, ctypes.c_int]
        lib.ho_get_failures.argtypes = [vp, ctypes.POINTER(ctypes.c_int), dp, dp]
        lib.ho_get_fail.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        lib.ho_get_fail.restype = None
        _oracle = lib
    return _oracle


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """The C restatement run on given geometry and state."""

    def __init__(self, n1, n2, geom, *, lim=3, fluxmethod=1, cour=0.8, gam=4.0 / 3.0, dx1, dx2, safe=1.3,
                 defcon=1.0, gammamax=25.0, gammafail=2500.0, bsqorholimit=20.0, bsqoulimit=100.0, tf=1e30, eom=0,
                 bc=0, omegastar=0.0, fluxadjust=0, gammadamp=5.0):
        self.lib = oracle_lib()
        self.cfg = OracleConfig(n1, n2, lim, fluxmethod, eom, cour, gam, dx1, dx2, safe, defcon, gammamax, gammafail,
                                bsqorholimit, bsqoulimit, tf, bc, omegastar, fluxadjust, gammadamp)
        self.geom = {k: np.ascontiguousarray(geom[k], dtype=np.float64) for k in ("gcov", "gcon", "gdet", "conn",
                                                                                     "floors")}
        g = self.geom
        self.h = self.lib.ho_create(ctypes.byref(self.cfg), _dp(g["gcov"]), _dp(g["gcon"]), _dp(g["gdet"]),
                                    _dp(g["conn"]), _dp(g["floors"]))
        self.n1m, self.n2m = n1 + 2 * NG, n2 + 2 * NG

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ho_destroy(self.h)
            self.h = None

    def init_currents(self, p, dt):
        self.lib.ho_init_currents(self.h, _dp(np.ascontiguousarray(p)), dt)

    def currents(self):
        jc, fc, cf = np.zeros((self.n1m, self.n2m, 4)), np.zeros((self.n1m, self.n2m, 6)), np.zeros(
            (self.n1m, self.n2m, 5, 3))
        self.lib.ho_get_currents(self.h, _dp(jc), _dp(fc), _dp(cf))
        return jc, fc, cf

    def set_end_time(self, tf, t, dt):
        """moves the end time; returns the re-clamped dt"""
        d = ctypes.c_double(dt)
        self.lib.ho_set_end_time(self.h, tf, t, ctypes.byref(d))
        return d.value

    def bound(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64).copy()
        self.lib.ho_bound(self.h, _dp(p))
        return p

    def step(self, p, pflag, t, dt):
        """one step in place; returns (rc, t, dt)"""
        tt, dd = ctypes.c_double(t), ctypes.c_double(dt)
        rc = self.lib.ho_step(self.h, _dp(p), pflag.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(tt),
                              ctypes.byref(dd))
        return rc, tt.value, dd.value

    def fluxes(self):
        f1 = np.zeros((self.n1m, self.n2m, 8))
        f2 = np.zeros((self.n1m, self.n2m, 8))
        self.lib.ho_get_fluxes(self.h, _dp(f1), _dp(f2))
        return f1, f2

    def fail(self):
        """(code, i, j) of the first fatal check of the last step (code 0: none)"""
        out = np.zeros(3, dtype=np.int32)
        self.lib.ho_get_fail(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return tuple(int(v) for v in out)

    def ncyclebreak(self):
        return self.lib.ho_ncyclebreak(self.h)

    def horizon(self):
        out = np.zeros(6)
        self.lib.ho_get_horizon(self.h, _dp(out))
        return out

    def record_failures(self, max_cases):
        """records the inputs of the next max_cases failed inversions"""
        self._rec_max = max_cases
        assert self.lib.ho_record_failures(self.h, max_cases) == 0

    def failures(self):
        """(zones [n, 2], U [n, 8] evolved form, guesses [n, 8]) recorded"""
        m = self._rec_max
        ij, U, pr = np.zeros((m, 2), dtype=np.int32), np.zeros((m, 8)), np.zeros((m, 8))
        n = self.lib.ho_get_failures(self.h, ij.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(U), _dp(pr))
        return ij[:n].copy(), U[:n].copy(), pr[:n].copy()


# ---------------------------------------------------------------- reference
def ref_lib_path(n1, n2, problem="torus"):
    p = os.path.join(REF_DIR, f"libharmref_{problem}_{n1}x{n2}.so")
    return p if os.path.exists(p) else None


def _ref_worker(libpath, lim, flux, cour, nsteps, outpath, dump=False, limits=None):
    """Runs in a child process: reference init + nsteps steps, pickled to
    outpath.  limits: (BSQORHOLIMIT, BSQOULIMIT, GAMMADAMP) or None."""
    import pickle
    lib = ctypes.CDLL(libpath)
    lib.hr_configure.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double]
    lib.hr_get_ncyclebreak.restype = ctypes.c_long
    lib.hr_configure(lim, flux, 2, cour, 0, 1e30)
    if limits is not None:
        lib.hr_set_limits.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.hr_set_limits(*[float(x) for x in limits])
    work = tempfile.mkdtemp(prefix="harmref_")
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(2)
    os.dup2(devnull, 2)
    os.dup2(devnull, 1)
    rc = lib.hr_init(work.encode())
    os.dup2(saved, 2)
    if rc != 0:
        raise RuntimeError("reference init failed")
    n1, n2 = lib.hr_n1(), lib.hr_n2()
    m1, m2 = n1 + 2 * NG, n2 + 2 * NG
    V = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    s = np.zeros(32)
    lib.hr_get_scalars(V(s))
    geom = dict(gcov=np.zeros((m1, m2, 4, 4, 4)), gcon=np.zeros((m1, m2, 4, 4, 4)), gdet=np.zeros((m1, m2, 4)),
                conn=np.zeros((m1, m2, 4, 4, 4)), floors=np.zeros((m1, m2, 2)))
    lib.hr_get_geometry(V(geom["gcov"]), V(geom["gcon"]), V(geom["gdet"]), V(geom["conn"]))
    lib.hr_get_floors(V(geom["floors"]))
    scal0 = s.copy()
    extra = {"eomtype": lib.hr_eomtype()}
    if hasattr(lib, "hr_get_omegastar"):
        lib.hr_get_omegastar.restype = ctypes.c_double
        extra["omegastar"] = lib.hr_get_omegastar()
    ps, pfs, ts, hz, cur = [], [], [], [], []
    for n in range(nsteps + 1):
        p = np.zeros((m1, m2, 8))
        pf = np.zeros((m1, m2, 5), dtype=np.int32)
        lib.hr_get_prims(V(p))
        lib.hr_get_pflag(V(pf))
        lib.hr_get_scalars(V(s))
        ps.append(p)
        pfs.append(pf)
        ts.append((s[0], s[1]))
        h6 = np.zeros(6)
        lib.hr_get_horizon(V(h6))
        hz.append(h6)
        jc, fc, cf = np.zeros((m1, m2, 4)), np.zeros((m1, m2, 6)), np.zeros((m1, m2, 5, 3))
        lib.hr_get_currents(V(jc), V(fc), V(cf))
        cur.append((jc, fc, cf))
        if n < nsteps:
            os.dup2(devnull, 2)
            rcs = lib.hr_step(1)
            os.dup2(saved, 2)
            if rcs != 0:
                raise RuntimeError("reference step failed")
    f1 = np.zeros((m1, m2, 8))
    f2 = np.zeros((m1, m2, 8))
    lib.hr_get_fluxes(V(f1), V(f2))
    if dump:
        # the reference's own dump file of the final state (cwd is the work dir)
        os.dup2(devnull, 2)
        lib.hr_dump.argtypes = [ctypes.c_char_p, ctypes.c_long]
        rcd = lib.hr_dump(work.encode(), 0)
        os.dup2(saved, 2)
        if rcd != 0:
            raise RuntimeError("reference dump failed")
        with open(os.path.join(work, "dumps", "dump0000"), "rb") as fd:
            extra["dump"] = fd.read()
        lib.hr_restart_write.argtypes = [ctypes.c_char_p, ctypes.c_long]
        os.dup2(devnull, 2)
        rcr = lib.hr_restart_write(work.encode(), 0)
        os.dup2(saved, 2)
        if rcr != 0:
            raise RuntimeError("reference restart_write failed")
        with open(os.path.join(work, "dumps", "rdump-0"), "rb") as fd:
            extra["rdump"] = fd.read()
        co = np.zeros((m1, m2, 4))
        lib.hr_get_coords(V(co))
        extra["coords"] = co
        extra["defcoord"] = lib.hr_get_defcoord()
    with open(outpath, "wb") as f:
        pickle.dump(dict(n1=n1, n2=n2, scalars=scal0, geom=geom, prims=ps, pflag=pfs, times=ts, horizon=hz, F1=f1, F2=f2,
                         currents=cur,
                         ncyclebreak=lib.hr_get_ncyclebreak(), **extra), f, protocol=4)


def ref_run(n1, n2, lim=3, flux=1, cour=0.8, nsteps=1, problem="torus", timeout=1800, dump=False, limits=None):
    """Runs the compiled reference (init + nsteps steps) in a fresh child
    process (its init() can run once per process) and returns its arrays."""
    import pickle
    import sys
    path = ref_lib_path(n1, n2, problem)
    if path is None:
        return None
    fd, out = tempfile.mkstemp(suffix=".pkl", prefix="harmref_")
    os.close(fd)
    code = ("import sys; sys.path.insert(0, %r); import harmtest; "
            "harmtest._ref_worker(%r, %d, %d, %r, %d, %r, %r, %r)"
            % (os.path.dirname(os.path.abspath(__file__)), path, lim, flux, float(cour), nsteps, out, bool(dump),
               None if limits is None else tuple(float(x) for x in limits)))
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference run failed (rc=%d): %s" % (r.returncode, r.stderr[-2000:]))
        with open(out, "rb") as f:
            return pickle.load(f)
    finally:
        os.unlink(out)


def _ref_pick_worker(libpath, methods, ij, U, pr, outpath):
    """Runs in a child process: reference init, then Utoprimgen_pick of each
    method on each case (zone ij, evolved U, guess pr)."""
    import pickle
    lib = ctypes.CDLL(libpath)
    lib.hr_configure.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double]
    lib.hr_configure(3, 1, 2, 0.8, 0, 1e30)
    work = tempfile.mkdtemp(prefix="harmref_")
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved, saved1 = os.dup(2), os.dup(1)
    os.dup2(devnull, 2)
    os.dup2(devnull, 1)
    try:
        if lib.hr_init(work.encode()) != 0:
            raise RuntimeError("reference init failed")
        V = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        out = {}
        for m in methods:
            prs = np.zeros_like(pr)
            codes = np.zeros(len(ij), dtype=np.int32)
            for c in range(len(ij)):
                pc = pr[c].copy()
                pf = ctypes.c_int(0)
                lib.hr_utoprim_pick(int(m), int(ij[c, 0]), int(ij[c, 1]), V(np.ascontiguousarray(U[c])), V(pc),
                                    ctypes.byref(pf))
                prs[c] = pc
                codes[c] = pf.value
            out[int(m)] = (prs, codes)
        chain_pr = np.zeros_like(pr)
        chain_codes = np.zeros(len(ij), dtype=np.int32)
        lib.hr_utoprimgen.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        for c in range(len(ij)):
            pc = pr[c].copy()
            pf = ctypes.c_int(0)
            lib.hr_utoprimgen(int(ij[c, 0]), int(ij[c, 1]), V(np.ascontiguousarray(U[c])), V(pc), ctypes.byref(pf))
            chain_pr[c] = pc
            chain_codes[c] = pf.value
        out["chain"] = (chain_pr, chain_codes)
    finally:
        os.dup2(saved, 2)
        os.dup2(saved1, 1)
    with open(outpath, "wb") as f:
        pickle.dump(out, f, protocol=4)


def ref_utoprim_pick(n1, n2, methods, ij, U, pr, problem="torusta", timeout=1800):
    """Each method of the retry chain (Utoprimgen_pick, step_ch.h:39-53 ids)
    and the whole Utoprimgen (the chain itself in the torusta build) of the
    compiled reference on the given cases: {method: (pr, pflag)} plus
    "chain".  None when that build is absent."""
    import pickle
    import sys
    path = ref_lib_path(n1, n2, problem)
    if path is None:
        return None
    fd, out = tempfile.mkstemp(suffix=".pkl", prefix="harmref_")
    os.close(fd)
    fi, inp = tempfile.mkstemp(suffix=".npz", prefix="harmref_")
    os.close(fi)
    np.savez(inp, ij=ij, U=U, pr=pr)
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import harmtest; d = np.load(%r); "
            "harmtest._ref_pick_worker(%r, %r, d['ij'], d['U'], d['pr'], %r)"
            % (os.path.dirname(os.path.abspath(__file__)), inp, path, list(methods), out))
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference run failed (rc=%d): %s" % (r.returncode, r.stderr[-2000:]))
        with open(out, "rb") as f:
            return pickle.load(f)
    finally:
        os.unlink(out)
        os.unlink(inp)


def _ref_fail_worker(libpath, lim, flux, prims, outpath):
    """Runs in a child process: reference init, then its step from the given
    state; records the step's return and the first fail() (code, i, j)."""
    import pickle
    lib = ctypes.CDLL(libpath)
    lib.hr_configure.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double]
    lib.hr_configure(lim, flux, 2, 0.8, 0, 1e30)
    work = tempfile.mkdtemp(prefix="harmref_")
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved, saved1 = os.dup(2), os.dup(1)
    os.dup2(devnull, 2)
    os.dup2(devnull, 1)
    try:
        if lib.hr_init(work.encode()) != 0:
            raise RuntimeError("reference init failed")
        V = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        lib.hr_set_prims(V(np.ascontiguousarray(prims, dtype=np.float64)))
        lib.hr_clear_fail()
        rc = lib.hr_step(1)
        out = np.zeros(3, dtype=np.int32)
        lib.hr_get_fail(V(out))
    finally:
        os.dup2(saved, 2)
        os.dup2(saved1, 1)
    with open(outpath, "wb") as f:
        pickle.dump(dict(rc=rc, fail=tuple(int(v) for v in out)), f, protocol=4)


def ref_fail(n1, n2, prims, lim=3, flux=1, problem="torus", timeout=600):
    """The compiled reference's step from `prims` (reference layout, ghosts
    included): {rc, fail: (code, i, j)} of its first fail() call, or None
    when that build is absent."""
    import pickle
    import sys
    path = ref_lib_path(n1, n2, problem)
    if path is None:
        return None
    fd, out = tempfile.mkstemp(suffix=".pkl", prefix="harmref_")
    os.close(fd)
    fi, inp = tempfile.mkstemp(suffix=".npy", prefix="harmref_")
    os.close(fi)
    np.save(inp, np.ascontiguousarray(prims, dtype=np.float64))
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import harmtest; "
            "harmtest._ref_fail_worker(%r, %d, %d, np.load(%r), %r)"
            % (os.path.dirname(os.path.abspath(__file__)), path, lim, flux, inp, out))
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference run failed (rc=%d): %s" % (r.returncode, r.stderr[-2000:]))
        with open(out, "rb") as f:
            return pickle.load(f)
    finally:
        os.unlink(out)
        os.unlink(inp)


def ref_config(r):
    """harm config keyword arguments from a reference run's scalars."""
    s = r["scalars"]
    return dict(cour=s[12], gam=s[3], dx1=s[10], dx2=s[11], safe=s[20], defcon=s[21], gammamax=s[16],
                gammafail=s[17], bsqorholimit=s[18], bsqoulimit=s[19], gammadamp=s[28], fluxadjust=int(s[29]))


def interior(a):
    return a[NG:-NG, NG:-NG]


# ---------------------------------------------------------------- retry chain
TA_HOST_SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tryagain_host.cu")
TA_HOST_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "libtryagain_host.so")
TA_HDRS = [os.path.join(ROOT, "harm_ramt_b200", "csrc", f) for f in ("harm_tryagain.cuh", "harm_device.cuh")]


def tryagain_host_lib():
    """The retry chain's inversions (harm_tryagain.cuh) compiled for the CPU
    (tests/tryagain_host.cu), or None without nvcc."""
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        return None
    deps = [TA_HOST_SRC] + TA_HDRS
    if not os.path.exists(TA_HOST_LIB) or any(os.path.getmtime(d) > os.path.getmtime(TA_HOST_LIB) for d in deps):
        os.makedirs(os.path.dirname(TA_HOST_LIB), exist_ok=True)
        subprocess.run([nvcc, "-O2", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o",
                        TA_HOST_LIB + ".tmp", TA_HOST_SRC], check=True, capture_output=True)
        os.replace(TA_HOST_LIB + ".tmp", TA_HOST_LIB)
    lib = ctypes.CDLL(TA_HOST_LIB)
    P = ctypes.POINTER(ctypes.c_double)
    d = ctypes.c_double
    lib.ta_pick.argtypes = [ctypes.c_int, P, P, d, d, d, P, P]
    lib.ta_chain.argtypes = [P, P, d, d, d, P, P, P, ctypes.c_int]
    lib.ta_primtoU.argtypes = [P, P, d, d, P, P]
    lib.ta_primtoU.restype = None
    return lib


def cent_geometry(geom, i, j):
    """(gcov 4x4, gcon 4x4, sqrt(-g)) at the zone centre (i, j)"""
    return (np.ascontiguousarray(geom["gcov"][i + NG, j + NG, 3]), np.ascontiguousarray(geom["gcon"][i + NG, j + NG, 3]),
            float(geom["gdet"][i + NG, j + NG, 3]))
