"""B200 (sm_100a) implementation of HARM's per-step finite-volume update.

Python host mirror of the C ABI in include/harm_b200.h (loaded with ctypes
from the in-tree libharm_b200.so).  The operator is the reference's
``step_ch()`` (step_ch.c:16): :class:`HarmGPU` holds the device-resident copy
of the reference globals it reads and writes (p, pflag, t, dt and the
geometry tables) and :meth:`HarmGPU.step_ch` advances them by whole steps.

Arrays use the reference's layout (defs.h) over the full grid including the
3 ghost zones on each side: prims ``[n1+6, n2+6, 8]``, pflag
``[n1+6, n2+6, 5]``, gcov/gcon ``[n1+6, n2+6, 4, 4, 4]``, gdet
``[n1+6, n2+6, 4]``, conn ``[n1+6, n2+6, 4, 4, 4]``, floors
``[n1+6, n2+6, 2]``.

There is no CPU fallback: the step runs only on the CUDA device and fails
loudly when the library or the device is missing.  The torus set-up helpers
(:func:`torus_geometry`, :func:`torus_init`) are host code of the plugin
surface and run anywhere.
"""
import ctypes
import os

import numpy as np

__all__ = ["HarmGPU", "HarmError", "torus_params", "torus_geometry", "torus_init", "load_library", "LIB_PATH",
           "LIM_MC", "LIM_PARA", "FLUX_LAXF", "FLUX_HLL", "PREC_FP64", "PREC_MIXED", "EOM_GRMHD", "EOM_FFDE",
           "BC_TORUS", "BC_STAR", "NG", "NPR", "pinned_empty", "torus_context", "torus_dump_coords", "Ensemble"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libharm_b200.so")
NG = 3
NPR = 8
LIM_MC, LIM_PARA = 3, 4
FLUX_LAXF, FLUX_HLL = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
EOM_GRMHD, EOM_FFDE = 0, 1
BC_TORUS, BC_STAR = 0, 1
# con-to-prim methods of Utoprimgen_pick (step_ch.h:39-53); INV_CHAIN: the
# whole Utoprimgen with the UTOPRIMTRYAGAIN retry chain
INV_5D1, INV_2D, INV_1D, INV_1DOPT, INV_1DFINAL, INV_2DFINAL, INV_5D2, INV_CHAIN = 0, 2, 3, 4, 5, 6, 7, -1
TRYAGAIN_CHAIN = (INV_5D1, INV_2D, INV_1D, INV_1DOPT, INV_1DFINAL, INV_2DFINAL, INV_5D2)

_ERRORS = {0: "ok", 1: "invalid argument", 2: "no usable CUDA device (sm_100 required)", 3: "CUDA runtime error",
           4: "device allocation failed", 5: "geometry tables missing or not symmetric",
           6: "fatal check of the reference step fired"}
# fail() codes of the reference, global.h:562-579
FAIL_NAMES = {1: "UTOPRIM_NEG", 2: "UTOPRIM_TEST", 3: "VCHAR_DISCR", 4: "COEFF_NEG", 5: "COEFF_SUP",
              6: "UTCALC_DISCR", 7: "FAIL_LDZ", 8: "FAIL_BCFIX", 9: "FAIL_VSQ_NEG",
              20: "FFDE_SPACELIKE (Utoprim_ffde, phys.ffde.c:281)"}


class HarmError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: {_ERRORS.get(code, 'error %d' % code)}" if what else _ERRORS.get(code, str(code)))


class _Config(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("lim", ctypes.c_int), ("fluxmethod", ctypes.c_int),
                ("eom", ctypes.c_int), ("precision", ctypes.c_int), ("cour", ctypes.c_double),
                ("gam", ctypes.c_double), ("dx1", ctypes.c_double), ("dx2", ctypes.c_double),
                ("safe", ctypes.c_double), ("defcon", ctypes.c_double), ("gammamax", ctypes.c_double),
                ("gammafail", ctypes.c_double), ("bsqorholimit", ctypes.c_double),
                ("bsqoulimit", ctypes.c_double), ("tf", ctypes.c_double), ("bc", ctypes.c_int),
                ("omegastar", ctypes.c_double), ("currents", ctypes.c_int), ("tryagain", ctypes.c_int),
                ("fluxadjust", ctypes.c_int), ("gammadamp", ctypes.c_double)]


class _DumpHeader(ctypes.Structure):
    _fields_ = [("startx1", ctypes.c_double), ("startx2", ctypes.c_double), ("a", ctypes.c_double),
                ("R0", ctypes.c_double), ("Rin", ctypes.c_double), ("Rout", ctypes.c_double),
                ("hslope", ctypes.c_double), ("defcoord", ctypes.c_int)]


class _Tiles(ctypes.Structure):
    _fields_ = [("update_x", ctypes.c_int), ("update_y", ctypes.c_int), ("small_x", ctypes.c_int),
                ("small_y", ctypes.c_int)]


class _Status(ctypes.Structure):
    _fields_ = [("fail_code", ctypes.c_int), ("fail_i", ctypes.c_int), ("fail_j", ctypes.c_int),
                ("fixups", ctypes.c_int), ("realnstep", ctypes.c_longlong), ("t", ctypes.c_double),
                ("dt", ctypes.c_double), ("newton_iters", ctypes.c_ulonglong), ("chk_multi", ctypes.c_int),
                ("deferred", ctypes.c_int), ("fail_step", ctypes.c_longlong)]


class _TorusParams(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("seed", ctypes.c_int), ("reserved", ctypes.c_int),
                ("a", ctypes.c_double), ("hslope", ctypes.c_double), ("rout", ctypes.c_double),
                ("rin_over_rhor", ctypes.c_double), ("gam", ctypes.c_double), ("torus_rin", ctypes.c_double),
                ("torus_rmax", ctypes.c_double), ("kappa", ctypes.c_double), ("beta", ctypes.c_double),
                ("randfact", ctypes.c_double), ("rhomin", ctypes.c_double), ("uumin", ctypes.c_double),
                ("rhominlimit", ctypes.c_double), ("uuminlimit", ctypes.c_double), ("gammamax", ctypes.c_double)]


class _DipoleParams(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("rin", ctypes.c_double), ("rout", ctypes.c_double),
                ("gam", ctypes.c_double), ("bpole", ctypes.c_double), ("omegastar", ctypes.c_double),
                ("rhomin", ctypes.c_double), ("uumin", ctypes.c_double), ("rhominlimit", ctypes.c_double),
                ("uuminlimit", ctypes.c_double), ("gammamax", ctypes.c_double)]


_lib = None

EXPORTS = ["harm_create", "harm_upload_geometry", "harm_set_prims", "harm_get_prims", "harm_bound_prims",
           "harm_set_time", "harm_step", "harm_sync", "harm_get_fluxes", "harm_destroy", "harm_error_string",
           "harm_torus_default_params", "harm_torus_geometry", "harm_torus_init", "harm_profile_step",
           "harm_kernel_name", "harm_get_horizon", "harm_set_end_time", "harm_get_currents", "harm_write_dump",
           "harm_torus_dump_coords", "harm_set_tiles", "harm_get_tiles", "harm_ensemble_create", "harm_ensemble_step",
           "harm_ensemble_sync", "harm_ensemble_destroy", "harm_adjoint_run", "harm_run_fixed_dt",
           "harm_torus_init_vpot", "harm_torus_vpot_to_field", "harm_torus_vpot_adjoint", "harm_invert_zones",
           "harm_measure_fp64_peak", "harm_dipole_default_params", "harm_dipole_geometry", "harm_dipole_init"]


def load_library(path=None):
    """Loads libharm_b200.so, building it first when its sources are newer
    (a failed build raises: a library older than its sources is never used
    silently).  With HARM_PREBUILT_ONLY=1 in the environment the library in
    the package is loaded as it is.  Raises if it cannot be loaded."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if path is None and not os.environ.get("HARM_PREBUILT_ONLY"):
        from . import build as _build
        if _build.needs_build():
            _build.build()
    lib = ctypes.CDLL(p)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lib.harm_create.argtypes = [ctypes.POINTER(_Config), vp, ctypes.POINTER(vp)]
    lib.harm_upload_geometry.argtypes = [vp, dp, dp, dp, dp, dp]
    lib.harm_set_prims.argtypes = [vp, dp, ip, ctypes.c_int]
    lib.harm_get_prims.argtypes = [vp, dp, ip]
    lib.harm_bound_prims.argtypes = [vp]
    lib.harm_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_longlong]
    lib.harm_set_end_time.argtypes = [vp, ctypes.c_double]
    lib.harm_step.argtypes = [vp, ctypes.c_int]
    lib.harm_invert_zones.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, dp, dp, ip]
    lib.harm_sync.argtypes = [vp, ctypes.POINTER(_Status)]
    lib.harm_get_fluxes.argtypes = [vp, dp, dp]
    lib.harm_destroy.argtypes = [vp]
    lib.harm_destroy.restype = None
    lib.harm_error_string.argtypes = [ctypes.c_int]
    lib.harm_error_string.restype = ctypes.c_char_p
    lib.harm_torus_default_params.argtypes = [ctypes.POINTER(_TorusParams)]
    lib.harm_torus_default_params.restype = None
    lib.harm_torus_geometry.argtypes = [ctypes.POINTER(_TorusParams), dp, dp, dp, dp, dp, dp]
    lib.harm_torus_init.argtypes = [ctypes.POINTER(_TorusParams), dp, dp, dp, dp]
    lib.harm_torus_init_vpot.argtypes = [ctypes.POINTER(_TorusParams), dp, dp, dp, dp, dp, dp]
    lib.harm_torus_vpot_to_field.argtypes = [ctypes.POINTER(_TorusParams), dp, dp, dp, dp]
    lib.harm_torus_vpot_adjoint.argtypes = [ctypes.POINTER(_TorusParams), dp, dp, dp, dp]
    lib.harm_profile_step.argtypes = [vp, dp, ip, ctypes.c_int]
    lib.harm_get_horizon.argtypes = [vp, dp]
    lib.harm_get_currents.argtypes = [vp, dp, dp, dp]
    lib.harm_write_dump.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(_DumpHeader), dp]
    lib.harm_set_tiles.argtypes = [vp, ctypes.POINTER(_Tiles)]
    lib.harm_adjoint_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp,
                                     dp]
    lib.harm_run_fixed_dt.argtypes = [vp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp]
    lib.harm_get_tiles.argtypes = [vp, ctypes.POINTER(_Tiles)]
    lib.harm_ensemble_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, vp, ctypes.POINTER(vp)]
    lib.harm_ensemble_step.argtypes = [vp, ctypes.c_int]
    lib.harm_ensemble_sync.argtypes = [vp, ctypes.POINTER(_Status)]
    lib.harm_ensemble_destroy.argtypes = [vp]
    lib.harm_ensemble_destroy.restype = None
    lib.harm_torus_dump_coords.argtypes = [ctypes.POINTER(_TorusParams), ctypes.POINTER(_DumpHeader), dp]
    lib.harm_dipole_default_params.argtypes = [ctypes.POINTER(_DipoleParams)]
    lib.harm_dipole_default_params.restype = None
    lib.harm_dipole_geometry.argtypes = [ctypes.POINTER(_DipoleParams), dp, dp, dp, dp, dp, dp]
    lib.harm_dipole_init.argtypes = [ctypes.POINTER(_DipoleParams), dp, dp, dp, dp]
    lib.harm_measure_fp64_peak.argtypes = [dp]
    lib.harm_kernel_name.argtypes = [ctypes.c_int]
    lib.harm_kernel_name.restype = ctypes.c_char_p
    if path is None:
        _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _check(rc, what):
    if rc != 0:
        raise HarmError(rc, what)


# ----------------------------------------------------------------- set-up
def torus_params(n1=128, n2=128, **kw):
    """The benchmark torus parameters (include/harm_setup.h) with overrides."""
    lib = load_library()
    p = _TorusParams()
    lib.harm_torus_default_params(ctypes.byref(p))
    p.n1, p.n2 = n1, n2
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def torus_geometry(params):
    """set_grid() for the torus grid: dict of gcov, gcon, gdet, conn, floors
    and the grid scalars (startx1, startx2, dx1, dx2, Rin, Rhor)."""
    lib = load_library()
    n1m, n2m = params.n1 + 2 * NG, params.n2 + 2 * NG
    g = dict(gcov=np.zeros((n1m, n2m, 4, 4, 4)), gcon=np.zeros((n1m, n2m, 4, 4, 4)), gdet=np.zeros((n1m, n2m, 4)),
             conn=np.zeros((n1m, n2m, 4, 4, 4)), floors=np.zeros((n1m, n2m, 2)))
    grid = np.zeros(6)
    _check(lib.harm_torus_geometry(ctypes.byref(params), _dp(g["gcov"]), _dp(g["gcon"]), _dp(g["gdet"]),
                                   _dp(g["conn"]), _dp(g["floors"]), _dp(grid)), "harm_torus_geometry")
    g.update(startx1=grid[0], startx2=grid[1], dx1=grid[2], dx2=grid[3], Rin=grid[4], Rhor=grid[5])
    return g


def torus_init(params, geom):
    """init() for the torus: active-zone primitives (ghosts still to bound)."""
    lib = load_library()
    n1m, n2m = params.n1 + 2 * NG, params.n2 + 2 * NG
    p = np.zeros((n1m, n2m, NPR))
    _check(lib.harm_torus_init(ctypes.byref(params), _dp(geom["gcov"]), _dp(geom["gcon"]), _dp(geom["gdet"]),
                               _dp(p)), "harm_torus_init")
    return p


def torus_init_vpot(params, geom):
    """torus_init() with the corner vector potential A_phi [n1+1, n2+1] and
    the two field normalisation factors: (prims, A, norm)."""
    lib = load_library()
    n1m, n2m = params.n1 + 2 * NG, params.n2 + 2 * NG
    p = np.zeros((n1m, n2m, NPR))
    A = np.zeros((params.n1 + 1, params.n2 + 1))
    norm = np.zeros(2)
    _check(lib.harm_torus_init_vpot(ctypes.byref(params), _dp(geom["gcov"]), _dp(geom["gcon"]), _dp(geom["gdet"]),
                                    _dp(p), _dp(A), _dp(norm)), "harm_torus_init_vpot")
    return p, A, norm


def vpot_to_field(params, geom, A, norm, prims):
    """A copy of prims whose active B1, B2 come from the vector potential A
    (normalised by the fixed factors norm)."""
    lib = load_library()
    p = np.ascontiguousarray(prims, dtype=np.float64).copy()
    A = np.ascontiguousarray(A, dtype=np.float64)
    norm = np.ascontiguousarray(norm, dtype=np.float64)
    _check(lib.harm_torus_vpot_to_field(ctypes.byref(params), _dp(geom["gdet"]), _dp(A), _dp(norm), _dp(p)),
           "harm_torus_vpot_to_field")
    return p


def vpot_adjoint(params, geom, grad, norm):
    """dJ/dA [n1+1, n2+1] from dJ/dprims (e.g. HarmGPU.adjoint's gradient)."""
    lib = load_library()
    g = np.ascontiguousarray(grad, dtype=np.float64)
    norm = np.ascontiguousarray(norm, dtype=np.float64)
    gA = np.zeros((params.n1 + 1, params.n2 + 1))
    _check(lib.harm_torus_vpot_adjoint(ctypes.byref(params), _dp(geom["gdet"]), _dp(g), _dp(norm), _dp(gA)),
           "harm_torus_vpot_adjoint")
    return gA


# ----------------------------------------------------------------- device
class HarmGPU:
    """Device-resident state of the reference's step and its step_ch()."""

    def __init__(self, n1, n2, dx1, dx2, *, lim=LIM_MC, fluxmethod=FLUX_HLL, cour=0.8, gam=4.0 / 3.0, safe=1.3,
                 defcon=1.0, gammamax=25.0, gammafail=2500.0, bsqorholimit=20.0, bsqoulimit=100.0, tf=1.0e30,
                 precision=PREC_FP64, stream=None, eom=EOM_GRMHD, bc=BC_TORUS, omegastar=0.0, currents=False,
                 tryagain=False, fluxadjust=0, gammadamp=5.0):
        self.lib = load_library()
        self.n1, self.n2 = n1, n2
        self.n1m, self.n2m = n1 + 2 * NG, n2 + 2 * NG
        self.safe = safe
        cfg = _Config(n1, n2, lim, fluxmethod, eom, precision, cour, gam, dx1, dx2, safe, defcon, gammamax, gammafail,
                      bsqorholimit, bsqoulimit, tf, bc, omegastar, int(bool(currents)), int(bool(tryagain)),
                      int(fluxadjust), float(gammadamp))
        h = ctypes.c_void_p()
        _check(self.lib.harm_create(ctypes.byref(cfg), ctypes.c_void_p(stream or 0), ctypes.byref(h)), "harm_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.harm_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload_geometry(self, gcov, gcon, gdet, conn, floors):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (gcov, gcon, gdet, conn, floors)]
        _check(self.lib.harm_upload_geometry(self._h, *[_dp(x) for x in arrs]), "harm_upload_geometry")

    def set_prims(self, prims, pflag=None, reset_gammacheck=True):
        p = np.ascontiguousarray(prims, dtype=np.float64)
        assert p.shape == (self.n1m, self.n2m, NPR)
        f = None if pflag is None else np.ascontiguousarray(pflag, dtype=np.int32)
        _check(self.lib.harm_set_prims(self._h, _dp(p), None if f is None else _ip(f), int(bool(reset_gammacheck))),
               "harm_set_prims")

    def get_prims(self, out=None, with_flags=True):
        """Device -> host copy; `out=(prims, pflag)` reuses caller buffers
        (pinned buffers from :func:`pinned_empty` make the copy fastest)."""
        if out is None:
            p = np.zeros((self.n1m, self.n2m, NPR))
            f = np.zeros((self.n1m, self.n2m, 5), dtype=np.int32) if with_flags else None
        else:
            p, f = out
            assert p.flags.c_contiguous and p.dtype == np.float64 and p.shape == (self.n1m, self.n2m, NPR)
            assert f is None or (f.flags.c_contiguous and f.dtype == np.int32 and f.shape == (self.n1m, self.n2m, 5))
        _check(self.lib.harm_get_prims(self._h, _dp(p), None if f is None else _ip(f)), "harm_get_prims")
        return p, f

    def bound_prims(self):
        _check(self.lib.harm_bound_prims(self._h), "harm_bound_prims")

    def set_time(self, t, dt, realnstep=0):
        _check(self.lib.harm_set_time(self._h, t, dt, realnstep), "harm_set_time")

    def set_end_time(self, tf):
        """Moves the end time (dt is clamped so that t + dt <= tf)."""
        _check(self.lib.harm_set_end_time(self._h, float(tf)), "harm_set_end_time")

    def run_to(self, tf, max_chunk=500):
        """Advances until t reaches tf and returns the status.  The end time
        is moved to tf, so the last step is clamped onto it, and steps are
        enqueued in chunks that cannot pass tf even if dt grows by the
        factor ``safe`` every step (a step past the end time runs at dt = 0
        and would still re-invert every zone)."""
        import math
        self.set_end_time(tf)
        st = self.sync()
        g = self.safe
        while st["t"] < tf:
            if st["dt"] <= 0.0:
                raise HarmError(1, f"run_to: dt = {st['dt']} at t = {st['t']} < {tf}")
            x = (tf - st["t"]) / st["dt"]
            k = int(math.log1p((g - 1.0) * x) / math.log(g)) if g > 1.0 else int(x)
            self.step_ch(min(max(k, 1), max_chunk))
            st = self.sync()
        return st

    def invert_zones(self, which, zones, U, guess):
        """One con-to-prim method of Utoprimgen_pick (step_ch.c:583-600;
        which: INV_5D1 ... INV_5D2, or INV_CHAIN for the whole Utoprimgen with
        the UTOPRIMTRYAGAIN retry chain) on the device at the given active
        zones (n x 2 array of i, j), U the evolved conserved vectors (n x 8),
        guess the initial primitives (n x 8).  Returns (primitives, pflag)."""
        zones = np.ascontiguousarray(zones, dtype=np.int32).reshape(-1, 2)
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(-1, NPR)
        pr = np.ascontiguousarray(guess, dtype=np.float64).reshape(-1, NPR).copy()
        fl = np.zeros(len(zones), dtype=np.int32)
        _check(self.lib.harm_invert_zones(self._h, int(which), len(zones), _ip(zones), _dp(U), _dp(pr), _ip(fl)),
               "harm_invert_zones")
        return pr, fl

    def step_ch(self, nsteps=1):
        """Enqueue nsteps reference steps (asynchronous)."""
        _check(self.lib.harm_step(self._h, int(nsteps)), "harm_step")

    def sync(self, raise_on_fail=True):
        st = _Status()
        rc = self.lib.harm_sync(self._h, ctypes.byref(st))
        d = dict(fail_code=st.fail_code, fail_i=st.fail_i, fail_j=st.fail_j, fixups=st.fixups,
                 realnstep=st.realnstep, t=st.t, dt=st.dt, newton_iters=st.newton_iters, chk_multi=st.chk_multi,
                 deferred=st.deferred, fail_step=st.fail_step)
        if rc == 6 and raise_on_fail:
            raise HarmError(rc, f"step failed with {FAIL_NAMES.get(st.fail_code, st.fail_code)} at zone "
                                f"({st.fail_i},{st.fail_j})")
        if rc not in (0, 6):
            raise HarmError(rc, "harm_sync")
        return d

    def profile_step(self):
        """One step with a CUDA event after every kernel: {name: (ms, launches)}."""
        nk = 15
        ms = np.zeros(nk)
        n = np.zeros(nk, dtype=np.int32)
        _check(self.lib.harm_profile_step(self._h, _dp(ms), _ip(n), nk), "harm_profile_step")
        return {self.lib.harm_kernel_name(k).decode(): (float(ms[k]), int(n[k])) for k in range(nk)}

    def get_horizon(self):
        """diag_flux()'s inner-face accounting: dict of pdot_rho, pdot_uu,
        em_bsq_term (pdotterms[3][UU]), em_bb_term (pdotterms[6][UU]),
        pcum_rho, pcum_uu."""
        out = np.zeros(6)
        _check(self.lib.harm_get_horizon(self._h, _dp(out)), "harm_get_horizon")
        return dict(zip(("pdot_rho", "pdot_uu", "em_bsq_term", "em_bb_term", "pcum_rho", "pcum_uu"), out.tolist()))

    def get_currents(self):
        """(jcon [n1m,n2m,4], fcon [n1m,n2m,6], cfaraday [n1m,n2m,5,3]) of a
        context created with currents=True (phys.c:1124-1455 layouts)."""
        jc = np.zeros((self.n1m, self.n2m, 4))
        fc = np.zeros((self.n1m, self.n2m, 6))
        cf = np.zeros((self.n1m, self.n2m, 5, 3))
        _check(self.lib.harm_get_currents(self._h, _dp(jc), _dp(fc), _dp(cf)), "harm_get_currents")
        return jc, fc, cf

    def write_dump(self, path, header, coords):
        """The reference's text dump file of the device state (dump.c).
        header: dict of startx1, startx2, a, R0, Rin, Rout, hslope, defcoord;
        coords: [n1m, n2m, 4] X1, X2, r, th at zone centres.  Needs
        currents=True."""
        h = _DumpHeader(**{k: header[k] for k in ("startx1", "startx2", "a", "R0", "Rin", "Rout", "hslope",
                                                   "defcoord")})
        co = np.ascontiguousarray(coords, dtype=np.float64)
        assert co.shape == (self.n1m, self.n2m, 4)
        _check(self.lib.harm_write_dump(self._h, os.fsencode(path), ctypes.byref(h), _dp(co)), "harm_write_dump")

    def set_tiles(self, update=(32, 4), small=(32, 4)):
        """Block shapes of k_update (<= 128 threads) and of the small
        stencil kernels (<= 1024 threads)."""
        t = _Tiles(int(update[0]), int(update[1]), int(small[0]), int(small[1]))
        _check(self.lib.harm_set_tiles(self._h, ctypes.byref(t)), "harm_set_tiles")

    def get_tiles(self):
        t = _Tiles()
        _check(self.lib.harm_get_tiles(self._h, ctypes.byref(t)), "harm_get_tiles")
        return (t.update_x, t.update_y), (t.small_x, t.small_y)

    def adjoint(self, nsteps, checkpoint_every=16, w_mass=1.0, w_em=0.0, lam_final=None):
        """Forward nsteps from the current state (its ghost zones first
        refilled by the boundary conditions), then the adjoint back: returns
        (J, dJ/dp_0 [n1m, n2m, 8] on the active zones (ghost entries 0), dt
        sequence, (forward ms, backward ms)).  The context ends at the
        forward run's final state."""
        J = ctypes.c_double()
        grad = np.zeros((self.n1m, self.n2m, NPR))
        dts = np.zeros(int(nsteps))
        ms = np.zeros(2)
        lam = None if lam_final is None else np.ascontiguousarray(lam_final, dtype=np.float64)
        _check(self.lib.harm_adjoint_run(self._h, int(nsteps), int(checkpoint_every), float(w_mass), float(w_em),
                                         None if lam is None else _dp(lam), ctypes.byref(J), _dp(grad), _dp(dts),
                                         _dp(ms)), "harm_adjoint_run")
        return J.value, grad, dts, (ms[0], ms[1])

    def run_fixed_dt(self, dts, w_mass=1.0, w_em=0.0, lam_final=None):
        """The adjoint's objective for len(dts) steps with the given dt."""
        J = ctypes.c_double()
        d = np.ascontiguousarray(dts, dtype=np.float64)
        lam = None if lam_final is None else np.ascontiguousarray(lam_final, dtype=np.float64)
        _check(self.lib.harm_run_fixed_dt(self._h, _dp(d), len(d), float(w_mass), float(w_em),
                                          None if lam is None else _dp(lam), ctypes.byref(J)), "harm_run_fixed_dt")
        return J.value

    def get_fluxes(self):
        f1 = np.zeros((self.n1m, self.n2m, NPR))
        f2 = np.zeros((self.n1m, self.n2m, NPR))
        _check(self.lib.harm_get_fluxes(self._h, _dp(f1), _dp(f2)), "harm_get_fluxes")
        return f1, f2


def measure_fp64_peak():
    """The device's FP64 instruction rates: {dadd, dmul, dfma} per second."""
    out = np.zeros(3)
    _check(load_library().harm_measure_fp64_peak(_dp(out)), "harm_measure_fp64_peak")
    return dict(zip(("dadd", "dmul", "dfma"), out.tolist()))


def pinned_empty(shape, dtype=np.float64):
    """A page-locked host array (allocated through torch), for fast
    host<->device copies of the reference-layout state."""
    import torch
    t = torch.empty(tuple(shape), dtype={np.float64: torch.float64, np.int32: torch.int32}[np.dtype(dtype).type],
                    pin_memory=True)
    return t.numpy()


class Ensemble:
    """Several HarmGPU contexts advanced together: each ensemble step is one
    CUDA graph launch holding every member's step as an independent branch
    (harm_ensemble_create); steps_per_launch > 1 unrolls steps into it."""

    def __init__(self, members, steps_per_launch=1, stream=None):
        self.lib = load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        h = ctypes.c_void_p()
        _check(self.lib.harm_ensemble_create(arr, len(self.members), int(steps_per_launch),
                                             ctypes.c_void_p(stream or 0), ctypes.byref(h)), "harm_ensemble_create")
        self._h = h
        self.steps_per_launch = int(steps_per_launch)

    def step(self, nsteps):
        _check(self.lib.harm_ensemble_step(self._h, int(nsteps)), "harm_ensemble_step")

    def sync(self, raise_on_fail=True):
        st = (_Status * len(self.members))()
        rc = self.lib.harm_ensemble_sync(self._h, st)
        out = [dict(fail_code=s.fail_code, fail_i=s.fail_i, fail_j=s.fail_j, fixups=s.fixups, realnstep=s.realnstep,
                    t=s.t, dt=s.dt, newton_iters=s.newton_iters, deferred=s.deferred, fail_step=s.fail_step)
               for s in st]
        if rc == 6 and raise_on_fail:
            bad = [k for k, s in enumerate(out) if s["fail_code"]]
            raise HarmError(rc, f"ensemble members {bad} failed")
        if rc not in (0, 6):
            raise HarmError(rc, "harm_ensemble_sync")
        return out

    def close(self):
        if getattr(self, "_h", None):
            self.lib.harm_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def torus_dump_coords(params):
    """(header dict, coords [n1m, n2m, 4]) of the torus grid for write_dump()."""
    lib = load_library()
    h = _DumpHeader()
    co = np.zeros((params.n1 + 2 * NG, params.n2 + 2 * NG, 4))
    _check(lib.harm_torus_dump_coords(ctypes.byref(params), ctypes.byref(h), _dp(co)), "harm_torus_dump_coords")
    return {k: getattr(h, k) for k, _ in _DumpHeader._fields_}, co


def dipole_params(n1=512, n2=256, **kw):
    """The force-free aligned rotator's parameters (include/harm_setup.h)
    with overrides."""
    lib = load_library()
    p = _DipoleParams()
    lib.harm_dipole_default_params(ctypes.byref(p))
    p.n1, p.n2 = n1, n2
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def dipole_geometry(params):
    """set_grid() for the dipole grid (defcoord 6, flat space): dict of gcov,
    gcon, gdet, conn, floors and the grid scalars (startx1, startx2, dx1,
    dx2, Rin, Rout)."""
    lib = load_library()
    n1m, n2m = params.n1 + 2 * NG, params.n2 + 2 * NG
    g = dict(gcov=np.zeros((n1m, n2m, 4, 4, 4)), gcon=np.zeros((n1m, n2m, 4, 4, 4)), gdet=np.zeros((n1m, n2m, 4)),
             conn=np.zeros((n1m, n2m, 4, 4, 4)), floors=np.zeros((n1m, n2m, 2)))
    grid = np.zeros(6)
    _check(lib.harm_dipole_geometry(ctypes.byref(params), _dp(g["gcov"]), _dp(g["gcon"]), _dp(g["gdet"]),
                                    _dp(g["conn"]), _dp(g["floors"]), _dp(grid)), "harm_dipole_geometry")
    g.update(startx1=grid[0], startx2=grid[1], dx1=grid[2], dx2=grid[3], Rin=grid[4], Rout=grid[5])
    return g


def dipole_init(params, geom):
    """init() for the dipole: every zone's primitives, ghosts included
    (the state still to be bounded)."""
    lib = load_library()
    n1m, n2m = params.n1 + 2 * NG, params.n2 + 2 * NG
    p = np.zeros((n1m, n2m, NPR))
    _check(lib.harm_dipole_init(ctypes.byref(params), _dp(geom["gcov"]), _dp(geom["gcon"]), _dp(geom["gdet"]),
                                _dp(p)), "harm_dipole_init")
    return p


def dipole_context(n1=512, n2=256, *, lim=LIM_MC, fluxmethod=FLUX_LAXF, cour=0.8, precision=PREC_FP64, tf=1.0e30,
                   stream=None, currents=False, **dipole_kw):
    """Builds the force-free aligned rotator on the host (MC + LAXF, the
    reference's force-free defaults) and returns (HarmGPU, geometry, initial
    prims) with the state uploaded, bounded and t=0, dt=1e-5 set."""
    par = dipole_params(n1, n2, **dipole_kw)
    geom = dipole_geometry(par)
    p0 = dipole_init(par, geom)
    h = HarmGPU(n1, n2, geom["dx1"], geom["dx2"], lim=lim, fluxmethod=fluxmethod, cour=cour, gam=par.gam,
                gammamax=par.gammamax, precision=precision, tf=tf, stream=stream, eom=EOM_FFDE, bc=BC_STAR,
                omegastar=par.omegastar, currents=currents)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p0)
    h.bound_prims()
    h.set_time(0.0, 1.0e-5, 0)
    return h, geom, p0


def torus_context(n1=128, n2=128, *, lim=LIM_MC, fluxmethod=FLUX_HLL, cour=0.8, precision=PREC_FP64, tf=1.0e30,
                  stream=None, currents=False, tryagain=False, fluxadjust=0, **torus_kw):
    """Builds the benchmark torus on the host and returns (HarmGPU, geometry,
    initial prims) with the state uploaded, bounded and t=0, dt=1e-5 set as
    init_defglobal() leaves them (initbase.c:158)."""
    par = torus_params(n1, n2, **torus_kw)
    geom = torus_geometry(par)
    p0 = torus_init(par, geom)
    h = HarmGPU(n1, n2, geom["dx1"], geom["dx2"], lim=lim, fluxmethod=fluxmethod, cour=cour, gam=par.gam,
                gammamax=par.gammamax, precision=precision, tf=tf, stream=stream, currents=currents,
                tryagain=tryagain, fluxadjust=fluxadjust)
    h.upload_geometry(geom["gcov"], geom["gcon"], geom["gdet"], geom["conn"], geom["floors"])
    h.set_prims(p0)
    h.bound_prims()
    h.set_time(0.0, 1.0e-5, 0)  # with currents, also their t = 0 evaluation
    return h, geom, p0
