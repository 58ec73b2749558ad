#!/usr/bin/env python3
"""Build recipe for the reference oracle (test infrastructure only).

Compiles the reference HARM sources *where they lie* (read from the reference
tree given by ``--src``) into a shared library under ``oracle/_ref/``.  The
sources are copied to a scratch build directory inside ``oracle/_ref/build/``,
a fixed list of build patches is applied there (never to the reference tree),
and the result is linked together with ``oracle/ref_harness.c`` (the probe API
the tests call through ctypes).  Nothing produced here is committed
(``oracle/_ref/`` is git-ignored) and nothing here is shipped by the product.

Grid size (N1, N2), the physics mode and the metric are compile-time constants
in the reference (global.h:126-127, global.h:202, metric.h:11), so each
problem/size pair is its own library: ``libharmref_<problem>_<N1>x<N2>.so``.

Build patches (each one asserted to apply exactly):
  1. mympi.h:15          USEMPI 1 -> 0            (no MPI here; serial oracle)
  2. global.h:202        EOMTYPE per problem      (EOMGRMHD torus, EOMFFDE dipole)
  3. metric.h:11         MCOORD per problem       (KSCOORDS torus, SPCMINKMETRIC dipole)
  4. global.h:126-127    N1, N2 per build
  5. torus: init.fishmon.c -> init.c, bounds.fishmon.c -> bounds.c;
     dipole: init.ns.c -> init.c, bounds.ns.c -> bounds.c
  6. gcc >= 10 needs -fcommon (tentative definitions in defs.h)
  7. dudp_calc.c, utoprim_{1d,2d,5d2}_final.c are left out (gcc rejects their
     block-scope static prototypes); they are only reached through the
     UTOPRIMTRYAGAIN chain, which patch 10 disables, so ref_harness.c gives
     them stubs that fail loudly if ever called.
  8. init_postfield() and cot() shims (init.fishmon.c predates the former,
     metric.c:1444 comments out the latter) live in ref_harness.c.
  9. init_mpi.c:2341-2418 logging: va_copy before every vfprintf (the
     reference re-uses one va_list, which is undefined behaviour and crashed).
 10. global.h:213 UTOPRIMTRYAGAIN 1 -> 0, global.h:34 MAILWHENDONE 1 -> 0,
     global.h:24 PRODUCTION 0 -> 1 (progress printing only).
 11. utoprim_2d.c:669 the Newton cycle-break factor rand()/RAND_MAX is
     replaced by hr_cycle_break_uniform(x[0], x[1], n_iter), a counter-based
     hash of the iterate (same function as the GPU kernel and the C
     restatement use), so that the factor no longer depends on a serial
     global RNG stream.
 12. init.fishmon.c init_grid()/init_global(), dump.c dump() and fail.c
     fail() are renamed; ref_harness.c wraps the first two to apply the
     benchmark knobs (defcoord 0, Rin = 0.98 r_h, MC/PARA, HLL/LAXF, RK2,
     courant, floors), turns dump files off, and records the code and zone
     of the first fail() call before calling the original.
 13. compiled -O2 -ffp-contract=off -fno-fast-math so that no FMA
     contraction changes the FP64 rounding.

The "torusfa" problem is the torus with the per-zone HLL/LAXF switch of
the benchmark's larger configurations: global.h:292 FLUXADJUST FLUXFIXED ->
FLUXBSQORHOANDU (the alternative line 293 carries), so get_bsqflags sets
pflag[FLAGREALFLUX] (fixup.c:1284-1290) and choose_flux follows it
(step_ch.c:703-738).

The "torusta" problem is the torus with the UTOPRIMTRYAGAIN chain on
(step_ch.c:608-626), the build that pins the retry chain.  It differs from
"torus" in three patches:
  7'. dudp_calc.c and utoprim_{1d,2d,5d2}_final.c are built: their
      block-scope static prototypes (and u2p_util.c's, which the last two
      include) are moved to file scope, where gcc accepts them.
 10'. UTOPRIMTRYAGAIN stays 1.
 11'. the same cycle-break replacement in the three 1D Newton solvers
      (utoprim_1d.c:559, utoprim_1d_opt.c:618, utoprim_1d_final.c:580):
      hr_cycle_break_uniform(x[0], 0.0, n_iter).
"""
import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# reference file list of the default build (maketail.harm.inc:1-9), minus main.c
# (the harness is the driver) and the four files of patch 7.
BASE_SRCS = """bounds.c boundsint.c coord.c diag.c dudp_calc_3vel.c dump.c dump_ener.c
fixup.c gaussj.c image.c initbase.c init.c interp.c lubksb.c ludcmp.c metric.c mnewt.c
nrutil.c phys.c ranc.c restart.c set_arrays.c set_grid.c step_ch.c tensor.c utoprim.c
utoprim_2d.c utoprim_1d.c utoprim_1d_opt.c vchar.c transforms.c fail.c utoprim_ldz.c
init_mpi.c boundmpi.c boundmpiint.c sources.c phys.ffde.c advance.c reconstructeno.c""".split()

# patch 7': the files of the retry chain that gcc rejects as they are
TRYAGAIN_SRCS = ["dudp_calc.c", "utoprim_1d_final.c", "utoprim_2d_final.c", "utoprim_5d2_final.c"]

PROBLEMS = {
    # Fishbone-Moncrief torus in modified Kerr-Schild coordinates (GRMHD).
    "torus": dict(eom="EOMGRMHD", mcoord="KSCOORDS", init="init.fishmon.c", bounds="bounds.fishmon.c", defs=[]),
    # the same with the UTOPRIMTRYAGAIN retry chain of inversions on
    "torusta": dict(eom="EOMGRMHD", mcoord="KSCOORDS", init="init.fishmon.c", bounds="bounds.fishmon.c",
                    defs=["-DHR_TRYAGAIN"], tryagain=True),
    # the torus with the per-zone HLL/LAXF switch: FLUXADJUST FLUXBSQORHOANDU
    # (the alternative global.h:293 keeps commented out), HYDROFLUXADJUSTONLY 1
    "torusfa": dict(eom="EOMGRMHD", mcoord="KSCOORDS", init="init.fishmon.c", bounds="bounds.fishmon.c", defs=[],
                    fluxadjust=True),
    # Force-free aligned rotator (dipole field, rotating stellar surface) in
    # flat space, spherical polar log-r coordinates (FFDE).
    "dipole": dict(eom="EOMFFDE", mcoord="SPCMINKMETRIC", init="init.ns.c", bounds="bounds.ns.c",
                   defs=["-DHR_PROBLEM_DIPOLE"]),
}

CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fcommon", "-fPIC", "-w", "-std=gnu99"]


def sub1(text, pattern, repl, fname, count=1, regex=False):
    """Replace exactly `count` occurrences, failing loudly otherwise."""
    if regex:
        new, n = re.subn(pattern, repl, text)
    else:
        n = text.count(pattern)
        new = text.replace(pattern, repl)
    if n != count:
        raise SystemExit(f"patch failed in {fname}: expected {count} match(es) of {pattern!r}, got {n}")
    return new


def patch_tree(bdir, problem, n1, n2):
    prob = PROBLEMS[problem]

    def edit(fname, fn):
        path = os.path.join(bdir, fname)
        with open(path, "r", encoding="latin-1") as f:
            txt = f.read()
        txt = fn(txt, fname)
        with open(path, "w", encoding="latin-1") as f:
            f.write(txt)

    edit("mympi.h", lambda t, f: sub1(t, "#define USEMPI 1", "#define USEMPI 0", f))

    def g(t, f):
        t = sub1(t, r"#define N1\s+64", f"#define N1 {n1}", f, regex=True)
        t = sub1(t, r"#define N2\s+64", f"#define N2 {n2}", f, regex=True)
        t = sub1(t, "#define EOMTYPE EOMFFDE", f"#define EOMTYPE {prob['eom']}", f)
        if not prob.get("tryagain"):
            t = sub1(t, "#define UTOPRIMTRYAGAIN 1", "#define UTOPRIMTRYAGAIN 0", f)
        if prob.get("fluxadjust"):
            t = sub1(t, "#define FLUXADJUST FLUXFIXED", "#define FLUXADJUST FLUXBSQORHOANDU", f)
        t = sub1(t, "#define MAILWHENDONE 1", "#define MAILWHENDONE 0", f)
        t = sub1(t, "#define PRODUCTION 0", "#define PRODUCTION 1", f)
        return t
    edit("global.h", g)
    edit("metric.h", lambda t, f: sub1(t, "#define MCOORD CYLMINKMETRIC", f"#define MCOORD {prob['mcoord']}", f))

    shutil.copyfile(os.path.join(bdir, prob["init"]), os.path.join(bdir, "init.c"))
    shutil.copyfile(os.path.join(bdir, prob["bounds"]), os.path.join(bdir, "bounds.c"))

    def ini(t, f):
        t = sub1(t, "int init_grid(void)", "int hr_orig_init_grid(void)", f)
        t = sub1(t, "int init_global(void)", "int hr_orig_init_global(void)", f)
        return t
    edit("init.c", ini)
    edit("dump.c", lambda t, f: sub1(t, "int dump(long dump_cnt)\n", "int hr_orig_dump(long dump_cnt)\n", f))
    edit("fail.c", lambda t, f: sub1(t, "int fail(int fail_type)\n", "int hr_orig_fail(int fail_type)\n", f))

    def logfix(t, f):
        # every vfprintf(X, format, arglist) consumes a private copy of the list
        return sub1(t, r"vfprintf \((\w+), format, arglist\);",
                    r"{ va_list hr_ac; va_copy(hr_ac, arglist); vfprintf (\1, format, hr_ac); va_end(hr_ac); }",
                    f, count=8, regex=True)
    edit("init_mpi.c", logfix)

    def u2d(t, f):
        t = sub1(t, "randtmp = ( (1.*rand())/(1.*RAND_MAX) );",
                 "randtmp = hr_cycle_break_uniform(x[0], x[1], n_iter);", f)
        t = sub1(t, '#include "utoprim_2d.h"',
                 '#include "utoprim_2d.h"\nextern FTYPE hr_cycle_break_uniform(FTYPE x0, FTYPE x1, int n_iter);', f)
        return t
    edit("utoprim_2d.c", u2d)
    if not prob.get("tryagain"):
        return

    proto = re.compile(r"^[ \t]+(static\s+(?:void|int|FTYPE)\s+\w+\s*\([^;{]*\)\s*;)[ \t]*$", re.M)

    def hoist(anchor):
        # block-scope static prototypes -> file scope, right after `anchor`
        def fn(t, f):
            found = proto.findall(t)
            if not found:
                raise SystemExit(f"patch failed in {f}: no block-scope static prototypes")
            t = proto.sub("", t)
            decl = "\n".join(dict.fromkeys(found))
            return sub1(t, anchor, anchor + "\n" + decl + "\n", f)
        return fn
    edit("dudp_calc.c", hoist('#include "decs.h"'))
    edit("u2p_util.c", hoist('//#include "u2p_defs.h"'))
    edit("utoprim_1d_final.c", hoist("#define NEWT_DIM 1"))
    edit("utoprim_2d_final.c", hoist("#define NEWT_DIM 2"))
    edit("utoprim_5d2_final.c", hoist("#define NEWT_DIM 5"))

    def u1d(t, f):
        t = sub1(t, "randtmp = ( (1.*rand())/(1.*RAND_MAX) );", "randtmp = hr_cycle_break_uniform(x[0], 0.0, n_iter);", f)
        return "extern double hr_cycle_break_uniform(double x0, double x1, int n_iter);\n" + t
    for name in ("utoprim_1d.c", "utoprim_1d_opt.c", "utoprim_1d_final.c"):
        edit(name, u1d)


def build(src, problem, n1, n2, jobs, force=False):
    tag = f"{problem}_{n1}x{n2}"
    lib = os.path.join(OUT, f"libharmref_{tag}.so")
    harness = os.path.join(HERE, "ref_harness.c")
    if (not force and os.path.exists(lib)
            and os.path.getmtime(lib) >= os.path.getmtime(harness)
            and os.path.getmtime(lib) >= os.path.getmtime(__file__)):
        return lib
    bdir = os.path.join(OUT, "build", tag)
    if os.path.isdir(bdir):
        shutil.rmtree(bdir)
    os.makedirs(bdir)
    for name in os.listdir(src):
        if name.endswith((".c", ".h")):
            shutil.copyfile(os.path.join(src, name), os.path.join(bdir, name))
    patch_tree(bdir, problem, n1, n2)
    shutil.copyfile(harness, os.path.join(bdir, "hr_harness.c"))
    srcs = BASE_SRCS + (TRYAGAIN_SRCS if PROBLEMS[problem].get("tryagain") else []) + ["hr_harness.c"]

    def cc(name):
        obj = os.path.join(bdir, name[:-2] + ".o")
        cmd = ["gcc"] + CFLAGS + PROBLEMS[problem]["defs"] + ["-c", os.path.join(bdir, name), "-o", obj]
        r = subprocess.run(cmd, cwd=bdir, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {name}\n{r.stderr[-3000:]}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(cc, srcs))
    tmp = lib + ".tmp"
    r = subprocess.run(["gcc", "-shared", "-Wl,-Bsymbolic", "-o", tmp] + objs + ["-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed\n" + r.stderr[-3000:])
    os.replace(tmp, lib)
    return lib


NATIVE_CFLAGS = ["-O3", "-march=native", "-ffp-contract=off", "-fno-fast-math", "-fcommon", "-fPIC", "-w",
                 "-std=gnu99"]


def _host_cpu():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def build_native(problem, n1, n2, jobs):
    """The CPU baseline: the already patched scratch tree of a build
    (oracle/_ref/build/<problem>_<N1>x<N2>, which the parity build left
    behind) compiled -O3 -march=native -ffp-contract=off for the host this
    runs on, into oracle/_ref/native/.  Rebuilt when the host CPU model
    differs from the one the library was built for.  Needs no reference
    tree (it may run where only the scratch tree was carried)."""
    tag = f"{problem}_{n1}x{n2}"
    bdir = os.path.join(OUT, "build", tag)
    if not os.path.isdir(bdir):
        raise SystemExit(f"no scratch tree {bdir}: run the parity build of {tag} first")
    ndir = os.path.join(OUT, "native")
    os.makedirs(ndir, exist_ok=True)
    lib = os.path.join(ndir, f"libharmref_{tag}.so")
    stamp = lib + ".cpu"
    cpu = _host_cpu()
    if os.path.exists(lib) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read() == cpu:
                return lib
    odir = os.path.join(ndir, "obj_" + tag)
    os.makedirs(odir, exist_ok=True)
    srcs = BASE_SRCS + (TRYAGAIN_SRCS if PROBLEMS[problem].get("tryagain") else []) + ["hr_harness.c"]

    def cc(name):
        obj = os.path.join(odir, name[:-2] + ".o")
        cmd = ["gcc"] + NATIVE_CFLAGS + PROBLEMS[problem]["defs"] + ["-c", os.path.join(bdir, name), "-o", obj]
        r = subprocess.run(cmd, cwd=bdir, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {name}\n{r.stderr[-3000:]}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(cc, srcs))
    tmp = lib + ".tmp%d" % os.getpid()
    r = subprocess.run(["gcc", "-shared", "-Wl,-Bsymbolic", "-o", tmp] + objs + ["-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed\n" + r.stderr[-3000:])
    os.replace(tmp, lib)
    with open(stamp, "w") as f:
        f.write(cpu)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=os.environ.get("HARM_REFERENCE_SRC", "/root/reference"),
                    help="the reference source tree (default: $HARM_REFERENCE_SRC)")
    ap.add_argument("--problem", default="torus", choices=sorted(PROBLEMS))
    ap.add_argument("--sizes", default="16x16,32x32,64x64,128x128")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--native", action="store_true",
                    help="compile the existing scratch tree -O3 -march=native for this host (the CPU baseline)")
    a = ap.parse_args()
    if a.native:
        for sz in a.sizes.split(","):
            n1, n2 = (int(v) for v in sz.split("x"))
            print(build_native(a.problem, n1, n2, a.jobs))
        return 0
    if not os.path.isdir(a.src):
        print(f"reference tree {a.src} not present; nothing built", file=sys.stderr)
        return 0
    for s in a.sizes.split(","):
        n1, n2 = (int(v) for v in s.split("x"))
        print(build(a.src, a.problem, n1, n2, a.jobs, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
