"""Builds the reference's own program (its main.c run loop, init(), diag(),
the boundary and fixup code, compiled from the patched scratch tree that
oracle/build_ref.py leaves in oracle/_ref/build) twice: once as it is, with
its CPU step_ch(), and once with step_ch() replaced by the B200 shim
(harm_ramt_b200/shim/step_ch_b200.c) linked against libharm_b200.so.
Test infrastructure for the drop-in tests."""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_ref  # noqa: E402

SHIM = os.path.join(ROOT, "harm_ramt_b200", "shim", "step_ch_b200.c")
NG = 3


def scratch_tree(tag="torus_32x32"):
    d = os.path.join(ROOT, "oracle", "_ref", "build", tag)
    return d if os.path.isfile(os.path.join(d, "main.c")) and os.path.isfile(os.path.join(d, "hr_harness.c")) else None


def build_program(tag, with_shim, outdir):
    """The reference's program from the scratch tree of build `tag`; with
    the shim in place of step_ch.c's step_ch() when with_shim.  Returns the
    executable's path."""
    src = scratch_tree(tag)
    problem = tag.rsplit("_", 1)[0]
    wdir = os.path.join(outdir, "shim" if with_shim else "cpu")
    shutil.copytree(src, wdir, ignore=shutil.ignore_patterns("*.o"))
    srcs = list(build_ref.BASE_SRCS) + ["main.c", "hr_harness.c"]
    if build_ref.PROBLEMS[problem].get("tryagain"):
        srcs += build_ref.TRYAGAIN_SRCS
    inc = []
    libs = ["-lm"]
    if with_shim:
        path = os.path.join(wdir, "step_ch.c")
        with open(path, encoding="latin-1") as f:
            txt = f.read()
        assert txt.count("int step_ch()\n{") == 1
        with open(path, "w", encoding="latin-1") as f:
            f.write(txt.replace("int step_ch()\n{", "int hr_reference_step_ch()\n{"))
        shutil.copyfile(SHIM, os.path.join(wdir, "step_ch_b200.c"))
        srcs.append("step_ch_b200.c")
        inc = ["-I", os.path.join(ROOT, "include")]
        libdir = os.path.join(ROOT, "harm_ramt_b200")
        libs = ["-L", libdir, "-lharm_b200", "-Wl,-rpath," + libdir] + libs
    objs = []
    for name in srcs:
        obj = os.path.join(wdir, name[:-2] + ".o")
        r = subprocess.run(["gcc"] + build_ref.CFLAGS + build_ref.PROBLEMS[problem]["defs"] + inc +
                           ["-c", os.path.join(wdir, name), "-o", obj], cwd=wdir, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {name}\n{r.stderr[-3000:]}")
        objs.append(obj)
    exe = os.path.join(wdir, "harm")
    r = subprocess.run(["gcc", "-o", exe] + objs + libs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed\n" + r.stderr[-3000:])
    return exe


def run_program(exe, tf, lim=3, flux=1, timeout=900):
    """Runs the program in a fresh work directory to end time tf; returns
    (prims [n1m, n2m, 8], pflag [n1m, n2m, 5], t, dt, realnstep) of its
    final state."""
    work = tempfile.mkdtemp(prefix="harm_main_")
    state = os.path.join(work, "final.bin")
    env = dict(os.environ, HR_TF=repr(float(tf)), HR_LIM=str(lim), HR_FLUX=str(flux), HR_FINAL_STATE=state)
    r = subprocess.run([exe], cwd=work, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0 or not os.path.exists(state):
        raise RuntimeError(f"{exe} failed (rc={r.returncode}): {r.stderr[-2000:]}")
    raw = np.fromfile(state, dtype=np.uint8)
    shutil.rmtree(work, ignore_errors=True)
    return raw


def split_state(raw, n1, n2):
    n1m, n2m = n1 + 2 * NG, n2 + 2 * NG
    np_ = n1m * n2m * 8 * 8
    nf = n1m * n2m * 5 * 4
    p = raw[:np_].view(np.float64).reshape(n1m, n2m, 8)
    f = raw[np_:np_ + nf].view(np.int32).reshape(n1m, n2m, 5)
    t, dt, nst = raw[np_ + nf:np_ + nf + 24].view(np.float64)
    return p, f, float(t), float(dt), int(nst)
