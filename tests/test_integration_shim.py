"""The reference-side binding, harm_ramt_b200/shim/step_ch_b200.c (the C
shim that replaces the reference's step_ch()): it compiles against the
reference's own headers and include/harm_b200.h, and the reference's whole
program -- its main.c run loop, init(), diag() and the rest, from the patched
scratch tree that oracle/build_ref.py leaves in oracle/_ref/build -- builds
and links with it in place of step_ch.c's step_ch().  The same program with
its own CPU step_ch() runs here; tests/test_gpu_dropin.py runs both and
compares them on a GPU.  Skipped where that scratch tree is absent."""
import os
import shutil
import subprocess
import tempfile

import pytest

import dropin

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _tree():
    t = dropin.scratch_tree("torus_32x32")
    if t is None or shutil.which("gcc") is None:
        pytest.skip("patched reference tree (oracle/_ref/build) or gcc not present")
    return t


def test_shim_compiles_against_reference_headers():
    tree = _tree()
    with open(dropin.SHIM) as f:
        src = f.read()
    assert "harm_create" in src and "harm_step" in src and "int step_ch(void)" in src
    r = subprocess.run(["gcc", "-fsyntax-only", "-fcommon", "-Wall", "-Wno-unused", "-I", os.path.join(ROOT, "include"),
                        "-I", tree, dropin.SHIM], capture_output=True, text=True, cwd=tree)
    own = [line for line in r.stderr.splitlines() if "step_ch_b200.c" in line]
    assert r.returncode == 0, r.stderr[-3000:]
    assert not own, "\n".join(own)


def test_reference_program_builds_with_the_shim_and_runs_without_it():
    _tree()
    d = tempfile.mkdtemp(prefix="harm_dropin_")
    try:
        cpu = dropin.build_program("torus_32x32", False, d)
        shim = dropin.build_program("torus_32x32", True, d)
        assert os.path.exists(shim)
        p, f, t, dt, nstep = dropin.split_state(dropin.run_program(cpu, 0.1), 32, 32)
        # the reference's own loop: t reaches the end time exactly (the last
        # step clamped onto it), 31 steps from dt = 1e-5
        assert t == 0.1 and dt == 0.0 and nstep == 31
        assert (p[3:-3, 3:-3, 0] > 0).all()
    finally:
        shutil.rmtree(d, ignore_errors=True)
