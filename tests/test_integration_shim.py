"""The reference-side binding shown in INTEGRATION.md (the C shim that
replaces step_ch()) compiles against the reference's own headers and this
repository's include/harm_b200.h: gcc -fsyntax-only -Wall in the patched
scratch copy of the reference that oracle/build_ref.py leaves under
oracle/_ref/build (skipped where that build is absent)."""
import os
import re
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REFBUILD = os.path.join(ROOT, "oracle", "_ref", "build", "torus_32x32")


def _shim_source():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as f:
        text = f.read()
    m = re.search(r"## The shim.*?```c\n(.*?)```", text, re.S)
    assert m, "no C block under 'The shim' in INTEGRATION.md"
    return m.group(1)


def test_shim_compiles_against_reference_headers():
    if not os.path.isfile(os.path.join(REFBUILD, "decs.h")) or shutil.which("gcc") is None:
        pytest.skip("patched reference tree (oracle/_ref/build) or gcc not present")
    src = _shim_source()
    assert "harm_create" in src and "harm_step" in src and "int step_ch(void)" in src
    fd, path = tempfile.mkstemp(suffix=".c", prefix="step_ch_b200_")
    with os.fdopen(fd, "w") as f:
        f.write(src)
    try:
        r = subprocess.run(["gcc", "-fsyntax-only", "-fcommon", "-Wall", "-Wno-unused", "-I", os.path.join(ROOT, "include"),
                            "-I", REFBUILD, path], capture_output=True, text=True, cwd=REFBUILD)
    finally:
        os.unlink(path)
    own = [line for line in r.stderr.splitlines() if os.path.basename(path) in line]
    assert r.returncode == 0, r.stderr[-3000:]
    assert not own, "\n".join(own)
