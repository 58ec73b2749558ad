"""The C ABI: the shared library loads and exports every entry point that
include/*.h declares; without a CUDA device the step refuses to start
(no CPU fallback) while the host-side set-up still works."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in ("harm_b200.h", "harm_setup.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(harm_\w+)\s*\(", txt, flags=re.M))
    return names


def test_library_exports_every_declared_symbol(harm):
    declared = _declared()
    assert len(declared) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", harm.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s+(harm_\w+)", out))
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    lib = harm.load_library()
    for name in declared:
        assert hasattr(lib, name)


def test_error_strings(harm):
    lib = harm.load_library()
    for code in range(0, 7):
        assert lib.harm_error_string(code)


def test_no_cpu_fallback(harm):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(harm.HarmError) as e:
        harm.HarmGPU(16, 16, 0.1, 0.0625)
    assert e.value.code == 2


def test_invalid_config_rejected(harm):
    with pytest.raises(harm.HarmError):
        harm.HarmGPU(2, 2, 0.1, 0.1)
    with pytest.raises(harm.HarmError):
        harm.HarmGPU(16, 16, 0.1, 0.1, lim=7)


def test_setup_tables_are_symmetric(harm):
    """The step packs g_{mu nu}, g^{mu nu} and Gamma^k_{(lj)} as symmetric;
    the set-up must produce exactly symmetric tables."""
    g = harm.torus_geometry(harm.torus_params(24, 20))
    for k in ("gcov", "gcon"):
        assert np.array_equal(g[k], np.swapaxes(g[k], -1, -2))
    assert np.array_equal(g["conn"], np.swapaxes(g["conn"], -1, -2))
    assert np.all(g["gdet"] > 0)
