"""The drop-in claim, run: the reference's own program (main.c's run loop,
init(), diag(), postdt(), the error checks) built with the B200 shim
(harm_ramt_b200/shim/step_ch_b200.c) in place of its step_ch(), against the
same program with the reference's CPU step_ch().  Both run from the
reference's init() to the same end time; the final p (ghost zones
included), the inversion flags, t, dt and realnstep must be equal (IEEE ==).
Skipped where the patched reference tree (oracle/_ref/build) is absent."""
import shutil
import tempfile

import numpy as np
import pytest

import dropin

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lim,flux,tf", [(3, 1, 0.5), (4, 1, 0.5), (4, 0, 0.2)])
def test_reference_program_with_shim_matches_cpu_program(harm, lim, flux, tf):
    if dropin.scratch_tree("torus_32x32") is None or shutil.which("gcc") is None:
        pytest.skip("patched reference tree (oracle/_ref/build) or gcc not present")
    d = tempfile.mkdtemp(prefix="harm_dropin_")
    try:
        cpu = dropin.build_program("torus_32x32", False, d)
        shim = dropin.build_program("torus_32x32", True, d)
        pc, fc, tc, dtc, nc = dropin.split_state(dropin.run_program(cpu, tf, lim, flux), 32, 32)
        pg, fg, tg, dtg, ng = dropin.split_state(dropin.run_program(shim, tf, lim, flux), 32, 32)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    assert nc > 25, nc
    assert (tg, dtg, ng) == (tc, dtc, nc)
    if not np.array_equal(pg, pc):
        bad = np.argwhere(pg != pc)
        raise AssertionError(f"{len(bad)} values differ after {nc} steps, first {bad[:4].tolist()}")
    assert np.array_equal(fg[..., 0], fc[..., 0])
    print(f"\nreference program, lim {lim} flux {flux}: {nc} steps to t={tc} on the device == on the CPU")
