"""Tile-shape autotuner for the step's kernels.

The block shape of k_update (at most 128 threads, it is register-bound at
three blocks per SM) and of the small stencil / boundary / check-solution
kernels changes how a grid of a given size fills the 148 SMs and how many
partial tiles its edges leave.  ``tune`` measures candidate shapes on a
context with ``harm_profile_step`` (per-kernel device time of one step
outside the graph, best of ``reps``), first the k_update shape with the
default small shape, then the small shape with the chosen k_update shape,
and leaves the context set to the winners.  Measuring advances the
context's state by the profiled steps; tune a scratch context, or restore
the state afterwards (``torus_context`` / ``set_prims``).
"""
# k_update's width must be even (its TMA box starts on an even column)
UPDATE_CANDIDATES = ((32, 4), (64, 2), (128, 1), (16, 8), (32, 2))
SMALL_CANDIDATES = ((32, 4), (32, 8), (64, 4), (128, 2), (64, 2))
SMALL_KERNELS = ("k_bsqflags", "k_emf", "k_bound", "k_poledeath", "k_gammacheck", "k_checksol",
                 "k_fixup_compute", "k_bound_fix")

_cache = {}


def _measure(h, reps, names):
    best = None
    for _ in range(reps):
        prof = h.profile_step()
        ms = sum(prof[k][0] for k in names if k in prof)
        best = ms if best is None else min(best, ms)
    return best


def tune(h, reps=3, key=None):
    """Picks and sets the k_update and small-kernel shapes for context h;
    returns (update, small, table of measured ms).  With `key`, the result
    is remembered and reused by ``apply``."""
    if key is not None and key in _cache:
        up, sm = _cache[key]
        h.set_tiles(up, sm)
        return up, sm, {}
    table = {}
    default_small = SMALL_CANDIDATES[0]
    for up in UPDATE_CANDIDATES:
        h.set_tiles(up, default_small)
        table[("update",) + up] = _measure(h, reps, ("k_update",))
    best_up = min(UPDATE_CANDIDATES, key=lambda u: table[("update",) + u])
    for sm in SMALL_CANDIDATES:
        h.set_tiles(best_up, sm)
        table[("small",) + sm] = _measure(h, reps, SMALL_KERNELS)
    best_sm = min(SMALL_CANDIDATES, key=lambda s: table[("small",) + s])
    h.set_tiles(best_up, best_sm)
    if key is not None:
        _cache[key] = (best_up, best_sm)
    return best_up, best_sm, table


def apply(h, key):
    """Sets a remembered result for `key`; False if none was tuned."""
    if key not in _cache:
        return False
    h.set_tiles(*_cache[key])
    return True
