"""Layout autotuning with a cache (no counterpart in the reference).

``ws_solver_autotune`` times the kernel layouts a grid supports - fast or
generic kernels, radix schedules of the generic ones, the split step's x
pencils, the TMA pencil's stages, tile shapes - on the loop as it runs and
keeps the fastest.  ``tune`` wraps it with a JSON cache keyed by the kind of
field and the grid size, so that a grid is timed once and later solvers of
the same size take the cached choice (``ws_solver_set_layout``) without
timing anything:

    from wavesim_b200.autotune import tune
    info = tune(sim, cache="layouts.json")    # {"cached": ..., "choice": [...], ...}
"""
from __future__ import annotations

import ctypes as C
import json
import os
import tempfile

from . import _lib

FIELDS = ("inner", "outer", "csize", "ncols", "ty", "sched", "xp")


def cache_key(sim):
    """'scalar:Ny x Nx x Nz' or 'vector:...': what a layout depends on."""
    kind = "vector" if getattr(sim, "vector", False) else "scalar"
    return kind + ":" + "x".join(str(int(v)) for v in sim.N[:3])


def _read(path):
    if not path or not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def _write(path, data):
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=d, suffix=".tmp")
    with os.fdopen(fd, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def get_layout(sim):
    c = (C.c_int32 * 7)()
    _lib.check(_lib.lib.ws_solver_get_layout(sim.solver(), c))
    return list(c)


def set_layout(sim, choice):
    c = (C.c_int32 * 7)(*[int(v) for v in choice])
    _lib.check(_lib.lib.ws_solver_set_layout(sim.solver(), c))


def tune(sim, cache=None, iterations=8):
    """Tunes the layout of `sim`'s solver, or applies the cached choice for
    its grid.  Returns a dict: cached (bool), choice (7 integers, see FIELDS),
    and for a fresh tune the candidates tried and the time of one iteration
    before and after (ms)."""
    key = cache_key(sim)
    data = _read(cache)
    if key in data:
        set_layout(sim, data[key]["choice"])
        return dict(data[key], cached=True)
    tried, before, after = C.c_int(), C.c_float(), C.c_float()
    _lib.check(_lib.lib.ws_solver_autotune(sim.solver(), iterations, C.byref(tried), C.byref(before),
                                           C.byref(after)))
    entry = {"choice": get_layout(sim), "fields": list(FIELDS), "tried": int(tried.value),
             "ms_before": float(before.value), "ms_after": float(after.value)}
    if cache:
        data = _read(cache)  # another process may have written meanwhile
        data[key] = entry
        _write(cache, data)
    return dict(entry, cached=False)
