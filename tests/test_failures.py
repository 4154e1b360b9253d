"""Failure detection on the host (no GPU needed): the product rejects what the
reference rejects before any device work.

* a medium with gain (negative imaginary part of n) is refused, as
  Medium.m:37-39 refuses it;
* a source that lies entirely outside the grid warns and returns no field
  (Simulation.m:157-161), without creating a solver;
* bad arguments to the C ABI are refused with WS_ERR_INVALID_ARGUMENT before
  any CUDA call.
"""
import ctypes as C
import warnings

import numpy as np
import pytest


def test_gain_is_rejected_by_the_product():
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8], "energy_threshold": 1e-3}
    n = np.ones((32, 32), complex)
    n[10, 10] = 1.2 - 0.01j
    with pytest.raises(ValueError, match="gain"):
        ws.WaveSim(n, opt)
    n3 = np.ones((16, 16, 16), complex)
    n3[4, 4, 4] = 1.0 - 1e-6j
    with pytest.raises(ValueError, match="gain"):
        ws.WaveSimVector(n3, dict(opt, boundary_widths=[4, 4, 4]))


def test_source_outside_the_grid_warns_and_returns_nothing():
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8], "energy_threshold": 1e-3}
    sim = ws.WaveSim(np.ones((32, 32)), opt)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        E, st = sim.exec(ws.Source(1.0, [500, 500]))
    assert E is None and st.source_energy == 0
    assert any("no source inside the grid" in str(x.message) for x in w)
    assert sim._solver is None  # nothing was set up on a device


def test_c_abi_rejects_bad_arguments_before_any_cuda_call():
    from wavesim_b200 import _lib
    L = _lib.lib
    o = _lib.default_options()
    # null solver handle
    assert L.ws_solver_solve(None, 0, None, 0, C.byref(o), None, 0, None, None, None) == _lib.WS_ERR_INVALID_ARGUMENT
    assert L.ws_solver_set_wait_limit(None, 0) == _lib.WS_ERR_INVALID_ARGUMENT
    # N(4) must be 1 or 3; Nwiggles must be positive
    g = np.zeros(16 * 16, np.complex64)
    h = C.c_void_p()
    wig = (_lib.ws_wiggle * 1)()
    roi = (C.c_int64 * 8)(1, 16, 1, 16, 1, 1, 1, 1)
    rc = L.ws_solver_create((C.c_int64 * 4)(16, 16, 1, 2), g.ctypes.data, 1, wig, C.c_float(3.0),
                            _lib.ws_complex(1, 1), roi, 0, 0, C.byref(h))
    assert rc == _lib.WS_ERR_INVALID_ARGUMENT
    rc = L.ws_solver_create((C.c_int64 * 4)(16, 16, 1, 1), g.ctypes.data, 0, wig, C.c_float(3.0),
                            _lib.ws_complex(1, 1), roi, 0, 0, C.byref(h))
    assert rc == _lib.WS_ERR_INVALID_ARGUMENT
    # roi outside the grid
    rc = L.ws_solver_create((C.c_int64 * 4)(16, 16, 1, 1), g.ctypes.data, 1, wig, C.c_float(3.0),
                            _lib.ws_complex(1, 1), (C.c_int64 * 8)(1, 17, 1, 16, 1, 1, 1, 1), 0, 0, C.byref(h))
    assert rc == _lib.WS_ERR_INVALID_ARGUMENT
    assert L.ws_last_error()
