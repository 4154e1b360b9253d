"""Failure detection on the GPU, with no fault, trap or hang.

* A NaN in gamma, passed on the host through ws_run_algorithm (the
  RunWaveSimAlgorithmMex argument list), makes the residual energy non-finite;
  the device stop rule ends the loop and the call returns WS_ERR_DIVERGED.
  (The reference would run on to max_iterations; this is an addition.)
* An Inf in the source does the same through WaveSim.exec.
* The bounded waits of the TMA-pipelined outer pass: with a wait limit of one
  clock (ws_solver_set_wait_limit; such a short bound polls the barrier
  without suspending) the tile loads cannot arrive in time, the blocks give up, wait for their copies in flight with the default bound, set
  the error flag and return; the solve returns WS_ERR_CUDA ("timed out").
  The CUDA context stays usable: with the default limit restored, the same
  solver solves again and reproduces the result of a normal solve.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mex_call(sim, gamma, source):
    from wavesim_b200 import _lib
    s, blocks, keep = sim.source_blocks(source)
    maxit = 64
    E = np.zeros(int(np.prod(sim.N)), np.complex64)
    hist = np.zeros(maxit + len(sim.wiggles) + 1)
    n = C.c_int64()
    g = np.asfortranarray(gamma.astype(np.complex64))
    rc = _lib.lib.ws_run_algorithm(
        (C.c_int64 * 4)(*[int(v) for v in sim.N]), g.ctypes.data, len(sim.wiggles), sim._wiggle_structs(),
        len(s.values), blocks, C.c_float(sim.epsilon), _lib.ws_complex(sim.k02e.real, sim.k02e.imag), sim._roi8(),
        maxit, 1e-12, b"NoCallback", 50, _lib.CALLBACK(), None, _lib.WS_HOST, E.ctypes.data,
        hist.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n))
    return rc, int(n.value), hist[:n.value]


def test_nan_in_gamma_returns_diverged(gpu):
    import wavesim_b200 as ws
    from wavesim_b200 import _lib
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-12}
    sim = ws.WaveSim(1.0 + 0.1 * np.random.default_rng(1).random((96, 96)), opt)
    src = ws.Source(1.0, [48, 48])
    rc, n_ok, _ = _mex_call(sim, sim.gamma, src)
    assert rc == _lib.WS_OK
    g = np.array(sim.gamma)
    g[60, 60, 0] = np.nan
    rc, n_it, hist = _mex_call(sim, g, src)
    assert rc == _lib.WS_ERR_DIVERGED, (rc, _lib.lib.ws_last_error())
    assert b"finite" in _lib.lib.ws_last_error() or b"diverged" in _lib.lib.ws_last_error().lower()
    assert n_it <= n_ok and not np.all(np.isfinite(hist))
    _lib.lib.ws_run_algorithm_release()


def test_inf_in_source_returns_diverged(gpu):
    import wavesim_b200 as ws
    from wavesim_b200 import WaveSimError, _lib
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8, 8], "energy_threshold": 1e-3}
    sim = ws.WaveSim(np.full((48, 48, 48), 1.33), opt)
    val = np.ones((48, 48), complex)
    val[3, 7] = np.inf
    with pytest.raises(WaveSimError) as e:
        sim.exec(ws.Source(val, [1, 1, 1]))
    assert e.value.status == _lib.WS_ERR_DIVERGED
    # the solver is still usable
    E, st = sim.exec(ws.Source(np.ones((48, 48)), [1, 1, 1]))
    assert np.all(np.isfinite(E)) and st.converged
    sim.close()


def test_tma_wait_limit_runs_out_and_reports(gpu):
    import wavesim_b200 as ws
    from wavesim_b200 import WaveSimError, _lib
    rng = np.random.default_rng(3)
    # 128^3 grid: K2 is the TMA-pipelined pencil kernel (z = 128)
    n = np.where(rng.random((96, 96, 96)) < 0.1, 1.5, 1.33)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16, 16], "energy_threshold": 1e-99,
           "max_iterations": 16}
    sim = ws.WaveSim(n, opt)
    src = ws.Source(np.ones((96, 96)), [1, 1, 1])
    E0, st0 = sim.exec(src)
    h = sim.solver()
    for use_graph in (True, False):
        sim.use_graph = use_graph
        _lib.check(_lib.lib.ws_solver_set_wait_limit(h, 1))
        with pytest.raises(WaveSimError) as e:
            sim.exec(src)
        assert e.value.status == _lib.WS_ERR_CUDA
        assert b"timed out" in _lib.lib.ws_last_error()
        _lib.check(_lib.lib.ws_solver_set_wait_limit(h, 0))
        E1, st1 = sim.exec(src)
        assert st1.it == st0.it
        assert np.array_equal(E1, E0)
    sim.close()
