"""ws_run_algorithm (the RunWaveSimAlgorithmMex argument list) keeps its
device buffers between calls on the same grid and uploads only the medium:
consecutive calls on different media, sources and roi give the same fields
as the solver API, and after ws_run_algorithm_release the next call starts
afresh."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(sim, source, maxit=100000):
    from wavesim_b200 import _lib
    s, blocks, keep = sim.source_blocks(source)
    E = np.zeros(int(np.prod(sim.N)), np.complex64)
    hist = np.zeros(maxit + len(sim.wiggles) + 1)
    n = C.c_int64()
    gamma = np.asfortranarray(sim.gamma)
    _lib.check(_lib.lib.ws_run_algorithm(
        (C.c_int64 * 4)(*[int(v) for v in sim.N]), gamma.ctypes.data, len(sim.wiggles),
        sim._wiggle_structs(), len(s.values), blocks, C.c_float(sim.epsilon),
        _lib.ws_complex(sim.k02e.real, sim.k02e.imag), sim._roi8(), maxit, sim.energy_threshold, b"NoCallback",
        sim.callback_interval, _lib.CALLBACK(), None, _lib.WS_HOST, E.ctypes.data,
        hist.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)))
    return E, int(n.value)


def test_consecutive_calls_reuse_buffers(gpu):
    import wavesim_b200 as ws
    from wavesim_b200 import _lib
    from wavesim_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(5)
    cases = []
    for k, (contrast, roi) in enumerate([(0.2, None), (0.3, None), (0.1, [[5, 5], [60, 70]])]):
        n = np.clip(1.0 + contrast * gaussian_random_field((96, 96), 4, rng), 0.8, 1.6)
        opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-3}
        if roi is not None:
            opt["roi"] = roi
        cases.append((ws.WaveSim(n, opt), ws.Source(1.0 + 0.5 * k, [30 + 10 * k, 40])))
    got = [_call(sim, src) for sim, src in cases]
    for (sim, src), (E, n_it) in zip(cases, got):
        Ep, st = sim.exec(src, output="eprime")
        assert n_it == st.it - 1
        assert float(np.linalg.norm(E - np.ravel(Ep, order="F")) / np.linalg.norm(Ep)) < 1e-6
    _lib.lib.ws_run_algorithm_release()
    E2, n2 = _call(*cases[0])
    assert n2 == got[0][1] and float(np.linalg.norm(E2 - got[0][0]) / np.linalg.norm(got[0][0])) < 1e-6
    _lib.lib.ws_run_algorithm_release()
