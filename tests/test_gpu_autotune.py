"""The layout autotuner (ws_solver_autotune, no counterpart in the
reference): after tuning, solves give the same fields and iteration counts,
and the chosen layout is no slower than the heuristic one."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,bw,src", [((96, 80), [16, 16], (1.0, [48, 40])),
                                          ((48, 48, 48), [8, 8, 8], (np.ones((48, 48)), [1, 1, 1]))])
def test_autotune_keeps_results(gpu, shape, bw, src):
    import wavesim_b200 as ws
    from wavesim_b200 import _lib
    from wavesim_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(3)
    n = np.clip(1.0 + 0.2 * gaussian_random_field(shape, 4, rng), 0.9, 1.5)
    sim = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-4})
    source = ws.Source(*src)
    E0, s0 = sim.exec(source)
    tried, before, after = C.c_int(), C.c_float(), C.c_float()
    _lib.check(_lib.lib.ws_solver_autotune(sim.solver(), 8, C.byref(tried), C.byref(before), C.byref(after)))
    assert tried.value >= 2
    assert after.value <= before.value * 1.05 + 1e-3
    E1, s1 = sim.exec(source)
    assert s1.it == s0.it
    assert float(np.linalg.norm(E1 - E0) / np.linalg.norm(E0)) < 1e-5
