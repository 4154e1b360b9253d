"""The layout autotuner (ws_solver_autotune, no counterpart in the
reference): after tuning, solves give the same fields and iteration counts,
the chosen layout is no slower than the heuristic one, and a cached choice
(wavesim_b200.autotune, ws_solver_get_layout / ws_solver_set_layout) is
applied to a new solver of the same grid without timing anything."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [((96, 80), [16, 16], (1.0, [48, 40])),
         ((48, 48, 48), [8, 8, 8], (np.ones((48, 48)), [1, 1, 1])),
         ((224, 224, 16), [16, 16, 8], (np.ones((224, 224)), [1, 1, 1])),   # split step, x pencils
         ((64, 64, 64), [8, 8, 8], (np.ones((64, 64)), [1, 1, 1]))]         # 80^3: generic, radix schedules


def _sim(ws, shape, bw):
    from wavesim_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(3)
    n = np.clip(1.0 + 0.2 * gaussian_random_field(shape, 4, rng), 0.9, 1.5)
    return ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-4})


@pytest.mark.parametrize("shape,bw,src", CASES)
def test_autotune_keeps_results(gpu, shape, bw, src):
    import wavesim_b200 as ws
    from wavesim_b200 import _lib
    sim = _sim(ws, shape, bw)
    source = ws.Source(*src)
    E0, s0 = sim.exec(source)
    tried, before, after = C.c_int(), C.c_float(), C.c_float()
    _lib.check(_lib.lib.ws_solver_autotune(sim.solver(), 8, C.byref(tried), C.byref(before), C.byref(after)))
    assert tried.value >= 2
    assert after.value <= before.value * 1.05 + 1e-3
    E1, s1 = sim.exec(source)
    assert s1.it == s0.it
    assert float(np.linalg.norm(E1 - E0) / np.linalg.norm(E0)) < 1e-5


def test_autotune_cache(gpu, tmp_path):
    import wavesim_b200 as ws
    from wavesim_b200.autotune import get_layout, tune
    shape, bw, src = CASES[3]
    cache = str(tmp_path / "layouts.json")
    sim = _sim(ws, shape, bw)
    source = ws.Source(*src)
    E0, s0 = sim.exec(source)
    first = tune(sim, cache=cache)
    assert not first["cached"] and first["tried"] >= 2
    sim2 = _sim(ws, shape, bw)
    second = tune(sim2, cache=cache)
    assert second["cached"] and second["choice"] == first["choice"]
    assert get_layout(sim2) == first["choice"]
    E2, s2 = sim2.exec(source)
    assert s2.it == s0.it
    assert float(np.linalg.norm(E2 - E0) / np.linalg.norm(E0)) < 1e-5
    # every radix schedule of the generic kernels gives the same field
    for sched in (1, 2):
        sim3 = _sim(ws, shape, bw)
        from wavesim_b200.autotune import set_layout
        set_layout(sim3, [2, 2, 0, 0, 0, sched, 0])
        E3, s3 = sim3.exec(source)
        assert s3.it == s0.it
        assert float(np.linalg.norm(E3 - E0) / np.linalg.norm(E0)) < 1e-5
