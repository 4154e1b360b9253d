"""PSTD on the GPU (ws_pstd_* through wavesim_b200.PSTD) against the PSTD
restatement in oracle/pstd_oracle.py, and against the GPU MBS solver on a
medium where both reach the same steady state."""
import warnings

import numpy as np
import pytest

from oracle import mbs_oracle as ref
from oracle.pstd_oracle import PSTD as OraclePSTD

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore:The PSTD code")]

TOL = 1e-4  # relative L2 of the ROI field vs the FP32 restatement


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def cw(ncycle):
    """A CW source without the slow start, so that every cycle may terminate."""
    return np.exp(-2.0j * np.pi * ncycle)


def medium(shape, seed):
    rng = np.random.default_rng(seed)
    return 1.0 + 0.2 * rng.random(shape) + 0.02j


CASES = {
    # name: (roi shape, boundary widths, steps)
    "2d_64": ((48, 48), [8, 8], 200),
    "2d_256_fast": ((240, 240), [8, 8], 120),
    "3d_32": ((24, 24, 24), [4, 4, 4], 80),
    "3d_64_fast": ((48, 48, 48), [8, 8, 8], 60),
    "3d_256_cluster": ((240, 240, 8), [8, 8, 4], 40),
    "3d_mixed_192": ((176, 176, 8), [8, 8, 4], 40),
}


@pytest.mark.parametrize("name", list(CASES))
def test_pstd_fixed_steps_match_oracle(gpu, name):
    import wavesim_b200 as ws
    shape, bw, steps = CASES[name]
    n = medium(shape, 5)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "boundary_type": "ARL",
           "energy_threshold": 1e-30, "source_amplitude": cw}
    val = np.ones(shape[:2]) + 0.5j
    pos = [1] * len(shape)
    p = ws.PSTD(n, opt)
    E, st = p.exec(ws.Source(val, pos), max_iterations=steps)
    p.close()
    o = OraclePSTD(n, dict(opt, single_precision=True))
    Eo, so = o.exec(ref.Source(val, pos), max_iterations=steps)
    Eo = Eo[..., 0] if len(shape) == 2 else Eo
    E = E[..., 0] if len(shape) == 2 else E
    assert st.it == so.it
    assert rel(E, Eo) < TOL, rel(E, Eo)
    np.testing.assert_allclose(st.diff_energy, so.diff_energy, rtol=1e-3)


def test_pstd_default_source_run_matches_oracle(gpu):
    """The reference's default run: slow start over 100 cycles, then the energy stop rule."""
    import wavesim_b200 as ws
    n = medium((40, 40), 6)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8], "boundary_type": "ARL",
           "energy_threshold": 1e-3}
    src = (np.ones((1, 1)), [20, 20])
    p = ws.PSTD(n, opt)
    E, st = p.exec(ws.Source(*src))
    o = OraclePSTD(n, dict(opt, single_precision=True))
    Eo, so = o.exec(ref.Source(*src))
    assert st.converged == so.converged
    assert st.it == so.it
    assert rel(E[..., 0], Eo[..., 0]) < 1e-3, rel(E[..., 0], Eo[..., 0])


def test_pstd_reaches_the_mbs_steady_state(gpu):
    """Absorbing periodic medium: PSTD with a small time step converges to the
    Helmholtz solution that MBS computes."""
    import wavesim_b200 as ws
    L = 64
    rng = np.random.default_rng(1)
    n = 1.0 + 0.1 * rng.random((L, L)) + 0.05j
    src = ws.Source(np.ones((1, 1)), [L // 2, L // 2])
    m = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "energy_threshold": 1e-9})
    Em, _ = m.exec(src)
    m.close()
    p = ws.PSTD(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "boundary_type": "ARL",
                    "energy_threshold": 1e-7, "dt_relative": 0.1})
    Ep, sp = p.exec(src)
    assert sp.converged
    assert rel(Ep[..., 0], Em[..., 0]) < 6e-3, rel(Ep[..., 0], Em[..., 0])


def test_pstd_no_source_in_grid(gpu):
    import wavesim_b200 as ws
    p = ws.PSTD(np.ones((16, 16)), {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [4, 4],
                                    "boundary_type": "ARL"})
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        E, st = p.exec(ws.Source(np.ones((1, 1)), [100, 100]))
    assert E is None and st.source_energy == 0
