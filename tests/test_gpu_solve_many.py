"""Concurrent solves of media of different sizes (wavesim_b200.batch): each
result equals the same solve run alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems():
    import wavesim_b200 as ws
    from wavesim_b200.workloads import gaussian_random_field, sphere_medium
    rng = np.random.default_rng(11)
    out = []
    for k, side in enumerate([64, 96, 128, 80]):
        n = np.clip(1.0 + 0.3 * gaussian_random_field((side, side), 4, rng), 0.8, 1.6) + 0.01j
        sim = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-3})
        out.append((sim, ws.Source(np.ones((side, 1)), [1, 1])))
    for side in (32, 48):
        n = sphere_medium(side, rng)
        sim = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8, 8], "energy_threshold": 1e-3})
        out.append((sim, ws.Source(np.ones((side, side)), [1, 1, 1])))
    return out


def test_concurrent_media_match_sequential(gpu):
    from wavesim_b200.batch import solve_many
    probs = _problems()
    E_seq, s_seq, _ = solve_many(probs, workers=1)
    E_par, s_par, _ = solve_many(probs, workers=4)
    for a, b, sa, sb in zip(E_seq, E_par, s_seq, s_par):
        assert sa.it == sb.it
        assert float(np.linalg.norm(a - b) / np.linalg.norm(a)) < 1e-6
