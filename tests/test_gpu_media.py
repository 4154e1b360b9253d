"""Several media of one grid in one batched solve (ws_solver_create_media,
wavesim_b200.batch.solve_media): every kernel launch covers all the media of
a group, and each medium runs the reference loop and stop rule on its own.
The per-medium arithmetic is that of a single solve, so every field must
equal the medium's own exec bit for bit, at the same iteration count; media
of two sizes go in two groups, solved concurrently."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(ws, sides, seeds, device_setup):
    from wavesim_b200.workloads import sphere_medium
    out = []
    for side, seed in zip(sides, seeds):
        n = sphere_medium(side, np.random.default_rng(seed))
        opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16, 16], "energy_threshold": 1e-3,
               "device_setup": device_setup}
        out.append((ws.WaveSim(n, opt), ws.Source(np.ones((side, side)), [1, 1, 1])))
    return out


@pytest.mark.parametrize("device_setup", [False, True])
def test_media_batch_equals_single_solves(gpu, device_setup):
    import wavesim_b200 as ws
    from wavesim_b200.batch import group_media, solve_media
    probs = _problems(ws, [32, 96, 32, 32, 96], [1, 2, 3, 4, 5], device_setup)
    groups = group_media(probs)
    assert sorted(len(g) for g in groups) == [2, 3]
    singles = [sim.exec(src) for sim, src in probs]
    fields, states, dt, batches = solve_media(probs, workers=2)
    for (Es, ss), E, st in zip(singles, fields, states):
        assert st.it == ss.it and st.converged == ss.converged
        np.testing.assert_array_equal(E, Es)
        np.testing.assert_array_equal(st.diff_energy, ss.diff_energy)
    # the same batches again, reused
    fields2, states2, _, _ = solve_media(probs, workers=1, batches=batches)
    for E, E2 in zip(fields, fields2):
        np.testing.assert_array_equal(E, E2)
    for b in batches:
        if b is not None:
            b.close()


def test_media_batch_refuses_media_that_differ(gpu):
    import wavesim_b200 as ws
    from wavesim_b200.batch import MediaBatch
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16, 16], "energy_threshold": 1e-3}
    a = ws.WaveSim(np.full((32, 32, 32), 1.33), opt)
    b = ws.WaveSim(np.where(np.random.default_rng(0).random((32, 32, 32)) < 0.1, 1.5, 1.33), opt)
    assert a.epsilon != b.epsilon
    with pytest.raises(ValueError):
        MediaBatch([a, b])
