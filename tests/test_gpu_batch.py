"""Batched solves (ws_solver_solve_batch): many sources on one medium in one
set of launches give the same fields, iteration counts and energy histories as
one solve per source, each source stopping on its own."""
import numpy as np
import pytest

from oracle import mbs_oracle as ref

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def plane_wave(n, angle):
    return np.exp(1j * 2 * np.pi * np.sin(angle) * 0.25 * np.arange(n))[:, None]


@pytest.mark.parametrize("shape,bw", [((96, 80), [16, 16]), ((45, 60), [5, 7]), ((32, 32, 32), [16, 16, 16])])
def test_batch_equals_single_solves(gpu, shape, bw):
    import wavesim_b200 as ws
    rng = np.random.default_rng(5)
    n = 1.0 + 0.25 * rng.random(shape) + 0.01j
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-3}
    sim = ws.WaveSim(n, opt)
    if len(shape) == 2:
        sources = [ws.Source(plane_wave(shape[0], a), [1, 1]) for a in np.linspace(-0.5, 0.5, 5)]
        sources.append(ws.Source(1.0, [shape[0] // 2, shape[1] // 2]))  # converges at a different iteration
    else:
        sources = [ws.Source(np.ones(shape[:2]) * (1 + k), [1, 1, 1 + 4 * k]) for k in range(3)]
    Eb, sb = sim.exec_batch(sources)
    for src, E, st in zip(sources, Eb, sb):
        Es, ss = sim.exec(src)
        assert st.it == ss.it and st.converged == ss.converged
        assert rel(E, Es) < 1e-6
        np.testing.assert_allclose(st.diff_energy, ss.diff_energy, rtol=1e-6)
    # and each batched field agrees with the oracle
    o = ref.WaveSim(n, opt)
    e0, s0 = o.exec(ref.Source(sources[0].values[0], sources[0].positions[0]))
    assert sb[0].it == s0.it and rel(Eb[0], e0) < 1e-4


def test_batch_stops_each_source_separately(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-4}
    sim = ws.WaveSim(np.ones((64, 64)), opt)
    # a point source and a line source converge after different iteration counts
    srcs = [ws.Source(1.0, [33, 33]), ws.Source(np.ones((64, 1)), [1, 1])]
    Eb, sb = sim.exec_batch(srcs)
    singles = [sim.exec(s)[1].it for s in srcs]
    assert [s.it for s in sb] == singles
    assert singles[0] != singles[1]


def test_plane_wave_descriptors_match_dense_sources(gpu):
    """PlaneWave descriptors (generated on the device) give the fields of the
    same plane waves given as dense Source blocks to the oracle
    (ref.Source(...).add_to, Source.m:139-172, in the reference loop),
    including a block that the grid crops."""
    from oracle import mbs_oracle as ref
    import wavesim_b200 as ws
    from wavesim_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(12)
    n = np.clip(1.0 + 0.2 * gaussian_random_field((96, 80), 4, rng), 0.9, 1.4)
    sim = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-4})
    k = 2 * np.pi * 0.25
    waves = [ws.PlaneWave((96, 1), [1, 1], amplitude=1.0, phase=(k * np.sin(t), 0.0)) for t in (-0.5, 0.0, 0.4)]
    waves.append(ws.PlaneWave((140, 1), [-20, 5], amplitude=0.5 + 0.5j, phase=(0.3, 0.0)))  # cropped by the grid
    Ew, sw = sim.exec_batch(waves)
    orc = ref.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-4})
    for w, E, s in zip(waves, Ew, sw):
        Eo, so = orc.exec(ref.Source(w.values()[..., 0, 0][:, None], list(w.position)))
        assert s.it == so.it
        assert float(np.linalg.norm(np.ravel(E) - np.ravel(Eo)) / np.linalg.norm(np.ravel(Eo))) < 1e-4


def _sweep_medium(ws):
    from wavesim_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(11)
    shape = (192, 192)
    n = np.clip(1.0 + 0.2 * gaussian_random_field(shape, 4, rng), 0.8, 1.5) + 0.01j
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [32, 32], "energy_threshold": 1e-3}
    return ws.WaveSim(n, opt), shape, opt, n


def _waves(ws, ny, degrees):
    k = 2 * np.pi * 0.25
    return [ws.PlaneWave((ny, 1), [1, 1], amplitude=1.0, phase=(k * np.sin(np.radians(a)), 0.0)) for a in degrees]


def test_plane_wave_warm_start_matches_dense_source(gpu):
    """A warm start given with PlaneWave descriptors runs as the same start
    with the wave as a dense Source block."""
    import wavesim_b200 as ws
    from wavesim_b200.batch import plane_wave_start
    sim, shape, _, _ = _sweep_medium(ws)
    w0, w1 = _waves(ws, shape[0], [0.0, 0.5])
    E0, _ = sim.exec_batch([w0])
    start = plane_wave_start(sim, E0[0], w0, w1)
    Ep, sp = sim.exec_batch([w1], warm_starts=[start])
    Ed, sd = sim.exec_batch([ws.Source(w1.values()[:, :, 0, 0], [1, 1])], warm_starts=[start])
    assert not sp[0].warm_discarded and sp[0].it == sd[0].it
    assert rel(Ep[0], Ed[0]) < 1e-5


def test_plane_wave_start_in_a_homogeneous_medium(gpu):
    """In free space a plane wave's field tilted to the next angle is close
    to that angle's field away from the grid edges (the start's premise; the
    source line's ends diffract, which the tilt does not follow: 6% here)."""
    import wavesim_b200 as ws
    from wavesim_b200.batch import plane_wave_start
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [32, 32], "energy_threshold": 1e-6}
    sim = ws.WaveSim(np.ones((128, 128)), opt)
    w0, w1 = _waves(ws, 128, [0.0, 0.5])
    E0, _ = sim.exec_batch([w0])
    E1, _ = sim.exec_batch([w1])
    est = plane_wave_start(sim, E0[0], w0, w1)
    core = (slice(32, 96), slice(8, 120))
    assert rel(est[core], E1[0][core]) < 0.1


def test_solve_sweep_continuation(gpu):
    """solve_sweep: later rounds start from their neighbours, need fewer
    iterations than cold solves, and end as close to a tight solve as the
    cold solves do."""
    import wavesim_b200 as ws
    from wavesim_b200.batch import solve_sweep
    sim, shape, opt, n = _sweep_medium(ws)
    waves = _waves(ws, shape[0], np.linspace(-1.5, 1.5, 7))
    Ew, sw, _ = solve_sweep(sim, waves, batch=2)
    Ec, sc = sim.exec_batch(waves)
    first = set(range(0, 7, 4))  # round 0 of 4 rounds: angles 0 and 4, solved cold
    for i in first:
        assert sw[i].it == sc[i].it and rel(Ew[i], Ec[i]) < 1e-6
    later = [i for i in range(7) if i not in first]
    assert all(not getattr(sw[i], "warm_discarded", False) for i in later)
    assert sum(sw[i].it for i in later) < sum(sc[i].it for i in later)
    simt = ws.WaveSim(n, dict(opt, energy_threshold=1e-9))
    Et, _ = simt.exec_batch([waves[i] for i in later])
    for i, et in zip(later, Et):
        assert rel(Ew[i], et) < 2 * rel(Ec[i], et) + 2e-3


def test_solve_sweep_device_path_matches_host_path(gpu):
    """The sweep with its fields kept on the device (starts built by
    WaveSim.device_starts) runs as the host path with the same starts."""
    import wavesim_b200 as ws
    from wavesim_b200.batch import solve_sweep
    sim, shape, _, _ = _sweep_medium(ws)
    waves = _waves(ws, shape[0], np.linspace(-1.0, 1.0, 5))
    Ed, sd, _ = solve_sweep(sim, waves, batch=2, device=True)
    Eh, sh, _ = solve_sweep(sim, waves, batch=2, device=False)
    assert [s.it for s in sd] == [s.it for s in sh]
    for a, b in zip(Ed, Eh):
        assert rel(a, b) < 1e-4
