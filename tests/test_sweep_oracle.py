"""The premise of the continuation start (wavesim_b200.batch.plane_wave_tilt),
checked with the oracle's solves (oracle/mbs_oracle.py, the reference loop of
WaveSimBase.m:157-197) in free space: the field of a plane wave tilted to the
next angle, including the change of the propagation phase along the source
line's normal, is close to that angle's own field away from the grid edges,
and much closer than with the transverse phase alone."""
import numpy as np

from oracle import mbs_oracle as ref


def _fields(angles, shape=(96, 96), bw=(32, 32)):
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": list(bw), "energy_threshold": 1e-5}
    k = 2 * np.pi * 0.25
    sim = ref.WaveSim(np.ones(shape), opt)
    out = []
    for a in angles:
        line = np.exp(1j * k * np.sin(np.radians(a)) * np.arange(shape[0]))[:, None]
        E, _ = sim.exec(ref.Source(line, [1, 1]))
        out.append(np.asarray(E).reshape(shape))
    return out, opt, k


def test_tilt_with_the_normal_phase_matches_the_next_angle():
    import wavesim_b200 as ws
    from wavesim_b200.batch import plane_wave_tilt
    angles = (20.0, 21.0)
    (E0, E1), opt, k = _fields(angles)
    sim = ws.WaveSim(np.ones((96, 96)), opt)  # host set-up only: roi, k0c, pixel size
    w0, w1 = [ws.PlaneWave((96, 1), [1, 1], phase=(k * np.sin(np.radians(a)), 0.0)) for a in angles]
    fy, fx, fz = plane_wave_tilt(sim, w0, w1)
    core = (slice(24, 72), slice(8, 88))

    def err(est):
        return float(np.linalg.norm(est[core] - E1[core]) / np.linalg.norm(E1[core]))

    full = err(E0 * fy[:, None] * fx[None, :])
    transverse_only = err(E0 * fy[:, None])
    # (about 0.1 is the finite source line's diffraction, which no tilt follows)
    assert full < 0.13, full
    assert full < 0.4 * transverse_only, (full, transverse_only)
