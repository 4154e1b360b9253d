"""Medium set-up on the device (ws_medium_reduce, ws_build_gamma): the same
epsilon, k0c, k02e and gamma as the oracle's restatement of the reference
set-up (oracle/mbs_oracle.py WaveSim.__init__: WaveSimBase.m:58-81, 201-258,
Medium.m:15-72), in its FP64 form, and the same solve as the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["2d_complex", "3d_spheres", "3d_vector"])
def test_device_setup_matches_host(gpu, case):
    import wavesim_b200 as ws
    from wavesim_b200.workloads import gaussian_random_field, sphere_medium
    rng = np.random.default_rng(9)
    if case == "2d_complex":
        n = np.clip(1.0 + 0.3 * gaussian_random_field((100, 90), 4, rng), 0.8, 1.6) + 0.01j
        opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 12], "energy_threshold": 1e-3}
        src, cls = ws.Source(np.ones((100, 1)), [1, 1]), ws.WaveSim
    elif case == "3d_spheres":
        n = sphere_medium(32, rng)
        opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8, 8], "energy_threshold": 1e-3}
        src, cls = ws.Source(np.ones((32, 32)), [1, 1, 1]), ws.WaveSim
    else:
        n = sphere_medium(24, rng)
        opt = {"lambda": 0.5, "pixel_size": 0.0625, "boundary_widths": [8, 8, 8], "energy_threshold": 1e-3}
        src, cls = ws.Source(np.ones((24, 24)), [1, 1, 1, 1]), ws.WaveSimVector
    from oracle import mbs_oracle as ref
    orc = (ref.WaveSimVector if cls is ws.WaveSimVector else ref.WaveSim)(n, dict(opt, single_precision=False))
    dev = cls(n, dict(opt, device_setup=True))
    assert dev.device_setup
    assert dev.epsilon == pytest.approx(float(orc.epsilon), rel=1e-6)
    assert dev.k0c == pytest.approx(orc.k0c, rel=1e-12)
    assert complex(dev.k02e) == pytest.approx(complex(orc.k02e), rel=1e-6)
    g = np.asarray(orc.gamma)
    # gamma is rounded once to complex64 from the FP64 value
    assert np.abs(dev.gamma - g).max() <= 2e-7 * np.abs(g).max()
    Ed, sd = dev.exec(src)
    orc32 = (ref.WaveSimVector if cls is ws.WaveSimVector else ref.WaveSim)(n, dict(opt, single_precision=True))
    Eo, so = orc32.exec(ref.Source(src.values[0], src.positions[0]))
    assert sd.it == so.it
    assert float(np.linalg.norm(np.ravel(Ed) - np.ravel(Eo)) / np.linalg.norm(np.ravel(Eo))) < 1e-4
