"""Medium set-up on the device (ws_medium_reduce, ws_build_gamma): the same
epsilon, k0c and gamma as the NumPy path of WaveSim, and the same solve."""
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
    host = cls(n, opt)
    dev = cls(n, dict(opt, device_setup=True))
    assert dev.device_setup
    assert dev.epsilon == pytest.approx(float(host.epsilon), rel=1e-6)
    assert dev.k0c == pytest.approx(host.k0c, rel=1e-12)
    assert complex(dev.k02e) == pytest.approx(complex(host.k02e), rel=1e-6)
    g = np.asarray(host.gamma)
    assert np.abs(dev.gamma - g).max() <= 2e-7 * np.abs(g).max()
    Eh, sh = host.exec(src)
    Ed, sd = dev.exec(src)
    assert sh.it == sd.it
    assert float(np.linalg.norm(Ed - Eh) / np.linalg.norm(Eh)) < 1e-5
