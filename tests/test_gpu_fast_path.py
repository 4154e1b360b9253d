"""The power-of-two fast kernels agree with the generic kernels and with the
oracle on every shape they are instantiated for (plane kernels with and
without a thread-block cluster, 2-D column kernels, pencil kernels)."""
import os

import numpy as np
import pytest

from oracle import mbs_oracle as ref

pytestmark = pytest.mark.gpu

TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def run_product(n, opt, val, pos, vector, path):
    import wavesim_b200 as ws
    old = os.environ.get("WAVESIM_B200_PATH")
    try:
        if path == "generic":
            os.environ["WAVESIM_B200_PATH"] = "generic"
        else:
            os.environ.pop("WAVESIM_B200_PATH", None)
        sim = (ws.WaveSimVector if vector else ws.WaveSim)(n, opt)
        E, st = sim.exec(ws.Source(val, pos))
        sim.close()
        return E, st
    finally:
        if old is None:
            os.environ.pop("WAVESIM_B200_PATH", None)
        else:
            os.environ["WAVESIM_B200_PATH"] = old


CASES = {
    # name: (roi shape, boundary widths, iterations, vector)
    "2d_64": ((32, 32), [16, 16], 24, False),
    "2d_128x256": ((96, 224), [16, 16], 24, False),
    "2d_512": ((448, 448), [32, 32], 16, False),
    "3d_64": ((32, 32, 32), [16, 16, 16], 16, False),
    "3d_128_cluster2": ((96, 96, 96), [16, 16, 16], 16, False),
    "3d_256_cluster8": ((224, 224, 16), [16, 16, 8], 16, False),
    "3d_64_vector": ((32, 32, 32), [16, 16, 16], 16, True),
    # mixed-radix kernels (192 = 12 x 4 x 4): planes on a cluster of 6, z pencils
    "3d_192_cluster6": ((160, 160, 8), [16, 16, 4], 16, False),
    "3d_192_cluster6_vector": ((160, 160, 4), [16, 16, 2], 16, True),
    "3d_pencil_192": ((16, 16, 160), [8, 8, 16], 16, False),
    "3d_pencil_192_vector": ((16, 16, 160), [8, 8, 16], 16, True),
    "3d_128_vector": ((96, 96, 96), [16, 16, 16], 8, True),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fast_matches_generic_and_oracle(gpu, name):
    shape, bw, iters, vector = CASES[name]
    rng = np.random.default_rng(7)
    n = 1.2 + 0.2 * rng.random(shape) + 0.005j
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-99,
           "max_iterations": iters}
    if vector:
        opt.update(pixel_size=0.125)
    val = rng.standard_normal(shape[:2]) + 1j * rng.standard_normal(shape[:2])
    pos = [1] * len(shape) + ([2] if vector else [])
    Ef, sf = run_product(n, opt, val, pos, vector, "fast")
    Eg, sg = run_product(n, opt, val, pos, vector, "generic")
    sim = (ref.WaveSimVector if vector else ref.WaveSim)(n, opt)
    Eo, so = sim.exec(ref.Source(val, pos), max_iterations=iters)
    assert sf.it == sg.it == so.it
    assert rel(Ef, Eo) < TOL, rel(Ef, Eo)
    assert rel(Eg, Eo) < TOL, rel(Eg, Eo)
    assert rel(Ef, Eg) < TOL
    np.testing.assert_allclose(sf.diff_energy, so.diff_energy, rtol=2e-4)
