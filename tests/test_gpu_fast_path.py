"""The fast kernels (power-of-two and register-resident mixed-radix) agree
with the generic kernels and with the oracle on every shape they are
instantiated for (plane kernels with and without a thread-block cluster, 2-D
column kernels, pencil kernels)."""
import os

import numpy as np
import pytest

from oracle import mbs_oracle as ref

pytestmark = pytest.mark.gpu

TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def run_product(n, opt, val, pos, vector, path, env=None):
    import wavesim_b200 as ws
    env = dict(env or {})
    env["WAVESIM_B200_PATH"] = "generic" if path == "generic" else None
    old = {k: os.environ.get(k) for k in env}
    try:
        for k, v in env.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        sim = (ws.WaveSimVector if vector else ws.WaveSim)(n, opt)
        E, st = sim.exec(ws.Source(val, pos))
        sim.close()
        return E, st
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


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
    "3d_pencil_192_vector_plain": ((16, 16, 160), [8, 8, 16], 16, True, {"WAVESIM_B200_K2": "plain"}),
    "3d_128_vector": ((96, 96, 96), [16, 16, 16], 8, True),
    # 96-point lines (12 x 4 x 2): a whole 96^2 plane on one block
    "3d_96": ((64, 64, 64), [16, 16, 16], 16, False),
    "3d_96_vector": ((64, 64, 64), [16, 16, 16], 8, True),
    # four-stage plans with more elements per thread than the first radix:
    # 160 = 10 x 4 x 4 (20 per thread), 224 = 14 x 4 x 4 (28 per thread);
    # planes on clusters of 5 and 7 blocks, z pencils
    "3d_160_cluster5": ((128, 128, 8), [16, 16, 4], 16, False),
    "3d_224_cluster7": ((192, 192, 8), [16, 16, 4], 16, False),
    "3d_pencil_160": ((16, 16, 128), [8, 8, 16], 16, False),
    "3d_pencil_224": ((16, 16, 192), [8, 8, 16], 16, False),
    # 2-D grids on mixed-radix lines: columns (kmc_col_*2d) and x pencils
    # (km_pencil along x); 320 = 4 x 4 x 4 x 5, 448 = 14 x 4 x 4 x 2,
    # 576 = 12 x 12 x 4; a partial last block of columns (Nx = 100); a
    # power-of-two column with mixed-radix x pencils
    "2d_320": ((256, 256), [32, 32], 16, False),
    "2d_448": ((384, 384), [32, 32], 16, False),
    "2d_576": ((512, 512), [32, 32], 16, False),
    "2d_192": ((160, 160), [16, 16], 16, False),
    "2d_320x100": ((256, 68), [32, 16], 16, False),
    "2d_256x192": ((224, 160), [16, 16], 16, False),
    # layout variants the autotuner may choose
    "3d_256_cluster16": ((224, 224, 16), [16, 16, 8], 16, False, {"WAVESIM_B200_CLUSTER": "16"}),
    "3d_pencil_192_vector_ty8": ((16, 16, 160), [8, 8, 16], 16, True, {"WAVESIM_B200_PENCIL_TY": "8"}),
    "3d_256_pencil_tma": ((16, 16, 224), [8, 8, 16], 16, False),
    "3d_256_pencil_tma_ty8": ((16, 16, 224), [8, 8, 16], 16, False, {"WAVESIM_B200_TMA_TY": "8"}),
    "3d_256_pencil_tma_ty8_s6": ((16, 16, 224), [8, 8, 16], 16, False,
                                 {"WAVESIM_B200_TMA_TY": "8", "WAVESIM_B200_TMA_STAGES": "6"}),
    "3d_256_pencil_tma_ty4": ((16, 16, 224), [8, 8, 16], 16, False, {"WAVESIM_B200_TMA_TY": "4"}),
    "3d_256_pencil_tma_ty16": ((16, 16, 224), [8, 8, 16], 16, False, {"WAVESIM_B200_TMA_TY": "16"}),
    "3d_256_pencil_plain": ((16, 16, 224), [8, 8, 16], 16, False, {"WAVESIM_B200_K2": "plain"}),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fast_matches_generic_and_oracle(gpu, name):
    shape, bw, iters, vector = CASES[name][:4]
    env = CASES[name][4] if len(CASES[name]) > 4 else None
    rng = np.random.default_rng(7)
    n = 1.2 + 0.2 * rng.random(shape) + 0.005j
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-99,
           "max_iterations": iters}
    if vector:
        opt.update(pixel_size=0.125)
    val = rng.standard_normal(shape[:2]) + 1j * rng.standard_normal(shape[:2])
    pos = [1] * len(shape) + ([2] if vector else [])
    Ef, sf = run_product(n, opt, val, pos, vector, "fast", env)
    Eg, sg = run_product(n, opt, val, pos, vector, "generic")
    sim = (ref.WaveSimVector if vector else ref.WaveSim)(n, opt)
    Eo, so = sim.exec(ref.Source(val, pos), max_iterations=iters)
    assert sf.it == sg.it == so.it
    assert rel(Ef, Eo) < TOL, rel(Ef, Eo)
    assert rel(Eg, Eo) < TOL, rel(Eg, Eo)
    assert rel(Ef, Eg) < TOL
    np.testing.assert_allclose(sf.diff_energy, so.diff_energy, rtol=2e-4)
