"""Generates the golden fixtures in this folder with the oracle (the FP32 and
FP64 restatements of the reference loop in oracle/mbs_oracle.py):

    python tests/golden/make_golden.py

Each case stores its inputs (by generator parameters), the ROI field E of
the FP32 and FP64 restatements after a fixed number of iterations (the
fixed-iteration protocol of examples/mie_sphere/mie_sphere_test.m:20-21),
the iteration count and the energy history.  Fixtures are small (<= 64^2 or
24^3) so that the CPU tests recompute them in seconds.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import mbs_oracle as ref  # noqa: E402


def case_inputs(name):
    """(refractive index, options, source value, source position, vector, iterations)."""
    rng = np.random.default_rng(sum(map(ord, name)))
    if name == "point2d":
        return np.ones((48, 48)), {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8]}, \
            1.0, [25, 25], False, 24
    if name == "disordered2d":
        n = 1.0 + 0.3 * rng.random((40, 56)) + 0.01j
        src = (rng.standard_normal((40, 1)) + 1j * rng.standard_normal((40, 1)))
        return n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 12]}, src, [1, 1], False, 32
    if name == "mixed_radix2d":
        n = 1.0 + 0.2 * rng.random((45, 60))
        return n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [5, 7]}, 1.0, [23, 31], False, 24
    if name == "sphere3d":
        L = 20
        y, x, z = np.meshgrid(*(np.arange(L) - L / 2,) * 3, indexing="ij")
        n = np.where(x ** 2 + y ** 2 + z ** 2 < 25, 1.5, 1.33)
        return n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [4, 4, 4]}, \
            np.ones((L, L)), [1, 1, 1], False, 24
    if name == "vector3d":
        L = 16
        y, x, z = np.meshgrid(*(np.arange(L) - L / 2,) * 3, indexing="ij")
        n = np.where(x ** 2 + y ** 2 + z ** 2 < 16, 1.5, 1.33)
        return n, {"lambda": 0.5, "pixel_size": 0.0625, "boundary_widths": [4, 4, 4]}, \
            np.ones((L, L)), [1, 1, 1, 1], True, 16
    if name == "line1d":
        return np.ones((128, 1)), {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 0]}, \
            1.0, [65, 1], False, 32
    raise KeyError(name)


CASES = ["point2d", "disordered2d", "mixed_radix2d", "sphere3d", "vector3d", "line1d"]


def run_oracle(name, single):
    n, opt, val, pos, vector, iters = case_inputs(name)
    cls = ref.WaveSimVector if vector else ref.WaveSim
    sim = cls(n, dict(opt, energy_threshold=1e-99, single_precision=single))
    E, st = sim.exec(ref.Source(val, pos), max_iterations=iters)
    return E, st


def main():
    for name in CASES:
        E32, s32 = run_oracle(name, True)
        E64, s64 = run_oracle(name, False)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), E32=E32.astype(np.complex64),
                            E64=E64.astype(np.complex128), iterations=s32.it - 1,
                            diff_energy32=np.array(s32.diff_energy), diff_energy64=np.array(s64.diff_energy))
        print(name, E32.shape, s32.it - 1)


if __name__ == "__main__":
    main()
