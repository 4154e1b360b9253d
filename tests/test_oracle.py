"""CPU tests of the oracle: pinned against the reference's own known-answer
function and against the committed golden fixtures."""
import os

import numpy as np
import pytest

from oracle import mbs_oracle as ref
from oracle.analytic import homogeneous_1d, homogeneous_2d, homogeneous_3d

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize("single,tol", [(True, 2e-5), (False, 1e-5)])
def test_analytic_1d_pin(single, tol):
    """utilities/homogeneous_medium_analytic_solution.m:1-37 (reference's known answer)."""
    L = 256
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [32, 0], "energy_threshold": 1e-9,
           "single_precision": single}
    E, st = ref.WaveSim(np.ones((L, 1)), opt).exec(ref.Source(1.0, [L // 2 + 1, 1]))
    assert st.converged
    x = (np.arange(L) - L // 2) * 0.25
    assert rel(E[:, 0, 0], homogeneous_1d(2 * np.pi, 0.25, x)) < tol


def test_analytic_1d_value_at_zero():
    """homogeneous_medium_analytic_solution.m:34-35 special value at x=0."""
    k, h = 2 * np.pi, 0.25
    v = homogeneous_1d(k, h, np.array([0.0]))[0]
    assert np.isclose(v, 1j * h / (2 * k) * (1 + 2j * np.arctanh(h * k / np.pi) / np.pi))


def test_continuum_2d():
    L = 96
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [24, 24], "energy_threshold": 1e-6}
    E, st = ref.WaveSim(np.ones((L, L)), opt).exec(ref.Source(1.0, [L // 2 + 1, L // 2 + 1]))
    y = (np.arange(L) - L // 2) * 0.25
    r = np.hypot(y[:, None], y[None, :])
    m = r > 2
    assert rel(E[..., 0][m], homogeneous_2d(2 * np.pi, 0.25, r[m])) < 2e-3


def test_continuum_3d():
    L = 40
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [12, 12, 12], "energy_threshold": 1e-5}
    E, st = ref.WaveSim(np.ones((L, L, L)), opt).exec(ref.Source(1.0, [L // 2 + 1] * 3))
    y = (np.arange(L) - L // 2) * 0.25
    r = np.sqrt(y[:, None, None] ** 2 + y[None, :, None] ** 2 + y[None, None, :] ** 2)
    m = r > 2
    assert rel(E[m], homogeneous_3d(2 * np.pi, 0.25, r[m])) < 5e-3


@pytest.mark.parametrize("name", ["point2d", "disordered2d", "mixed_radix2d", "sphere3d", "vector3d", "line1d"])
def test_golden_fixtures(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    E32, s32 = mg.run_oracle(name, True)
    E64, s64 = mg.run_oracle(name, False)
    assert s32.it - 1 == int(g["iterations"])
    assert rel(E32, g["E32"]) < 1e-5
    assert rel(E64, g["E64"]) < 1e-12
    np.testing.assert_allclose(s64.diff_energy, g["diff_energy64"], rtol=1e-10)
    # the FP32 and FP64 restatements agree to the parity bound
    assert rel(g["E32"], g["E64"]) < 1e-4


def test_wiggle_perm_order():
    """private/wiggle_perm.m:16-27 column order."""
    w2 = ref.wiggle_perm([1, 1, 0])
    assert w2.tolist() == [[1, -1, -1, 1], [1, 1, -1, -1], [0, 0, 0, 0]]
    w3 = ref.wiggle_perm([1, 1, 1])
    unshuffled = np.array([[(-1) ** (np.ceil(c / 2 ** (r - 1)) + 1) for c in range(1, 9)] for r in range(1, 4)])
    assert np.array_equal(w3, unshuffled[:, [0, 1, 2, 4, 3, 5, 6, 7]])
    assert ref.wiggle_perm([0, 0, 0]).shape == (3, 1)
    w1 = ref.wiggle_perm([0, 1, 0])
    assert w1.tolist() == [[0, 0], [1, -1], [0, 0]]


def test_efficient_size():
    """SimulationGrid.m:64-80."""
    assert ref.efficient_size([17, 97, 224 + 32, 960 + 64, 13, 143, 98]).tolist() == \
        [18, 99, 256, 1024, 14, 144, 99]


def test_nuttallwin():
    w = ref.nuttallwin(7)
    assert np.isclose(w[3], 1.0, atol=1e-7) and np.isclose(w[0], 3.628e-4, atol=1e-6)
    assert np.allclose(w, w[::-1])


def test_symrange_matches_matlab_fftshift():
    assert ref.symrange(4).tolist() == [0, 1, -2, -1]
    assert ref.symrange(5).tolist() == [1, 2, -2, -1, 0]  # MATLAB fftshift on an odd length


def test_source_shift_crop_add():
    s = ref.Source(np.arange(12.0).reshape(3, 4), [0, 2]) + ref.Source(5.0, [10, 10])
    c = s.shift([2, 2, 1, 1]).crop(np.array([[1, 1, 1, 1], [4, 4, 1, 1]]))
    assert len(c.positions) == 1 and c.positions[0].tolist() == [1, 3, 1, 1]
    assert c.values[0].shape == (3, 2, 1, 1)
    E = c.add_to(np.zeros((4, 4, 1)), 2.0)
    assert E[0, 2, 0] == 2 * 0 and E[2, 3, 0] == 2 * 9


def test_gain_rejected():
    with pytest.raises(ValueError):
        ref.WaveSim(np.ones((8, 8)) - 0.1j, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [2, 2]})


def test_zero_source_returns_nothing():
    sim = ref.WaveSim(np.ones((16, 16)), {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [4, 4]})
    with pytest.warns(UserWarning):
        E, st = sim.exec(ref.Source(1.0, [100, 100]))
    assert E is None
