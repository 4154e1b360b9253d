"""Parity of the CUDA loop (through the C ABI) with the CPU oracle.

The oracle (oracle/mbs_oracle.py) restates the reference's MATLAB loop; it is
run here on the same seeded inputs.  The bar (from the reference comparison
it replaces) is a relative L2 error of the ROI field of at most 1e-4 against
the FP32 restatement at an identical iteration count; the error against the
FP64 restatement is checked at the same bound.  Iteration counts and the
energy history must match the reference's stop rule exactly.
"""
import numpy as np
import pytest

from oracle import mbs_oracle as ref
from oracle.analytic import homogeneous_1d

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative L2 of the ROI field vs the reference restatement


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def make_pair(n, opt, vector=False):
    import wavesim_b200 as ws
    P = ws.WaveSimVector if vector else ws.WaveSim
    O = ref.WaveSimVector if vector else ref.WaveSim
    return P(n, opt), O(n, dict(opt, single_precision=True)), O(n, dict(opt, single_precision=False))


def to_ref_source(src_value, pos):
    return ref.Source(src_value, pos)


def check_fixed(n, opt, value, pos, iters, vector=False, tol=TOL):
    import wavesim_b200 as ws
    opt = dict(opt, energy_threshold=1e-99, max_iterations=iters)
    sim, o32, o64 = make_pair(n, opt, vector)
    E, st = sim.exec(ws.Source(value, pos))
    e32, s32 = o32.exec(ref.Source(value, pos), max_iterations=iters)
    e64, s64 = o64.exec(ref.Source(value, pos), max_iterations=iters)
    assert st.it == s32.it
    err32, err64 = rel(E, e32), rel(E, e64)
    assert err32 < tol, (err32, err64)
    assert err64 < tol, (err32, err64)
    np.testing.assert_allclose(st.diff_energy, s32.diff_energy, rtol=2e-4)
    sim.close()
    return err32, err64


def test_2d_point_source_fixed_iterations(gpu):
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16]}
    check_fixed(np.ones((64, 64)), opt, 1.0, [33, 33], 40)


def test_2d_disordered_rectangular(gpu):
    rng = np.random.default_rng(1)
    n = 1.0 + 0.3 * rng.random((48, 80)) + 0.01j
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16]}
    check_fixed(n, opt, rng.standard_normal((48, 1)) + 0j, [1, 1], 48)


def test_3d_sphere_fixed_iterations(gpu):
    L = 24
    y, x, z = np.meshgrid(*(np.arange(L) - L / 2,) * 3, indexing="ij")
    n = np.where(x ** 2 + y ** 2 + z ** 2 < 36, 1.5, 1.33)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [4, 4, 4]}
    check_fixed(n, opt, np.ones((L, L)), [1, 1, 1], 32)


def test_3d_cluster_split_planes(gpu):
    # 256 x 256 planes do not fit one block: the x transform goes through a cluster
    rng = np.random.default_rng(2)
    n = 1.33 + 0.05 * rng.random((240, 240, 8))
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8, 4]}
    check_fixed(n, opt, np.ones((240, 240)), [1, 1, 4], 16)


def test_vector_sphere_fixed_iterations(gpu):
    L = 20
    y, x, z = np.meshgrid(*(np.arange(L) - L / 2,) * 3, indexing="ij")
    n = np.where(x ** 2 + y ** 2 + z ** 2 < 25, 1.5, 1.33)
    opt = {"lambda": 0.5, "pixel_size": 0.0625, "boundary_widths": [6, 6, 6]}
    check_fixed(n, opt, np.ones((L, L)), [1, 1, 1, 1], 24, vector=True)


@pytest.mark.parametrize("shape", [(45, 60), (77, 33), (50, 1)])
def test_mixed_radix_sizes(gpu, shape):
    rng = np.random.default_rng(3)
    n = 1.0 + 0.2 * rng.random(shape)
    bw = [5, 7] if shape[1] > 1 else [6, 0]
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw}
    check_fixed(n, opt, 1.0, [shape[0] // 2 + 1, shape[1] // 2 + 1], 24)


def test_reference_stop_rule_iterations(gpu):
    """Stop decided on the device with the reference's stale-energy schedule."""
    import wavesim_b200 as ws
    rng = np.random.default_rng(4)
    n = 1.0 + 0.2 * rng.random((96, 64))
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-4}
    sim, o32, _ = make_pair(n, opt)
    E, st = sim.exec(ws.Source(1.0, [48, 32]))
    e32, s32 = o32.exec(ref.Source(1.0, [48, 32]))
    assert st.converged and s32.converged
    assert st.it == s32.it
    np.testing.assert_allclose(st.diff_energy, s32.diff_energy, rtol=2e-4)
    assert rel(E, e32) < TOL


def test_fresh_stop_rule(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-4,
           "stop_rule": "fresh"}
    sim = ws.WaveSim(np.ones((64, 64)), opt)
    E, st = sim.exec(ws.Source(1.0, [33, 33]))
    o = ref.WaveSim(np.ones((64, 64)), opt)
    _, s = o.exec(ref.Source(1.0, [33, 33]), fresh_energy=True)
    fe = np.array(s.fresh_energy)
    # first multiple of Nw whose fresh energy ratio is below the threshold
    nw = len(o.wiggles)
    k = next(i for i in range(nw, len(fe) + 1, nw) if fe[i - 1] / fe[0] < 1e-4)
    assert st.it - 1 == k


def test_analytic_1d(gpu):
    """utilities/homogeneous_medium_analytic_solution.m as the known answer."""
    import wavesim_b200 as ws
    L = 256
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [32, 0], "energy_threshold": 1e-9}
    sim = ws.WaveSim(np.ones((L, 1)), opt)
    E, st = sim.exec(ws.Source(1.0, [L // 2 + 1, 1]))
    x = (np.arange(L) - L // 2) * 0.25
    ana = homogeneous_1d(2 * np.pi, 0.25, x)
    err = rel(E[:, 0, 0], ana)
    # the FP32 restatement reaches 7e-6 on this case
    assert err < 3e-5, err


def test_graph_and_host_loop_agree(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-3}
    a = ws.WaveSim(np.ones((64, 64)), opt)
    b = ws.WaveSim(np.ones((64, 64)), dict(opt, use_graph=False))
    Ea, sa = a.exec(ws.Source(1.0, [33, 33]))
    Eb, sb = b.exec(ws.Source(1.0, [33, 33]))
    assert sa.it == sb.it
    assert rel(Ea, Eb) < 1e-6


def test_repeated_solves_reuse_solver(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-3}
    a = ws.WaveSim(np.ones((64, 64)), opt)
    E1, s1 = a.exec(ws.Source(1.0, [33, 33]))
    E2, s2 = a.exec(ws.Source(2.0, [33, 33]))
    E3, s3 = a.exec(ws.Source(1.0, [33, 33]))
    assert rel(E2, 2 * E1) < 1e-5 and s1.it == s2.it  # linearity in the source
    assert np.array_equal(E1, E3)


def test_callbacks_called(gpu):
    import wavesim_b200 as ws
    calls = []
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-3,
           "callback": lambda sim, state: calls.append(state.it), "callback_interval": 8}
    sim = ws.WaveSim(np.ones((64, 64)), opt)
    E, st = sim.exec(ws.Source(1.0, [33, 33]))
    n = st.it - 1
    assert calls[-1] == n
    assert all(c % 8 == 0 for c in calls[:-1])
    assert len(calls) >= n // 8


def test_source_partly_outside_and_overlapping(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8], "energy_threshold": 1e-99,
           "max_iterations": 16}
    n = np.ones((40, 40))
    # a block that sticks out of the grid, plus two overlapping point sources
    v = np.arange(30, dtype=float).reshape(6, 5) + 1j
    sp = ws.Source(v, [-3, 36]) + ws.Source(1.0, [20, 20]) + ws.Source(2.0, [20, 20])
    so = ref.Source(v, [-3, 36]) + ref.Source(1.0, [20, 20]) + ref.Source(2.0, [20, 20])
    E, st = ws.WaveSim(n, opt).exec(sp)
    e, s = ref.WaveSim(n, opt).exec(so, max_iterations=16)
    assert rel(E, e) < TOL


def test_no_source_in_grid(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8]}
    with pytest.warns(UserWarning):
        E, st = ws.WaveSim(np.ones((32, 32)), opt).exec(ws.Source(1.0, [500, 500]))
    assert E is None


def test_max_iterations_not_converged(gpu):
    import wavesim_b200 as ws
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-12,
           "max_iterations": 10}
    E, st = ws.WaveSim(np.ones((64, 64)), opt).exec(ws.Source(1.0, [33, 33]))
    assert not st.converged and st.it - 1 == 12  # first multiple of Nw=4 past 10


def test_vector_polarisations(gpu):
    L = 16
    opt = {"lambda": 0.5, "pixel_size": 0.0625, "boundary_widths": [4, 4, 4]}
    for pol in (2, 3):
        check_fixed(np.full((L, L, L), 1.33), opt, np.ones((L, 1)), [1, 4, 8, pol], 16, vector=True)


def test_roi_option(gpu):
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [8, 8], "roi": [[5, 3], [20, 30]]}
    check_fixed(np.ones((32, 40)), opt, 1.0, [10, 10], 16)
