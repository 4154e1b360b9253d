"""The continuation sweep's bookkeeping (wavesim_b200.batch.solve_sweep and
plane_wave_start) on the host, with a stand-in solver: which sources go into
which round, which field each warm start comes from, and the tilt between
two plane waves."""
from types import SimpleNamespace

import numpy as np

from wavesim_b200.batch import plane_wave_start, solve_sweep
from wavesim_b200.problem import PlaneWave


class FakeSim:
    """exec_batch returns field = source index (as an array) and records the
    starts it was given."""

    def __init__(self, shape):
        self.roi = np.array([[1, 1, 1, 1], [shape[0], shape[1], 1, 1]])
        self.k0c, self.options = 2.0, {"pixel_size": 0.25}
        self.calls = []

    def exec_batch(self, sources, warm_starts=None):
        self.calls.append(([s.tag for s in sources], None if warm_starts is None else list(warm_starts)))
        return [np.full((2, 2, 1), s.tag, complex) for s in sources], \
            [SimpleNamespace(it=10, warm_discarded=False) for _ in sources]


def test_rounds_and_predecessors():
    sim = FakeSim((2, 2))
    sources = [SimpleNamespace(tag=i) for i in range(7)]
    fields, states, _ = solve_sweep(sim, sources, batch=3, start=lambda E, i, j: (int(E.real.flat[0]), i, j))
    # ceil(7 / 3) = 3 rounds: {0, 3, 6} cold, then {1, 4}, then {2, 5}
    assert [c[0] for c in sim.calls] == [[0, 3, 6], [1, 4], [2, 5]]
    assert sim.calls[0][1] is None
    assert sim.calls[1][1] == [(0, 0, 1), (3, 3, 4)]
    assert sim.calls[2][1] == [(1, 1, 2), (4, 4, 5)]
    assert [int(f.real.flat[0]) for f in fields] == list(range(7))
    assert solve_sweep(sim, [], batch=4) == ([], [], 0.0)


def test_plane_wave_start_tilt():
    sim = FakeSim((6, 5))
    w0 = PlaneWave((6, 1), [2, 1], amplitude=2.0, phase=(0.1, 0.0))
    w1 = PlaneWave((6, 1), [2, 1], amplitude=1.0, phase=(0.3, 0.05))
    E = np.ones((6, 5, 1), complex)
    s = plane_wave_start(sim, E, w0, w1)
    y = np.arange(6)[:, None] - 1  # rows from the block corner (position 2)
    x = np.arange(5)[None, :]
    # x is the block's normal: the phase per pixel there follows from the
    # background wavenumber kc = 2 * 0.25 and the transverse phase
    kn = np.sqrt(0.25 - 0.3 ** 2) - np.sqrt(0.25 - 0.1 ** 2)
    want = 0.5 * np.exp(1j * (0.2 * y + kn * x))
    np.testing.assert_allclose(s[..., 0], want, rtol=1e-6)
    assert s.dtype == np.complex64
    # [y, x] and [y, x, z, c] fields take the same factor
    np.testing.assert_allclose(plane_wave_start(sim, E[..., 0], w0, w1), want, rtol=1e-6)
    np.testing.assert_allclose(plane_wave_start(sim, E[..., None], w0, w1)[..., 0, 0], want, rtol=1e-6)


def test_device_starts_equal_initial_field():
    """WaveSim.device_starts (torch, here on CPU tensors) continues ROI
    fields over the grid as WaveSim.initial_field does."""
    import torch
    import wavesim_b200 as ws
    rng = np.random.default_rng(4)
    for shape, bw, vec in (((40, 24), [8, 5], False), ((12, 10, 8), [4, 3, 2], False), ((8, 8, 6), [2, 2, 2], True)):
        n = 1.0 + 0.1 * rng.random(shape)
        opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw}
        sim = (ws.WaveSimVector if vec else ws.WaveSim)(n, opt)
        r = sim.roi
        rs = tuple(int(r[1, d] - r[0, d] + 1) for d in range(4))
        roi = (rng.standard_normal(rs) + 1j * rng.standard_normal(rs)).astype(np.complex64)
        want = np.stack([np.ravel(sim.initial_field(f), order="F") for f in (roi, 2 * roi)])
        rows = torch.from_numpy(np.stack([np.ravel(f, order="F") for f in (roi, 2 * roi)]))
        got = sim.device_starts(rows).numpy()
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-7)


def test_host_stage_take():
    """The output staging buffer: take() gives a new array in the requested
    order with the buffer's values, also through its chunked threaded copy."""
    from wavesim_b200._lib import HostStage
    st = HostStage()
    for shape in ((3, 4, 5), (256, 128, 9)):  # the second is above the 4 MB of the chunked copy
        n = int(np.prod(shape))
        buf = st.get(n)
        buf[:] = (np.arange(n) + 1j * np.arange(n)[::-1]).astype(np.complex64)
        f = HostStage.take(buf, shape, "F")
        c = HostStage.take(buf, shape)
        assert f.flags.f_contiguous and c.flags.c_contiguous
        np.testing.assert_array_equal(np.ravel(f, order="F"), buf)
        np.testing.assert_array_equal(np.ravel(c), buf)
        buf[:] = 0  # the results are copies
        assert np.ravel(c)[1] != 0
    assert st.get(10).size == 10
