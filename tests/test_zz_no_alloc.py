"""ws_run_algorithm_noalloc against ws_run_algorithm.

ws_run_algorithm_noalloc serves callers that cannot allocate GPU memory
while they run (an application whose memory pool owns the device, a loop that
forbids allocation after start-up, a plug-in limited to the buffers it is
given): its working arrays live in one static device array instead of
cudaMalloc'd memory.  This test allocates the input and output buffers
itself (as such a caller would have done up front), runs the entry point
twice in a row - the static array keeps the first call's contents, so the
second call checks that everything that must start at zero is cleared - and
compares both results with the allocating entry point, within the 1e-4
relative L2 bound of the parity tests.  The file sorts last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def dense_source(sim, source):
    """The source blocks (after the shift and crop of Simulation.exec) summed
    into one column-major field of the grid's size."""
    s, blocks, keep = sim.source_blocks(source)
    F = np.zeros(tuple(int(v) for v in sim.N), dtype=np.complex64, order="F")
    for p, v in zip(s.positions, keep):
        t = [int(a) - 1 for a in p]
        F[t[0]:t[0] + v.shape[0], t[1]:t[1] + v.shape[1], t[2]:t[2] + v.shape[2], t[3]:t[3] + v.shape[3]] += v
    return s, blocks, keep, F


def run_allocating(sim, source, maxit):
    """The existing entry point (RunWaveSimAlgorithmMex argument list) on host buffers."""
    from wavesim_b200 import _lib
    s, blocks, keep = sim.source_blocks(source)
    E = np.zeros(int(np.prod(sim.N)), np.complex64)
    hist = np.zeros(maxit + len(sim.wiggles) + 1)
    n = C.c_int64()
    gamma = np.asfortranarray(sim.gamma)  # kept alive for the call
    _lib.check(_lib.lib.ws_run_algorithm(
        (C.c_int64 * 4)(*[int(v) for v in sim.N]), gamma.ctypes.data, len(sim.wiggles),
        sim._wiggle_structs(), len(s.values), blocks, C.c_float(sim.epsilon),
        _lib.ws_complex(sim.k02e.real, sim.k02e.imag), sim._roi8(), maxit, sim.energy_threshold, b"NoCallback",
        sim.callback_interval, _lib.CALLBACK(), None, _lib.WS_HOST, E.ctypes.data,
        hist.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)))
    return E, int(n.value), hist[:n.value]


def run_noalloc(sim, source, maxit, torch):
    """The allocation-free entry point on device buffers made by the caller."""
    from wavesim_b200 import _lib
    dev = torch.device("cuda", 0)

    def to_dev(a):
        a = np.ascontiguousarray(np.asarray(a).ravel(order="F"))
        return torch.from_numpy(a.view(np.float32) if np.iscomplexobj(a) else a).to(dev)

    s, blocks, keep, F = dense_source(sim, source)
    gamma = to_dev(np.asfortranarray(sim.gamma))
    src = to_dev(F)
    wkeep = []
    wig = (_lib.ws_wiggle * len(sim.wiggles))()
    for i, w in enumerate(sim.wiggles):
        parts = [to_dev(a) for a in (w.pxe, w.pye, w.pze, w.gx, w.gy, w.gz)]
        wkeep.extend(parts)
        wig[i] = _lib.ws_wiggle(*[t.data_ptr() for t in parts])
    E = torch.empty(2 * int(np.prod(sim.N)), dtype=torch.float32, device=dev)
    E.fill_(12345.0)  # garbage: the entry point must clear its output
    hist = torch.empty(maxit + len(sim.wiggles) + 1, dtype=torch.float64, device=dev)
    n = C.c_int64()
    conv = C.c_int()
    torch.cuda.synchronize()
    rc = _lib.lib.ws_run_algorithm_noalloc(
        (C.c_int64 * 4)(*[int(v) for v in sim.N]), gamma.data_ptr(), len(sim.wiggles), wig, src.data_ptr(),
        C.c_float(sim.epsilon), _lib.ws_complex(sim.k02e.real, sim.k02e.imag), sim._roi8(), maxit,
        sim.energy_threshold, sim.energy_calculation_interval, E.data_ptr(), hist.data_ptr(), C.byref(n),
        C.byref(conv), None)
    assert rc == 0, _lib.lib.ws_noalloc_last_error()
    torch.cuda.synchronize()
    Ec = E.cpu().numpy().view(np.complex64)
    return Ec, int(n.value), hist.cpu().numpy()[:n.value]


CASES = {
    "2d_disordered": (lambda rng: 1.0 + 0.3 * rng.random((96, 80)) + 0.01j, [16, 16], (48, 40)),
    "2d_mixed_radix": (lambda rng: 1.0 + 0.2 * rng.random((45, 60)), [5, 7], (23, 31)),
    "3d_spheres": (lambda rng: np.where(rng.random((32, 32, 32)) < 0.1, 1.5, 1.33), [16, 16, 16], (1, 1, 1)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_allocating_entry_twice(gpu, name):
    import torch

    import wavesim_b200 as ws
    make_n, bw, pos = CASES[name]
    rng = np.random.default_rng(11)
    n = make_n(rng)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-3}
    sim = ws.WaveSim(n, opt)
    val = np.ones(n.shape[:2]) if n.ndim == 3 else 1.0
    source = ws.Source(val, list(pos))
    maxit = 2000
    E_ref, n_ref, h_ref = run_allocating(sim, source, maxit)
    for _ in range(2):
        E, n_it, hist = run_noalloc(sim, source, maxit, torch)
        assert n_it == n_ref
        assert rel(E, E_ref) < TOL
        np.testing.assert_allclose(hist, h_ref, rtol=1e-5)


def test_noalloc_rejects_oversize_grid(gpu):
    """A grid larger than the static array is refused on the host, before any launch."""
    import torch

    from wavesim_b200 import _lib
    limit = _lib.lib.ws_noalloc_scratch_bytes()
    side = int(np.ceil((limit / 16) ** (1 / 3))) + 16  # more field elements than the array holds
    N = (C.c_int64 * 4)(side, side, side, 1)
    roi = (C.c_int64 * 8)(1, side, 1, side, 1, side, 1, 1)
    small = torch.zeros(64, dtype=torch.float32, device="cuda")  # never touched: the call stops first
    p = small.data_ptr()
    wig = (_lib.ws_wiggle * 1)(_lib.ws_wiggle(p, p, p, p, p, p))
    rc = _lib.lib.ws_run_algorithm_noalloc(N, p, 1, wig, p, C.c_float(3.0), _lib.ws_complex(1, 1), roi, 10, 1e-3,
                                           8, p, p, None, None, None)
    assert rc == _lib.WS_ERR_INVALID_ARGUMENT
    assert b"static scratch" in _lib.lib.ws_noalloc_last_error()
