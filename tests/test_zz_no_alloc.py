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
    # name: (medium, boundary widths, source position, vector, energy threshold, max iterations)
    "2d_disordered": (lambda rng: 1.0 + 0.3 * rng.random((96, 80)) + 0.01j, [16, 16], (48, 40), False, 1e-3, 2000),
    "2d_mixed_radix": (lambda rng: 1.0 + 0.2 * rng.random((45, 60)), [5, 7], (23, 31), False, 1e-3, 2000),
    "3d_spheres": (lambda rng: np.where(rng.random((32, 32, 32)) < 0.1, 1.5, 1.33), [16, 16, 16], (1, 1, 1),
                   False, 1e-3, 2000),
    # 128^3: the fast 128^2 planes on a cluster of 2 blocks (about 32 MiB of scratch)
    "3d_128_cluster": (lambda rng: np.where(rng.random((96, 96, 96)) < 0.1, 1.5, 1.33), [16, 16, 16], (1, 1, 1),
                       False, 1e-99, 24),
    # 48^3 x 3: vector fields on the generic mixed-radix kernels
    "3d_vector_48": (lambda rng: np.where(rng.random((32, 32, 32)) < 0.1, 1.5, 1.33), [8, 8, 8], (1, 1, 1, 1),
                     True, 1e-3, 2000),
}


def make_sim(ws, name):
    make_n, bw, pos, vector, thr, maxit = CASES[name]
    rng = np.random.default_rng(11)
    n = make_n(rng)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": thr}
    sim = (ws.WaveSimVector if vector else ws.WaveSim)(n, opt)
    val = np.ones(n.shape[:2]) if n.ndim == 3 else 1.0
    return n, opt, sim, (val, list(pos)), vector, maxit


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_allocating_entry_twice(gpu, name):
    import torch

    import wavesim_b200 as ws
    n, opt, sim, (val, pos), vector, maxit = make_sim(ws, name)
    source = ws.Source(val, pos)
    E_ref, n_ref, h_ref = run_allocating(sim, source, maxit)
    for _ in range(2):
        E, n_it, hist = run_noalloc(sim, source, maxit, torch)
        assert n_it == n_ref
        assert rel(E, E_ref) < TOL
        np.testing.assert_allclose(hist, h_ref, rtol=1e-5)


def test_noalloc_near_the_scratch_limit_matches_oracle(gpu):
    """A 320 x 7680 2-D grid (2.46 million elements, 39.3 of the 40 MiB)
    through the generic mixed-radix columns: Ny = 320 does not divide the
    8192 elements a block can hold, so the column count per block is capped
    by the kernel's element limit, not by shared memory.  Two calls in a row
    against the allocating entry point, and the field against the FP32
    oracle after the same 16 iterations."""
    import torch

    import wavesim_b200 as ws
    from oracle import mbs_oracle as ref
    rng = np.random.default_rng(5)
    n = 1.0 + 0.2 * rng.random((288, 7648)) + 0.01j
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16], "energy_threshold": 1e-99}
    sim = ws.WaveSim(n, opt)
    assert tuple(int(v) for v in sim.N[:2]) == (320, 7680)
    assert 16 * int(np.prod(sim.N)) < _lib_scratch_bytes()
    pos = [144, 3000]
    source = ws.Source(1.0, pos)
    maxit = 16
    E_ref, n_ref, h_ref = run_allocating(sim, source, maxit)
    for _ in range(2):
        E, n_it, hist = run_noalloc(sim, source, maxit, torch)
        assert n_it == n_ref == maxit
        assert rel(E, E_ref) < TOL
        np.testing.assert_allclose(hist, h_ref, rtol=1e-5)
    Eo, so = ref.WaveSim(n, opt).exec(ref.Source(1.0, pos), max_iterations=maxit)
    assert so.it - 1 == maxit
    # E' -> E = E' / gamma on the roi, as WaveSimBase.m:150-153 does
    Ef = E.reshape(tuple(int(v) for v in sim.N), order="F")[..., 0, 0] / sim.gamma[..., 0]
    r0 = sim.roi[0]
    Ef = Ef[r0[0] - 1:r0[0] - 1 + 288, r0[1] - 1:r0[1] - 1 + 7648]
    assert rel(Ef, np.squeeze(Eo)) < TOL


def _lib_scratch_bytes():
    from wavesim_b200 import _lib
    return int(_lib.lib.ws_noalloc_scratch_bytes())


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
