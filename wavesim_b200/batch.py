"""Many solves at once: media of different sizes, or many sources per medium.

No counterpart in the reference, whose ``exec`` runs one solve at a time
(e.g. the angle sweep of examples/pulse2d.m:31-40 calls it in a loop).

* Sources that share a medium go through ``WaveSim.exec_batch``: one batched
  solve, every kernel launch covering all of them.
* Media of one grid size whose set-up agrees (epsilon, k0c and so the
  wiggles: media whose refractive indices span the same range) go through
  ``solve_media``: one solver for all of them (``ws_solver_create_media``,
  one gamma per medium) and one batched solve, every kernel launch covering
  every medium of the group.
* An ordered sweep of sources on one medium (incidence angles) goes through
  ``solve_sweep``: batched solves in rounds, each source of a later round
  warm-started from its neighbour's field of the round before
  (``plane_wave_start`` tilts a plane wave's field to the next angle).
* Groups of different sizes cannot share a launch (each size has its own FFT
  plan and kernel shapes); ``solve_media`` and ``solve_many`` run them
  concurrently instead: each solver has its own CUDA stream, and ``workers``
  host threads drive them (the C calls release the interpreter lock), so
  small solves that would leave most SMs idle overlap on the GPU.
"""
from __future__ import annotations

import ctypes as C
import time
from concurrent.futures import ThreadPoolExecutor
from types import SimpleNamespace

import numpy as np

from . import _lib


def solve_many(problems, workers=4, warm_starts=None):
    """problems: list of (sim, source) pairs (sim a WaveSim or WaveSimVector,
    each pair its own medium).  Returns (fields, states, seconds) with the
    results in the order of `problems`; warm_starts (optional) one start per
    problem or None, as WaveSim.exec takes them."""
    starts = warm_starts if warm_starts is not None else [None] * len(problems)
    if len(starts) != len(problems):
        raise ValueError("one warm start per problem")

    def run(i):
        sim, src = problems[i]
        return sim.exec(src, warm_start=starts[i])

    t0 = time.perf_counter()
    if workers <= 1:
        out = [run(i) for i in range(len(problems))]
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            out = list(ex.map(run, range(len(problems))))
    dt = time.perf_counter() - t0
    return [o[0] for o in out], [o[1] for o in out], dt


def plane_wave_tilt(sim, w_from, w_to):
    """The ratio of plane wave w_to to plane wave w_from (blocks of the same
    size and place) continued over the ROI, as three 1-D factors along y, x
    and z (the amplitude ratio and the phase offset folded into the first).
    Along the block's own axes the phase per pixel changes by dphase; along
    an axis where the block is one pixel thick (its normal) the wave travels
    away from the block with the phase per pixel kn = sqrt(kc^2 - |phase|^2),
    kc = k0c times the pixel size (the loop's background wavenumber), so
    the factor there is exp(i (kn_to - kn_from) |r - corner|)."""
    r = sim.roi
    n = [int(r[1, d] - r[0, d] + 1) for d in range(3)]
    kc = float(np.real(sim.k0c)) * float(sim.options.get("pixel_size", 1.0))
    ph_from = np.asarray(w_from.phase, float)
    ph_to = np.asarray(w_to.phase, float)
    f = []
    for d in range(3):
        a = np.arange(n[d]) - (int(w_from.position[d]) - 1)
        if int(w_from.size[d]) > 1 or n[d] == 1:
            f.append(np.exp(1j * (ph_to[d] - ph_from[d]) * a))
        else:
            kt_from = sum(ph_from[e] ** 2 for e in range(3) if e != d)
            kt_to = sum(ph_to[e] ** 2 for e in range(3) if e != d)
            kn = np.sqrt(max(kc * kc - kt_to, 0.0)) - np.sqrt(max(kc * kc - kt_from, 0.0))
            f.append(np.exp(1j * kn * np.abs(a)))
    f[0] = f[0] * (w_to.amplitude / w_from.amplitude) * np.exp(1j * (w_to.phase0 - w_from.phase0))
    return f


def plane_wave_start(sim, E_from, w_from, w_to):
    """A start for plane wave w_to from the field E_from (on the ROI, [y, x],
    [y, x, z] or [y, x, z, c]) that plane wave w_from produced: E_from times
    plane_wave_tilt.  Exact in a homogeneous medium; in a scattering one it
    holds for small tilts (the memory effect)."""
    fy, fx, fz = plane_wave_tilt(sim, w_from, w_to)
    E = np.asarray(E_from)
    m = fy[:, None] * fx[None, :]
    if E.ndim >= 3:
        m = m[:, :, None] * fz[None, None, :]
    if E.ndim == 4:
        m = m[..., None]
    return (E * m).astype(np.complex64)


def _sweep_device(sim, sources, k):
    """solve_sweep for PlaneWave sources with the fields kept on the device:
    each round's starts are its predecessors' fields (rows of the round
    before) times the tilt, continued over the grid by WaveSim.device_starts,
    and passed to the solver as device memory."""
    import torch
    n = len(sources)
    r = sim.roi
    rs = [int(r[1, d] - r[0, d] + 1) for d in range(4)]
    fields, states = [None] * n, [None] * n
    prev = None
    for j in range(k):
        idx = list(range(j, n, k))
        srcs = [sources[i] for i in idx]
        starts = None
        if j:
            m = len(idx)
            dev = prev.device
            tl = [plane_wave_tilt(sim, sources[i - 1], sources[i]) for i in idx]
            fy = torch.from_numpy(np.stack([t[0] for t in tl]).astype(np.complex64)).to(dev)
            fx = torch.from_numpy(np.stack([t[1] for t in tl]).astype(np.complex64)).to(dev)
            fz = torch.from_numpy(np.stack([t[2] for t in tl]).astype(np.complex64)).to(dev)
            t = prev[:m].reshape(m, rs[3], rs[2], rs[1], rs[0])  # [rhs, c, z, x, y]
            t = t * fy[:, None, None, None, :] * fx[:, None, None, :, None] * fz[:, None, :, None, None]
            starts = sim.device_starts(t.reshape(m, -1))
        outs, st, prev = sim._exec_plane_waves(srcs, starts, time.perf_counter(), keep_device=True)
        for i, e, s_ in zip(idx, outs, st):
            fields[i], states[i] = e, s_
    return fields, states


def solve_sweep(sim, sources, batch=8, start=None, device=None):
    """An ordered sweep of sources on one medium (e.g. incidence angles in
    order, neighbours giving similar fields), batched and warm-started by
    continuation.  With k = ceil(len / batch) rounds, round 0 solves sources
    0, k, 2k, ... cold in one batched solve; round j solves j, j + k, ...,
    each started from the field of its predecessor (solved in round j - 1)
    mapped by start(E_prev, i_prev, i) (default: plane_wave_start for
    PlaneWave sources, the predecessor's field itself otherwise).  For
    PlaneWave sources with the default start the fields stay on the device
    between rounds (device=None: when CUDA is there; the host path does the
    same arithmetic on host arrays).  Each solve runs to the usual
    tolerance; a start whose initial residual is worse than a cold start's is
    discarded and rerun cold.  Returns (fields, states, seconds) in the order
    of `sources`.  No counterpart in the reference, whose sweeps call exec
    once per source (examples/pulse2d.m:31-40)."""
    from .problem import PlaneWave
    n = len(sources)
    if n == 0:
        return [], [], 0.0
    k = -(-n // max(1, int(batch)))
    t0 = time.perf_counter()
    waves = all(isinstance(s, PlaneWave) for s in sources)
    if device is None:
        try:
            import torch
            device = waves and start is None and torch.cuda.is_available()
        except ImportError:
            device = False
    if device:
        fields, states = _sweep_device(sim, sources, k)
        return fields, states, time.perf_counter() - t0
    if start is None:
        if waves:
            def start(E, i, j):
                return plane_wave_start(sim, E, sources[i], sources[j])
        else:
            def start(E, i, j):
                return E
    fields, states = [None] * n, [None] * n
    for j in range(k):
        idx = list(range(j, n, k))
        srcs = [sources[i] for i in idx]
        warm = None if j == 0 else [start(fields[i - 1], i - 1, i) for i in idx]
        E, st = sim.exec_batch(srcs, warm_starts=warm)
        for i, e, s_ in zip(idx, E, st):
            fields[i], states[i] = e, s_
    return fields, states, time.perf_counter() - t0


def media_key(sim):
    """What media must share to be solved together: grid, roi, epsilon, k02e,
    the wiggles (which follow from grid and epsilon), the kind of field and
    the loop's options."""
    o = sim._options()
    return (type(sim).__name__, tuple(int(v) for v in sim.N), tuple(sim._roi8()[:]), float(np.float32(sim.epsilon)),
            complex(np.complex64(sim.k02e)), len(sim.wiggles), int(o.max_iterations), float(o.energy_threshold),
            int(o.energy_interval), int(o.stop_rule))


class MediaBatch:
    """One solver for several media of the same grid and set-up
    (ws_solver_create_media): right-hand side r runs on medium r."""

    def __init__(self, sims):
        if not sims:
            raise ValueError("no media")
        k0 = media_key(sims[0])
        if any(media_key(s) != k0 for s in sims[1:]):
            raise ValueError("the media differ in grid, roi, epsilon, k02e, wiggles or loop options")
        self.sims = list(sims)
        first = self.sims[0]
        N = (C.c_int64 * 4)(*[int(v) for v in first.N])
        h = C.c_void_p()
        if all(getattr(s, "_gamma_dev", None) is not None for s in self.sims):
            import torch
            gam = torch.cat([s._gamma_dev.reshape(-1) for s in self.sims])
            self._keep = gam
            mem, ptr = _lib.WS_DEVICE, gam.data_ptr()
            wkeep = []
            wig = (_lib.ws_wiggle * len(first.wiggles))()
            for i, w in enumerate(first.wiggles):
                parts = [torch.from_numpy(np.ascontiguousarray(a).view(np.float32)).to(gam.device)
                         for a in (w.pxe, w.pye, w.pze, w.gx, w.gy, w.gz)]
                wkeep.extend(parts)
                wig[i] = _lib.ws_wiggle(*[t.data_ptr() for t in parts])
            device = gam.device.index or 0
        else:
            gam = np.concatenate([np.ravel(np.asfortranarray(s.gamma), order="F") for s in self.sims])
            self._keep = gam
            mem, ptr = _lib.WS_HOST, gam.ctypes.data
            wig = first._wiggle_structs()
            wkeep = None
            device = first.device
        _lib.check(_lib.lib.ws_solver_create_media(N, len(self.sims), ptr, len(first.wiggles), wig,
                                                   C.c_float(first.epsilon),
                                                   _lib.ws_complex(first.k02e.real, first.k02e.imag),
                                                   first._roi8(), mem, device, C.byref(h)))
        del wkeep
        self._keep = None
        self.h = h

    def solve(self, sources):
        """One source per medium; returns (fields, states) as WaveSim.exec_batch."""
        R = len(self.sims)
        if len(sources) != R:
            raise ValueError("one source per medium")
        groups, keep, counts = [], [], []
        for sim, src in zip(self.sims, sources):
            s, blocks, k = sim.source_blocks(src)
            if s.energy() == 0:
                raise ValueError("a source has no part inside the grid boundaries")
            groups.append(s)
            keep.append(k)
            counts.append(len(s.values))
        blocks = (_lib.ws_source_block * sum(counts))()
        i = 0
        for s, k in zip(groups, keep):
            for p, v in zip(s.positions, k):
                blocks[i] = _lib.ws_source_block((C.c_int64 * 4)(*[int(a) for a in p]),
                                                 (C.c_int64 * 4)(*[int(a) for a in v.shape]), v.ctypes.data)
                i += 1
        first = self.sims[0]
        o = first._options()
        r = first.roi
        shape = tuple(int(r[1, d] - r[0, d] + 1) for d in range(4))
        if getattr(self, "_hstage", None) is None:
            self._hstage = _lib.HostStage()
        buf = self._hstage.get(R * np.prod(shape))
        cap = o.max_iterations + len(first.wiggles) + 1
        hist = np.zeros((R, cap))
        n_it = np.zeros(R, dtype=np.int64)
        conv = np.zeros(R, dtype=np.int32)
        t0 = time.perf_counter()
        _lib.check(_lib.lib.ws_solver_solve_batch(
            self.h, R, (C.c_int64 * R)(*counts), blocks, _lib.WS_HOST, C.byref(o), buf.ctypes.data, _lib.WS_HOST,
            hist.ctypes.data_as(C.POINTER(C.c_double)), cap, n_it.ctypes.data_as(C.POINTER(C.c_int64)),
            conv.ctypes.data_as(C.POINTER(C.c_int))))
        E = _lib.HostStage.take(buf, (R,) + shape[::-1])
        dt = time.perf_counter() - t0
        del keep
        outs, states = [], []
        for i in range(R):
            Ei = E[i].transpose(3, 2, 1, 0)  # [y, x, z, c], column-major in memory
            if not first.vector:
                Ei = Ei[..., 0]
            outs.append(Ei)
            states.append(SimpleNamespace(source=groups[i], it=int(n_it[i]) + 1, converged=bool(conv[i]),
                                          diff_energy=hist[i, :n_it[i]].copy(), time=dt))
        return outs, states

    def close(self):
        if self.h:
            _lib.lib.ws_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def group_media(problems):
    """Indices of `problems` ((sim, source) pairs) grouped by media_key."""
    groups = {}
    for i, (sim, _) in enumerate(problems):
        groups.setdefault(media_key(sim), []).append(i)
    return list(groups.values())


def solve_media(problems, workers=4, batches=None):
    """problems: list of (sim, source) pairs, one medium each, of any sizes.
    Media that share a grid and set-up are solved together in one batched
    solve (MediaBatch: one launch per kernel for the whole group), groups of
    different sizes concurrently on their own streams.  `batches` (optional):
    MediaBatch objects from an earlier call on the same problems, reused.
    Returns (fields, states, seconds, batches) in the order of `problems`."""
    groups = group_media(problems)
    if batches is None:
        batches = [MediaBatch([problems[i][0] for i in g]) if len(g) > 1 else None for g in groups]

    def run(gi):
        g = groups[gi]
        if batches[gi] is None:
            sim, src = problems[g[0]]
            E, st = sim.exec(src)
            return [E], [st]
        return batches[gi].solve([problems[i][1] for i in g])

    t0 = time.perf_counter()
    if workers <= 1:
        res = [run(gi) for gi in range(len(groups))]
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            res = list(ex.map(run, range(len(groups))))
    dt = time.perf_counter() - t0
    fields, states = [None] * len(problems), [None] * len(problems)
    for g, (Es, sts) in zip(groups, res):
        for i, E, st in zip(g, Es, sts):
            fields[i], states[i] = E, st
    return fields, states, dt, batches
