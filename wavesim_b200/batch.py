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
        E = np.empty((R,) + shape[::-1], dtype=np.complex64)
        cap = o.max_iterations + len(first.wiggles) + 1
        hist = np.zeros((R, cap))
        n_it = np.zeros(R, dtype=np.int64)
        conv = np.zeros(R, dtype=np.int32)
        t0 = time.perf_counter()
        _lib.check(_lib.lib.ws_solver_solve_batch(
            self.h, R, (C.c_int64 * R)(*counts), blocks, _lib.WS_HOST, C.byref(o), E.ctypes.data, _lib.WS_HOST,
            hist.ctypes.data_as(C.POINTER(C.c_double)), cap, n_it.ctypes.data_as(C.POINTER(C.c_int64)),
            conv.ctypes.data_as(C.POINTER(C.c_int))))
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
