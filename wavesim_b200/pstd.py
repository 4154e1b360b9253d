"""PSTD: the reference's pseudo-spectral time-domain comparison solver
(PSTD.m), with the time stepping on the GPU (``ws_pstd_*`` in the C ABI).

The set-up follows PSTD.m:22-77 (time step from the stability condition, the
coefficient maps of the damped leapfrog, max_cycles + 100 for the slow
start); ``exec`` runs PSTD.run_algorithm (PSTD.m:79-127) with the step's
FFTs on the same kernels as the modified Born series.
"""
from __future__ import annotations

import ctypes as C
import math
import time
import warnings
from types import SimpleNamespace

import numpy as np

from . import _lib
from .problem import Medium, Source, _pad4


def default_source(ncycle):
    """PSTD.default_source (PSTD.m:130-137): a CW source exp(-2 pi i Ncycle)
    switched on with a raised cosine over the first 100 optical cycles."""
    A = np.exp(-2.0j * np.pi * ncycle)
    return A * (0.5 - 0.5 * np.cos(np.pi * min(ncycle / 100.0, 1.0)))


class PSTD:
    """PSTD.m: E_next = c2 E + c1 E_prev + c3 (ifftn(-|p|^2 fftn(E)) + A S)."""

    default_source = staticmethod(default_source)

    def __init__(self, refractive_index, options):
        o = dict(options)
        # PSTD.m:33-35: the reference demands boundary_type and refuses boundary_strength
        if "boundary_type" not in o or "boundary_strength" in o:
            raise ValueError("options field boundary_type and boundary_strength needs to be specified")
        warnings.warn("The PSTD code is only provided for comparison with wavesim, it is not optimized for real use.")
        o["ACC"] = False
        if not o.get("single_precision", True):
            raise ValueError("the B200 loop runs in complex single precision; single_precision must be true")
        self.options = o
        self.dt_relative = float(o.get("dt_relative", 0.95))
        self.source_amplitude = o.get("source_amplitude", None)  # None: default_source, evaluated in C
        self.lambda_ = float(o.get("lambda", 1.0))
        self.energy_threshold = float(o.get("energy_threshold", 1e-2))
        self.callback_interval = int(o.get("callback_interval", 50))
        self.energy_calculation_interval = min(int(o.get("energy_calculation_interval", 8)),
                                               self.callback_interval)  # Simulation.m:135
        self.max_cycles = o.get("max_cycles", math.inf)
        self.device = int(o.get("device", 0))
        self.sample = Medium(refractive_index, o)
        self.grid = self.sample.grid
        self.N = np.concatenate([self.grid.N, [1]]).astype(np.int64)
        lo = self.sample.Bl + 1
        hi = self.grid.N - self.sample.Br
        if o.get("roi") is None:
            self.roi = np.stack([_pad4(lo), _pad4(hi)])
        else:
            r = np.asarray(o["roi"])
            self.roi = np.stack([_pad4(r[0]), _pad4(r[1])])
            self.roi[:, :3] += lo - 1
        # PSTD.m:44-55: the time step from the stability condition
        dims = 2 if int(np.min(self.grid.N)) == 1 else 3
        self.dtmax = 2 / math.sqrt(dims) / math.pi * self.grid.dx * math.sqrt(self.sample.e_r_min)
        self.dt = self.dt_relative * self.dtmax
        self.iterations_per_cycle = self.lambda_ / self.dt
        # PSTD.m:57-63: coefficients of the damped leapfrog
        self.omega = 2 * math.pi / self.lambda_
        e_r = np.asarray(self.sample.e_r)
        er_re = np.real(e_r).astype(np.float64)
        er_im = np.imag(e_r).astype(np.float64) if np.iscomplexobj(e_r) else np.zeros_like(er_re)
        c2dt = self.dt ** 2 / er_re
        sdt = self.dt * self.omega * er_im / er_re
        self.c1 = ((sdt - 2) / (sdt + 2)).astype(np.float32)
        self.c2 = (4 / (sdt + 2)).astype(np.float32)
        self.c3 = (2 * c2dt / (sdt + 2)).astype(np.float32)
        self.max_cycles = self.max_cycles + 100  # PSTD.m:69
        self._h = None

    def _handle(self):
        if self._h is None:
            N = (C.c_int64 * 3)(*[int(v) for v in self.N[:3]])
            maps = [np.asfortranarray(m) for m in (self.c1, self.c2, self.c3)]
            p = [np.ascontiguousarray(r, dtype=np.float32)
                 for r in (self.grid.px_range, self.grid.py_range, self.grid.pz_range)]
            r = self.roi
            roi = (C.c_int64 * 8)(*[int(r[i, d]) for d in range(4) for i in range(2)])
            h = C.c_void_p()
            _lib.check(_lib.lib.ws_pstd_create(N, *[m.ctypes.data for m in maps], *[a.ctypes.data for a in p], roi,
                                               self.device, C.byref(h)))
            self._h = h
        return self._h

    def close(self):
        if self._h is not None:
            _lib.lib.ws_pstd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def max_iterations(self):
        if "max_iterations" in self.options:
            return int(self.options["max_iterations"])
        if math.isfinite(self.max_cycles):
            return int(math.ceil(self.max_cycles * self.iterations_per_cycle))
        return 10 ** 9

    def exec(self, source, max_iterations=None):
        """Simulation.exec + PSTD.run_algorithm.  Returns (E, state): E on the
        ROI [y, x, z], phase compensated as PSTD.m:125-126; state.it,
        state.diff_energy, state.converged, state.time.  max_iterations
        overrides ceil(max_cycles * iterations_per_cycle); as in
        Simulation.next the run stops there only on a step with real(A) > 0.9."""
        if not isinstance(source, Source):
            raise TypeError("Expecting a Source object as input parameter")
        t0 = time.perf_counter()
        s = source.shift(self.roi[0]).crop(np.ones(4, dtype=np.int64), self.N)
        state = SimpleNamespace(source=s, source_energy=s.energy())
        if state.source_energy == 0:
            warnings.warn("There is no source inside the grid boundaries, expect to get zero field everywhere.")
            return None, state
        blocks = (_lib.ws_source_block * len(s.values))()
        keep = []
        for i, (pos, v) in enumerate(zip(s.positions, s.values)):
            v = np.asfortranarray(v.astype(np.complex64))
            keep.append(v)
            blocks[i] = _lib.ws_source_block((C.c_int64 * 4)(*[int(a) for a in pos]),
                                             (C.c_int64 * 4)(*[int(a) for a in v.shape]), v.ctypes.data)
        h = self._handle()
        o = _lib.ws_pstd_options()
        _lib.lib.ws_pstd_default_options(C.byref(o))
        o.max_iterations = int(max_iterations) if max_iterations is not None else self.max_iterations()
        o.energy_threshold = self.energy_threshold
        o.energy_interval = self.energy_calculation_interval
        o.iterations_per_cycle = self.iterations_per_cycle
        amp_keep = None
        if self.source_amplitude is not None:
            fn = self.source_amplitude

            def _amp(ncycle, re, im, user):
                a = complex(fn(ncycle))
                re[0], im[0] = a.real, a.imag
            amp_keep = _lib.AMPLITUDE(_amp)
            o.amplitude = amp_keep
        r = self.roi
        shape = tuple(int(r[1, d] - r[0, d] + 1) for d in range(3))
        if getattr(self, "_hstage", None) is None:
            self._hstage = _lib.HostStage()
        buf = self._hstage.get(np.prod(shape))
        cap = min(o.max_iterations, 10 ** 6) + 4096
        hist = np.zeros(cap)
        n_it = C.c_int64()
        conv = C.c_int()
        _lib.check(_lib.lib.ws_pstd_run(h, len(s.values), blocks, _lib.WS_HOST, C.byref(o), buf.ctypes.data,
                                        hist.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(n_it),
                                        C.byref(conv)))
        E = _lib.HostStage.take(buf, shape, "F")
        del keep, amp_keep
        state.it = int(n_it.value) + 1
        state.diff_energy = hist[:min(n_it.value, cap)].copy()
        state.converged = bool(conv.value)
        state.time = time.perf_counter() - t0
        return E, state  # column-major in memory, as WaveSim.exec
