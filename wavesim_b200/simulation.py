"""WaveSim / WaveSimVector: the reference's solver classes over the CUDA loop.

Mirrors the MATLAB API of the reference (Simulation.m, WaveSimBase.m,
WaveSim.m, WaveSimVector.m): construct with a refractive-index map and an
options dict, then ``E, state = sim.exec(source)``.  Everything before the
loop (epsilon, V, gamma, ARL filters, wiggle descriptors, ROI, source shift
and crop) is computed here on the host exactly as the reference does; the
loop itself (WaveSimBase.m:157-197, the part RunWaveSimAlgorithmMex replaces)
runs in libwavesim_b200.so through ``ws_solver_solve``.

Options (names as in the reference): lambda, pixel_size, boundary_widths,
boundary_type, boundary_strength, energy_threshold, energy_calculation_interval,
max_cycles, callback, callback_interval, roi, epsilon, ACC / wiggle,
single_precision (must be true: the loop is complex FP32), gpu_enabled and
usemex (accepted and ignored).  Added: ``stop_rule`` ('reference' | 'fresh'),
``device`` (CUDA ordinal), ``max_iterations`` (overrides max_cycles),
``use_graph``.
"""
from __future__ import annotations

import ctypes as C
import math
import time
import warnings
from types import SimpleNamespace

import numpy as np

from . import _lib
from .problem import Medium, PlaneWave, Source, _pad4

ALPHA = 0.7  # private/f_mix.m:3


def nuttallwin(n):
    """Symmetric 4-term Blackman-Nuttall window (MATLAB nuttallwin)."""
    if n == 1:
        return np.ones(1)
    t = 2 * np.pi * np.arange(n) / (n - 1)
    return 0.3635819 - 0.4891775 * np.cos(t) + 0.1365995 * np.cos(2 * t) - 0.0106411 * np.cos(3 * t)


def wiggle_perm(flags):
    """private/wiggle_perm.m: sign combinations of the enabled directions, in
    the column order the reference uses to limit wrap-around artefacts."""
    flags = np.asarray(flags, dtype=bool).ravel()
    k = int(flags.sum())
    cols = 2 ** k
    out = np.zeros((flags.size, cols))
    rows = np.flatnonzero(flags)
    for r_i, d in enumerate(rows):
        period = 2 ** r_i
        out[d] = [1.0 if ((c // period) % 2 == 0) else -1.0 for c in range(cols)]
    order = {2: [0, 1, 3, 2], 3: [0, 1, 2, 4, 3, 5, 6, 7]}.get(k, list(range(cols)))
    return out[:, order]


class WaveSim:
    """Scalar modified Born series (WaveSim.m + WaveSimBase.m + Simulation.m)."""

    vector = False

    def __init__(self, refractive_index, options):
        o = dict(options)
        if "wiggle" in o:  # WaveSimBase.m:48-50
            o["ACC"] = o["wiggle"]
        if not o.get("single_precision", True):
            raise ValueError("the B200 loop runs in complex single precision; single_precision must be true")
        self.options = o
        self.lambda_ = float(o.get("lambda", 1.0))
        self.energy_threshold = float(o.get("energy_threshold", 1e-2))
        self.callback_interval = int(o.get("callback_interval", 50))
        self.energy_calculation_interval = min(int(o.get("energy_calculation_interval", 8)),
                                               self.callback_interval)  # Simulation.m:135
        self.max_cycles = o.get("max_cycles", math.inf)
        self.callback = o.get("callback", None)
        self.stop_rule = o.get("stop_rule", "reference")
        self.device = int(o.get("device", 0))
        self.use_graph = bool(o.get("use_graph", True))
        # a warm start whose initial residual is worse than the cold start's is
        # discarded (ratio 1); 0 keeps every start
        self.warm_discard_ratio = float(o.get("warm_discard_ratio", 1.0))

        # device_setup: e_r, V, the ARL window and gamma are built on the GPU
        # (wavesim_b200/csrc/ws_setup.cu) instead of in NumPy; same values
        self.device_setup = bool(o.get("device_setup", False)) and o.get("boundary_type", "ARL") == "ARL"
        self.sample = Medium(refractive_index, o, build_field=not self.device_setup)
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

        k0 = 2 * np.pi / self.lambda_
        self._gamma_host = self._gamma_dev = None
        if self.device_setup:
            eps, k0c = self._setup_on_device(k0, o)
        else:
            k0c = np.sqrt(self.sample.e_r_center) * k0
            if "epsilon" in o:
                eps = float(o["epsilon"])
            else:  # WaveSimBase.m:201-215
                eps = max(float(np.abs(self.sample.e_r * k0 ** 2 - k0c ** 2).max()) / 0.95, 3.0)
            V = self.sample.e_r * k0 ** 2 - k0c ** 2 - 1.0j * eps
            V = V * self._edge_filter()
            self._gamma_host = (1.0j / eps * V).astype(np.complex64)
        self.iterations_per_cycle = self.lambda_ / (2 * k0c / eps)
        self.k02e = np.complex64(k0c ** 2 / eps + 1.0j)
        self.epsilon = np.float32(eps)
        self.k0, self.k0c = k0, k0c
        self.wiggles, self.ACC = self._wiggles(o.get("ACC", True))
        if self.vector:
            if o.get("roi") is None:
                self.roi[1, 3] = 3  # WaveSimVector.m:14-16
            self.N[3] = 3
        self._solver = None

    # WaveSimBase.apply_edge_filters (WaveSimBase.m:217-258): separable ARL window
    def _edge_windows(self):
        """The three 1-D factors (y, x, z) of the ARL edge window."""
        out = [np.ones(int(self.grid.N[d])) for d in range(3)]
        if self.sample.boundary_type != "ARL" or (self.sample.Bl == 0).all():
            return out
        bw = np.ravel(self.options["boundary_widths"])
        linear = bool((self.grid.N > 1).all())
        for d in range(3):
            bl, br = int(self.sample.Bl[d]), int(self.sample.Br[d])
            if bl <= 0:
                continue
            L = int(bw[d])
            if linear:
                win = lambda B: (np.arange(1, B + 1) - 0.21) / (B + 0.66)  # noqa: E731
            else:
                nw = nuttallwin(2 * L - 1)
                win = lambda B, nw=nw: nw[:B]  # noqa: E731
            step = np.concatenate([[0.0], win(L - 1)]) if bl == br else win(L)
            core = int(self.grid.N[d]) - bl - br
            out[d] = np.concatenate([np.zeros(bl - L), step, np.ones(core), step[::-1], np.zeros(br - L)])
        return out

    def _edge_filter(self):
        fy, fx, fz = self._edge_windows()
        return fy[:, None, None] * fx[None, :, None] * fz[None, None, :]

    def _setup_on_device(self, k0, o):
        """e_r statistics, epsilon and gamma on the GPU (ws_setup.cu); returns
        (epsilon, k0c).  The same formulas as the host path, in double."""
        import torch
        dev = torch.device("cuda", self.device)
        n = self.sample.n[..., 0] if self.sample.n.ndim == 4 else self.sample.n
        cplx = bool(np.iscomplexobj(n))
        flat = np.ascontiguousarray(np.ravel(n, order="F").astype(np.complex128 if cplx else np.float64))
        nd = torch.from_numpy(flat.view(np.float64)).to(dev)
        stats = (C.c_double * 3)()
        L = _lib.lib
        _lib.check_setup(L.ws_medium_reduce(nd.data_ptr(), int(cplx), n.size, 0.0, 0.0, stats, None))
        s = self.sample
        s.e_r_min, s.e_r_max = stats[0], stats[1]
        s.e_r_center = 0.5 * (s.e_r_min + s.e_r_max)
        k0c = np.sqrt(s.e_r_center) * k0
        if "epsilon" in o:
            eps = float(o["epsilon"])
        else:  # WaveSimBase.m:201-215
            _lib.check_setup(L.ws_medium_reduce(nd.data_ptr(), int(cplx), n.size, k0 ** 2, k0c ** 2, stats, None))
            eps = max(stats[2] / 0.95, 3.0)
        wins = [torch.from_numpy(w.astype(np.float32)).to(dev) for w in self._edge_windows()]
        gamma = torch.empty(int(np.prod(self.grid.N)), dtype=torch.complex64, device=dev)
        N3 = (C.c_int64 * 3)(*[int(v) for v in self.grid.N])
        R3 = (C.c_int64 * 3)(*[int(v) for v in n.shape])
        lo = (C.c_int64 * 3)(*[int(v) for v in self.sample.Bl])
        _lib.check_setup(L.ws_build_gamma(nd.data_ptr(), int(cplx), R3, N3, lo, wins[0].data_ptr(), wins[1].data_ptr(),
                                          wins[2].data_ptr(), k0 ** 2, k0c ** 2, eps, gamma.data_ptr(), None))
        torch.cuda.synchronize(dev)
        self._gamma_dev = gamma
        return eps, k0c

    @property
    def gamma(self):
        """gamma = (i/epsilon) V F on the full grid, [y, x, z] complex64 (host)."""
        if self._gamma_host is None:
            self._gamma_host = self._gamma_dev.cpu().numpy().reshape(tuple(int(v) for v in self.grid.N), order="F")
        return self._gamma_host

    # WaveSimBase.compute_wiggles / wiggle_descriptor (WaveSimBase.m:272-316)
    def _wiggles(self, acc):
        acc = np.ravel(np.asarray(acc))
        if acc.size == 1:
            acc = ~self.grid.periodic if bool(acc[0]) else np.zeros(3, dtype=bool)
        acc = acc.astype(bool)
        g = self.grid
        se = np.sqrt(self.epsilon)
        out = []
        for w in wiggle_perm(acc).T:
            d = SimpleNamespace(wig=w)
            d.pye = ((g.py_range - g.dpy * w[0] / 4) / se).astype(np.float32)
            d.pxe = ((g.px_range - g.dpx * w[1] / 4) / se).astype(np.float32)
            d.pze = ((g.pz_range - g.dpz * w[2] / 4) / se).astype(np.float32)
            d.gy = np.exp(0.5j * np.pi * w[0] * np.arange(g.N[0]) / g.N[0]).astype(np.complex64)
            d.gx = np.exp(0.5j * np.pi * w[1] * np.arange(g.N[1]) / g.N[1]).astype(np.complex64)
            d.gz = np.exp(0.5j * np.pi * w[2] * np.arange(g.N[2]) / g.N[2]).astype(np.complex64)
            out.append(d)
        return out, acc

    # ------------------------------------------------------------------ C ABI
    def _roi8(self):
        r = self.roi
        return (C.c_int64 * 8)(*[int(r[i, d]) for d in range(4) for i in range(2)])

    def _wiggle_structs(self):
        self._wig_keep = []
        arr = (_lib.ws_wiggle * len(self.wiggles))()
        for i, w in enumerate(self.wiggles):
            parts = [np.ascontiguousarray(a) for a in (w.pxe, w.pye, w.pze, w.gx, w.gy, w.gz)]
            self._wig_keep.extend(parts)
            arr[i] = _lib.ws_wiggle(*[p.ctypes.data for p in parts])
        return arr

    def solver(self):
        """The ws_solver for this medium (created once; set-up uploaded once)."""
        if self._solver is None:
            N = (C.c_int64 * 4)(*[int(v) for v in self.N])
            h = C.c_void_p()
            if self._gamma_dev is not None:
                # everything from device memory: gamma stays where it was built
                import torch
                dev = self._gamma_dev.device
                keep = []
                wig = (_lib.ws_wiggle * len(self.wiggles))()
                for i, w in enumerate(self.wiggles):
                    parts = [torch.from_numpy(np.ascontiguousarray(a).view(np.float32)).to(dev)
                             for a in (w.pxe, w.pye, w.pze, w.gx, w.gy, w.gz)]
                    keep.extend(parts)
                    wig[i] = _lib.ws_wiggle(*[t.data_ptr() for t in parts])
                _lib.check(_lib.lib.ws_solver_create(
                    N, self._gamma_dev.data_ptr(), len(self.wiggles), wig, C.c_float(self.epsilon),
                    _lib.ws_complex(self.k02e.real, self.k02e.imag), self._roi8(), _lib.WS_DEVICE, self.device,
                    C.byref(h)))
                del keep
            else:
                gamma = np.asfortranarray(self.gamma)
                wig = self._wiggle_structs()
                _lib.check(_lib.lib.ws_solver_create(
                    N, gamma.ctypes.data, len(self.wiggles), wig, C.c_float(self.epsilon),
                    _lib.ws_complex(self.k02e.real, self.k02e.imag), self._roi8(), _lib.WS_HOST, self.device,
                    C.byref(h)))
            self._solver = h
        return self._solver

    def close(self):
        if self._solver is not None:
            _lib.lib.ws_solver_destroy(self._solver)
            self._solver = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def source_blocks(self, source):
        """Simulation.exec source handling (Simulation.m:151-161): shift to the
        ROI origin, crop to the grid, cast to complex single (column-major)."""
        if not isinstance(source, Source):
            raise TypeError("Expecting a Source object as input parameter")
        s = source.shift(self.roi[0]).crop(np.ones(4, dtype=np.int64), self.N)
        blocks = (_lib.ws_source_block * max(1, len(s.values)))()
        keep = []
        for i, (p, v) in enumerate(zip(s.positions, s.values)):
            v = np.asfortranarray(v.astype(np.complex64))
            keep.append(v)
            blocks[i] = _lib.ws_source_block((C.c_int64 * 4)(*[int(a) for a in p]),
                                             (C.c_int64 * 4)(*[int(a) for a in v.shape]), v.ctypes.data)
        return s, blocks, keep

    def max_iterations(self):
        if "max_iterations" in self.options:
            return int(self.options["max_iterations"])
        if math.isfinite(self.max_cycles):
            return int(math.ceil(self.max_cycles * self.iterations_per_cycle))
        return 100000  # WaveSimBase.m:127-131

    def roi_medium(self):
        """The (real) refractive index on the ROI, [y, x, z]."""
        r = self.roi
        lo = [int(r[0, d]) - 1 - int(self.sample.Bl[d]) for d in range(3)]  # into the medium as given
        hi = [int(r[1, d]) - int(self.sample.Bl[d]) for d in range(3)]
        n = np.asarray(self.sample.n)
        n = n[..., 0] if n.ndim == 4 else n
        return np.real(n[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]).astype(np.float32)

    def _stage(self):
        """This simulation's pinned staging buffer for solver outputs."""
        if getattr(self, "_hstage", None) is None:
            self._hstage = _lib.HostStage()
        return self._hstage

    def initial_field(self, psi0):
        """A starting field psi0 on the full grid (complex64, column-major, as
        the C ABI takes it).  psi0 is given on the full grid or on the ROI
        ([y, x, z] or [y, x, z, c]); an ROI field is continued into the
        absorbing boundary layers by its edge values under a cos^2 taper that
        reaches zero at the grid edge (a field cut to zero at the ROI edge
        would carry a step there, whose residual costs iterations)."""
        shape = tuple(int(v) for v in self.N)
        p = np.asarray(psi0, np.complex64)
        if p.ndim == 3:
            p = p[..., None]
        if p.shape == shape:
            return np.asfortranarray(p)
        r = self.roi
        lo = [int(r[0, d]) - 1 for d in range(4)]
        hi = [shape[d] - int(r[1, d]) for d in range(4)]
        if tuple(int(r[1, d]) - int(r[0, d]) + 1 for d in range(4)) != p.shape:
            raise ValueError(f"starting field shape {p.shape} matches neither the ROI nor the grid {shape}")
        full = np.pad(p, [(lo[d], hi[d]) for d in range(3)] + [(0, 0)], mode="edge")
        if lo[3] or hi[3]:
            full = np.pad(full, [(0, 0)] * 3 + [(lo[3], hi[3])])
        for d in range(3):
            w = np.ones(shape[d], np.float32)
            if lo[d]:
                w[:lo[d]] = np.cos(0.5 * np.pi * np.arange(lo[d], 0, -1) / (lo[d] + 1)) ** 2
            if hi[d]:
                w[shape[d] - hi[d]:] = np.cos(0.5 * np.pi * np.arange(1, hi[d] + 1) / (hi[d] + 1)) ** 2
            sh = [1, 1, 1, 1]
            sh[d] = shape[d]
            full = full * w.reshape(sh)
        return np.asfortranarray(full.astype(np.complex64))

    def _options(self, output="field"):
        o = _lib.default_options()
        o.max_iterations = self.max_iterations()
        o.energy_threshold = self.energy_threshold
        o.energy_interval = self.energy_calculation_interval
        o.stop_rule = _lib.WS_STOP_FRESH if self.stop_rule == "fresh" else _lib.WS_STOP_REFERENCE
        o.output = _lib.WS_OUTPUT_FIELD if output == "field" else _lib.WS_OUTPUT_EPRIME
        o.use_graph = 1 if self.use_graph else 0
        o.warm_discard_ratio = self.warm_discard_ratio
        return o

    def _warm_input(self, psi0):
        """(pointer owner, memory kind, primed) of a warm start given as a
        host array, a full-grid device tensor, or a model with predict_grid."""
        if hasattr(psi0, "predict_grid"):
            psi0 = psi0.predict_grid(self)
        if hasattr(psi0, "data_ptr"):
            if psi0.numel() != int(np.prod(self.N)):
                raise ValueError("a device warm start must hold the full grid")
            return psi0, _lib.WS_DEVICE
        return self.initial_field(psi0), _lib.WS_HOST

    def exec(self, source, warm_start=None, output="field"):
        """Simulation.exec (Simulation.m:138-190) with the loop on the GPU.
        Returns (E, state): E = E'/gamma on the ROI, indexed [y, x, z] (scalar)
        or [y, x, z, c] (vector), or with output="eprime" the full-grid E'
        that the MEX call returns (WaveSimBase.m:146); column-major in memory
        as the C ABI writes it and as MATLAB holds it (no reordering copy on
        the host); state.it, state.diff_energy, state.converged, state.time.

        warm_start (no counterpart in the reference): an estimate psi0 of the
        field - a host array on the ROI or the full grid, a flat complex64
        device tensor on the full grid (column-major), or a
        wavesim_b200.warmstart.WarmStart model, whose prediction then stays
        on the device.  The loop starts from it, injected over the first
        wiggle cycle as the reference injects its source, and runs to the
        same energy tolerance against the cold first-iteration energy.  A
        start whose initial residual is worse than the cold start's (ROI
        energy above warm_discard_ratio, option, default 1, times the cold
        start's) is given up before its first cycle and the solve reruns
        cold (state.warm_discarded; state.time covers both;
        state.cold_residual_energy, state.warm_residual_energy)."""
        if output not in ("field", "eprime"):
            raise ValueError("output must be 'field' or 'eprime'")
        t0 = time.perf_counter()
        s, blocks, keep = self.source_blocks(source)
        state = SimpleNamespace(source=s, source_energy=s.energy())
        if state.source_energy == 0:
            warnings.warn("There is no source inside the grid boundaries, expect to get zero field everywhere.")
            return None, state
        h = self.solver()
        o = self._options(output)
        init = None
        if warm_start is not None:
            init, o.initial_memory = self._warm_input(warm_start)
            o.initial_field = init.data_ptr() if hasattr(init, "data_ptr") else init.ctypes.data
        cb_keep = None
        if self.callback is not None:
            sim = self

            def _cb(kind, hist, n, thr, user):
                sim.callback(sim, SimpleNamespace(diff_energy=np.ctypeslib.as_array(hist, (n,)).copy(),
                                                  it=int(n), energy_threshold=thr))
            cb_keep = _lib.CALLBACK(_cb)
            o.callback = cb_keep
            o.callback_type = b"Custom"
            o.callback_interval = self.callback_interval
        r = self.roi
        if output == "field":
            shape = tuple(int(r[1, d] - r[0, d] + 1) for d in range(4))
        else:
            shape = tuple(int(v) for v in self.N)
        buf = self._stage().get(np.prod(shape))
        hist = np.zeros(o.max_iterations + len(self.wiggles) + 1)
        n_it = C.c_int64()
        conv = C.c_int()
        _lib.check(_lib.lib.ws_solver_solve(
            h, len(s.values), blocks, _lib.WS_HOST, C.byref(o), buf.ctypes.data, _lib.WS_HOST,
            hist.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n_it), C.byref(conv)))
        E = _lib.HostStage.take(buf, shape, "F")
        del keep, cb_keep
        state.it = int(n_it.value) + 1  # Simulation.next leaves it one past the last iteration
        state.diff_energy = hist[:n_it.value].copy()
        state.converged = bool(conv.value)
        if init is not None:
            cold, warm, disc = C.c_double(), C.c_double(), C.c_int()
            _lib.check(_lib.lib.ws_solver_warm_report(h, 0, C.byref(cold), C.byref(warm), C.byref(disc)))
            state.cold_first_energy, state.warm_cycle_energy = cold.value, warm.value
            state.warm_discarded = bool(disc.value)
            rc_, rw_ = C.c_double(), C.c_double()
            _lib.check(_lib.lib.ws_solver_warm_residual(h, 0, C.byref(rc_), C.byref(rw_)))
            state.cold_residual_energy, state.warm_residual_energy = rc_.value, rw_.value
            del init
            if state.warm_discarded:
                E, st2 = self.exec(source, output=output)
                for k in ("cold_first_energy", "warm_cycle_energy", "cold_residual_energy", "warm_residual_energy"):
                    setattr(st2, k, getattr(state, k))
                st2.warm_discarded, st2.warm_iterations = True, state.it - 1
                st2.time = time.perf_counter() - t0
                return E, st2
        state.time = time.perf_counter() - t0
        if not self.vector:
            E = E[..., 0]
        return E, state

    def exec_batch(self, sources, warm_starts=None):
        """Many sources on this medium in one batched solve (ws_solver_solve_batch).

        Equivalent to ``[self.exec(s) for s in sources]`` - every source runs
        the reference loop and stop rule on its own - but all of them share the
        medium's device data and each kernel launch covers the whole batch.
        warm_starts: None, one starting field per source (host arrays on the
        ROI or the full grid, see exec), or a CUDA tensor of the R full-grid
        starts as column-major rows (device_starts, WarmStart.predict_grid);
        the discarded starts are rerun cold together in one batched solve.
        Returns (list of E, list of state)."""
        t0 = time.perf_counter()
        if sources and all(isinstance(s, PlaneWave) for s in sources):
            return self._exec_plane_waves(sources, warm_starts, t0)
        groups, keep, counts = [], [], []
        for src in sources:
            s, blocks, k = self.source_blocks(src)
            if s.energy() == 0:
                raise ValueError("a source has no part inside the grid boundaries")
            groups.append(s)
            keep.append(k)
            counts.append(len(s.values))
        total = sum(counts)
        blocks = (_lib.ws_source_block * total)()
        i = 0
        for s, k in zip(groups, keep):
            for p, v in zip(s.positions, k):
                blocks[i] = _lib.ws_source_block((C.c_int64 * 4)(*[int(a) for a in p]),
                                                 (C.c_int64 * 4)(*[int(a) for a in v.shape]), v.ctypes.data)
                i += 1
        h = self.solver()
        o = self._options()
        R = len(sources)
        init = self._batch_starts(o, warm_starts, R)
        r = self.roi
        shape = tuple(int(r[1, d] - r[0, d] + 1) for d in range(4))
        buf = self._stage().get(R * np.prod(shape))
        cap = o.max_iterations + len(self.wiggles) + 1
        hist = np.zeros((R, cap))
        n_it = np.zeros(R, dtype=np.int64)
        conv = np.zeros(R, dtype=np.int32)
        _lib.check(_lib.lib.ws_solver_solve_batch(
            h, R, (C.c_int64 * R)(*counts), blocks, _lib.WS_HOST, C.byref(o), buf.ctypes.data, _lib.WS_HOST,
            hist.ctypes.data_as(C.POINTER(C.c_double)), cap, n_it.ctypes.data_as(C.POINTER(C.c_int64)),
            conv.ctypes.data_as(C.POINTER(C.c_int))))
        E = _lib.HostStage.take(buf, (R,) + shape[::-1])  # each field column-major
        del keep, init
        return self._batch_results(h, E, hist, n_it, conv, groups, time.perf_counter() - t0,
                                   warm_starts is not None, lambda idx: self.exec_batch([sources[i] for i in idx]))

    def _batch_starts(self, o, warm_starts, R):
        """Sets the options' starting fields for a batch of R: host arrays
        (one per source, on the ROI or the full grid; see initial_field), or a
        CUDA tensor of R full-grid starts, column-major rows (device_starts,
        WarmStart.predict_grid), passed without a host round trip.  Returns
        what must stay alive during the solve."""
        if warm_starts is None:
            return None
        if len(warm_starts) != R:
            raise ValueError("one warm start per source")
        if hasattr(warm_starts, "data_ptr"):
            if warm_starts.numel() != R * int(np.prod(self.N)) or not warm_starts.is_contiguous():
                raise ValueError("device warm starts must be R contiguous full-grid fields")
            o.initial_field = warm_starts.data_ptr()
            o.initial_memory = _lib.WS_DEVICE
            return warm_starts
        init = np.stack([np.ravel(self.initial_field(w), order="F") for w in warm_starts])
        o.initial_field = init.ctypes.data
        o.initial_memory = _lib.WS_HOST
        return init

    def _batch_results(self, h, E, hist, n_it, conv, srcs, dt, warm, rerun):
        """Fields and states of a batched solve; with warm starts, the warm
        report of each right-hand side, and one batched cold rerun
        (rerun(indices) -> (fields, states)) of the discarded starts."""
        R = len(srcs)
        outs, states = [], []
        for i in range(R):
            Ei = E[i].transpose(3, 2, 1, 0)  # [y, x, z, c], column-major in memory
            if not self.vector:
                Ei = Ei[..., 0]
            outs.append(Ei)
            states.append(SimpleNamespace(source=srcs[i], it=int(n_it[i]) + 1, converged=bool(conv[i]),
                                          diff_energy=hist[i, :n_it[i]].copy(), time=dt))
        if warm:
            for i in range(R):
                cold, wc, disc = C.c_double(), C.c_double(), C.c_int()
                _lib.check(_lib.lib.ws_solver_warm_report(h, i, C.byref(cold), C.byref(wc), C.byref(disc)))
                states[i].cold_first_energy, states[i].warm_cycle_energy = cold.value, wc.value
                states[i].warm_discarded = bool(disc.value)
                rc_, rw_ = C.c_double(), C.c_double()
                _lib.check(_lib.lib.ws_solver_warm_residual(h, i, C.byref(rc_), C.byref(rw_)))
                states[i].cold_residual_energy, states[i].warm_residual_energy = rc_.value, rw_.value
            idx = [i for i in range(R) if states[i].warm_discarded]
            if idx:
                re_E, re_st = rerun(idx)
                for i, e, st in zip(idx, re_E, re_st):
                    outs[i] = e
                    st.warm_discarded, st.warm_iterations = True, states[i].it - 1
                    for k in ("cold_first_energy", "warm_cycle_energy", "cold_residual_energy",
                              "warm_residual_energy"):
                        setattr(st, k, getattr(states[i], k))
                    st.time += dt
                    states[i] = st
        return outs, states


    def _start_windows(self):
        """initial_field's cos^2 tapers (y, x, z) over the boundary layers."""
        if getattr(self, "_swin", None) is None:
            shape = [int(v) for v in self.N]
            r = self.roi
            out = []
            for d in range(3):
                lo, hi = int(r[0, d]) - 1, shape[d] - int(r[1, d])
                w = np.ones(shape[d], np.float32)
                if lo:
                    w[:lo] = np.cos(0.5 * np.pi * np.arange(lo, 0, -1) / (lo + 1)) ** 2
                if hi:
                    w[shape[d] - hi:] = np.cos(0.5 * np.pi * np.arange(1, hi + 1) / (hi + 1)) ** 2
                out.append(w)
            self._swin = out
        return self._swin

    def device_starts(self, fields):
        """initial_field on the device: `fields` is a complex64 CUDA tensor of
        R ROI fields (one row each, column-major as the C ABI writes them);
        returns R full-grid starting fields (rows, column-major), each
        continued into the boundary layers by its edge values under the cos^2
        taper of initial_field."""
        import torch
        shape = [int(v) for v in self.N]
        r = self.roi
        rs = [int(r[1, d] - r[0, d] + 1) for d in range(4)]
        lo = [int(r[0, d]) - 1 for d in range(4)]
        R = fields.shape[0]
        dev = fields.device
        t = fields.reshape(R, rs[3], rs[2], rs[1], rs[0])  # [rhs, c, z, x, y]
        win = self._start_windows()
        for d, axis in ((0, 4), (1, 3), (2, 2)):
            if rs[d] != shape[d]:
                idx = (torch.arange(shape[d], device=dev) - lo[d]).clamp(0, rs[d] - 1)
                t = t.index_select(axis, idx)
            if (win[d] != 1).any():
                sh = [1, 1, 1, 1, 1]
                sh[axis] = shape[d]
                t = t * torch.from_numpy(win[d]).to(dev).view(sh)
        if rs[3] != shape[3]:
            full = torch.zeros((R, shape[3]) + tuple(t.shape[2:]), dtype=t.dtype, device=dev)
            full[:, lo[3]:lo[3] + rs[3]] = t
            t = full
        return t.reshape(R, -1).contiguous()

    def _exec_plane_waves(self, waves, warm_starts, t0, keep_device=False):
        """exec_batch for PlaneWave sources: the blocks are generated on the
        device (ws_solver_solve_plane_waves).  warm_starts may also be a CUDA
        tensor of full-grid starts (device_starts); keep_device=True also
        returns the fields as a CUDA tensor (one row each, column-major)."""
        R = len(waves)
        arr = (_lib.ws_plane_wave * R)()
        for i, w in enumerate(waves):
            pw = w.placed(self.roi[0], self.N)
            if pw is None:
                raise ValueError("a source has no part inside the grid boundaries")
            arr[i] = _lib.ws_plane_wave((C.c_int64 * 4)(*[int(a) for a in pw.position]),
                                        (C.c_int64 * 4)(*[int(a) for a in pw.size]),
                                        _lib.ws_complex(pw.amplitude.real, pw.amplitude.imag),
                                        (C.c_double * 3)(*[float(a) for a in pw.phase]), pw.phase0)
        h = self.solver()
        o = self._options()
        init = self._batch_starts(o, warm_starts, R)
        r = self.roi
        shape = tuple(int(r[1, d] - r[0, d] + 1) for d in range(4))
        cap = o.max_iterations + len(self.wiggles) + 1
        hist = np.zeros((R, cap))
        n_it = np.zeros(R, dtype=np.int64)
        conv = np.zeros(R, dtype=np.int32)
        Edev = None
        if keep_device:
            import torch
            Edev = torch.empty((R, int(np.prod(shape))), dtype=torch.complex64,
                               device=torch.device("cuda", self.device))
            out, mem = Edev.data_ptr(), _lib.WS_DEVICE
        else:
            buf = self._stage().get(R * np.prod(shape))
            out, mem = buf.ctypes.data, _lib.WS_HOST
        _lib.check(_lib.lib.ws_solver_solve_plane_waves(
            h, R, arr, C.byref(o), out, mem, hist.ctypes.data_as(C.POINTER(C.c_double)), cap,
            n_it.ctypes.data_as(C.POINTER(C.c_int64)), conv.ctypes.data_as(C.POINTER(C.c_int))))
        del init
        if keep_device:
            import torch
            buf = self._stage().get(Edev.numel())
            torch.from_numpy(buf).copy_(Edev.reshape(-1))
        E = _lib.HostStage.take(buf, (R,) + shape[::-1])
        outs, states = self._batch_results(
            h, E, hist, n_it, conv, list(waves), time.perf_counter() - t0, warm_starts is not None,
            lambda idx: self._exec_plane_waves([waves[i] for i in idx], None, time.perf_counter()))
        if not keep_device:
            return outs, states
        for i, st in enumerate(states):
            if getattr(st, "warm_discarded", False):  # the cold rerun's field replaces the discarded run's
                import torch
                Edev[i] = torch.from_numpy(np.ravel(np.asarray(outs[i], np.complex64), order="F")).to(Edev.device)
        return outs, states, Edev


class WaveSimVector(WaveSim):
    """Vector (Maxwell) MBS with the dyadic Green's function (WaveSimVector.m)."""

    vector = True
