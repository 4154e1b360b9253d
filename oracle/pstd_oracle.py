"""CPU oracle for the pseudo-spectral time-domain (PSTD) solver of IvoVellekoop/wavesim.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` may import this module; the product
(``wavesim_b200``) never does.

A NumPy/SciPy restatement of ``PSTD.m`` (the reference's comparison solver)
on top of the ``Simulation.m`` / ``Medium.m`` / ``Source.m`` restatements in
``oracle/mbs_oracle.py``:

* constructor (``PSTD.m:22-77``): option checks, time step
  dt = dt_relative * 2 / sqrt(D) / pi * dx * sqrt(e_r_min), the coefficient
  maps c1, c2, c3 of the damped leapfrog, the spectral Laplacian
  -(px^2 + py^2 + pz^2), max_cycles + 100 for the slow start;
* ``run_algorithm`` (``PSTD.m:79-127``): E_next = c2 E + c1 E_prev +
  c3 (ifftn(k fftn(E)) + A S), the step energy |E_next - E e^{i(arg A - arg A_prev)}|^2
  over the ROI divided by |A|^2, termination only once real(A) > 0.9, and the
  final phase compensation exp(-i arg A(it));
* ``default_source`` (``PSTD.m:130-137``).

Precision: ``single_precision=True`` (the reference default) keeps the fields
in complex64 with single-precision FFTs; the coefficient maps are computed in
float64 and rounded to float32 as MATLAB does when it combines them with
single arrays.

Parity status: no golden output of the reference's PSTD exists and MATLAB is
not installed; the restatement is checked against the MBS restatement (itself
pinned to the reference's analytic solution) on an absorbing periodic medium,
where both solve the same Helmholtz equation (tests/test_pstd_oracle.py).
"""
from __future__ import annotations

import math
import warnings

import numpy as np
import scipy.fft as sfft

from .mbs_oracle import Medium, State, make4


def default_source(ncycle):
    """PSTD.m:130-137: CW source exp(-2 pi i Ncycle), switched on with a
    raised cosine over the first 100 cycles."""
    A = np.exp(-2.0j * np.pi * ncycle)
    return A * (0.5 - 0.5 * np.cos(np.pi * min(ncycle / 100.0, 1.0)))


class PSTD:
    """PSTD.m restated (scalar fields)."""

    def __init__(self, refractive_index, opt):
        opt = dict(opt)
        if "boundary_type" not in opt or "boundary_strength" in opt:  # PSTD.m:33-35
            raise ValueError("options field boundary_type and boundary_strength needs to be specified")
        opt["ACC"] = False  # PSTD.m:36
        self.dt_relative = float(opt.get("dt_relative", 0.95))
        self.source_amplitude = opt.get("source_amplitude", default_source)
        self.lambda_ = float(opt.get("lambda", 1.0))
        self.single_precision = bool(opt.get("single_precision", True))
        self.callback_interval = opt.get("callback_interval", 50)
        self.energy_threshold = float(opt.get("energy_threshold", 1e-2))
        self.energy_calculation_interval = min(opt.get("energy_calculation_interval", 8), self.callback_interval)
        self.max_cycles = opt.get("max_cycles", math.inf)
        self.rdtype = np.float32 if self.single_precision else np.float64
        self.cdtype = np.complex64 if self.single_precision else np.complex128
        self.sample, self.grid = Medium.create(refractive_index, opt)  # Simulation.m:111
        self.N = np.concatenate([self.grid.N, [1]]).astype(np.int64)
        default_roi = np.stack([self.sample.Bl + 1, self.grid.N - self.sample.Br])
        roi_opt = opt.get("roi", None)
        if roi_opt is None:
            self.roi = np.stack([make4(default_roi[0]), make4(default_roi[1])])
        else:
            roi_opt = np.asarray(roi_opt)
            self.roi = np.stack([make4(roi_opt[0]), make4(roi_opt[1])])
            self.roi[:, :3] += default_roi[0] - 1
        # PSTD.m:44-55: time step from the stability condition
        dims = 2 if np.min(self.grid.N) == 1 else 3
        e_r = np.asarray(self.sample.e_r)
        self.dtmax = 2 / np.sqrt(dims) / np.pi * self.grid.dx * np.sqrt(self.sample.e_r_min)
        self.dt = self.dt_relative * self.dtmax
        self.iterations_per_cycle = self.lambda_ / self.dt
        # PSTD.m:57-63
        self.omega = 2 * np.pi / self.lambda_
        er_re = np.real(e_r).astype(np.float64)
        er_im = np.imag(e_r).astype(np.float64) if np.iscomplexobj(e_r) else np.zeros_like(er_re)
        c2dt = self.dt ** 2 / er_re
        sdt = self.dt * self.omega * er_im / er_re
        self.c1 = ((sdt - 2) / (sdt + 2)).astype(self.rdtype)
        self.c2 = (4 / (sdt + 2)).astype(self.rdtype)
        self.c3 = (2 * c2dt / (sdt + 2)).astype(self.rdtype)
        # PSTD.m:66-69: Laplacian in k space
        px = self.grid.px_range.reshape(1, -1, 1)
        py = self.grid.py_range.reshape(-1, 1, 1)
        pz = self.grid.pz_range.reshape(1, 1, -1)
        self.koperator = (-px ** 2 - py ** 2 - pz ** 2).astype(self.rdtype)
        self.max_cycles = self.max_cycles + 100  # PSTD.m:69

    def crop_field(self, E):
        r = self.roi
        return E[r[0, 0] - 1:r[1, 0], r[0, 1] - 1:r[1, 1], r[0, 2] - 1:r[1, 2]]

    def next(self, state, can_terminate):
        """Simulation.m:193-217."""
        state.diff_energy.append(state.last_step_energy)
        d = state.diff_energy
        ratio = d[-1] / d[0] if d[0] != 0 else (math.nan if d[-1] == 0 else math.inf)
        if can_terminate and ratio < self.energy_threshold:
            state.has_next, state.converged = False, True
        elif can_terminate and state.it >= state.max_iterations:
            state.has_next, state.converged = False, False
        else:
            state.has_next = True
        state.calculate_energy = (state.it - 1) % self.energy_calculation_interval == 0
        state.it += 1
        return state

    def exec(self, source, max_iterations=None):
        """Simulation.exec + PSTD.run_algorithm.  ``max_iterations`` overrides
        ceil(max_cycles * iterations_per_cycle)."""
        state = State()
        state.source = source.cast(self.cdtype).shift(self.roi[0]).crop(
            np.stack([np.ones(4, dtype=np.int64), self.N]))
        state.source_energy = state.source.energy()
        if state.source_energy == 0:
            warnings.warn("There is no source inside the grid boundaries, expect to get zero field everywhere.")
            return None, state
        if max_iterations is not None:
            state.max_iterations = max_iterations
        else:
            state.max_iterations = math.ceil(self.max_cycles * self.iterations_per_cycle) \
                if math.isfinite(self.max_cycles) else math.inf
        shape = tuple(int(v) for v in self.N[:3])
        E = np.zeros(shape, dtype=self.cdtype)
        E_prev = np.zeros(shape, dtype=self.cdtype)
        A = 1.0
        while state.has_next:
            ncycle = state.it / self.iterations_per_cycle
            A_prev = A
            A = complex(self.source_amplitude(ncycle))
            Etmp = sfft.ifftn(self.koperator * sfft.fftn(E, axes=(0, 1, 2), workers=-1), axes=(0, 1, 2),
                              workers=-1).astype(self.cdtype)
            Etmp = state.source.add_to(Etmp, A)
            E_next = self.c2 * E + self.c1 * E_prev + self.c3 * Etmp
            if state.calculate_energy:
                ps = np.exp(1.0j * (np.angle(A) - np.angle(A_prev)))
                dif = self.crop_field(E_next - E * self.cdtype(ps))
                state.last_step_energy = float(np.sum(np.abs(dif) ** 2, dtype=np.float64)) / abs(A) ** 2
            E_prev = E
            E = E_next
            can_terminate = A.real > 0.9  # MATLAB compares the real part of a complex A
            state = self.next(state, can_terminate)
        A_next = complex(self.source_amplitude(state.it / self.iterations_per_cycle))
        state.E = E
        return self.crop_field(E) * np.exp(-1.0j * np.angle(A_next)), state
