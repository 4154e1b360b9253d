"""Problem description: SimulationGrid, Medium and Source of the reference.

Host-side set-up (NumPy, float64) that mirrors the reference's MATLAB classes
so that the arrays handed to the CUDA loop are the ones the reference builds:

* ``SimulationGrid`` - SimulationGrid.m:20-80
* ``Medium``         - Medium.m:15-132
* ``Source``         - Source.m:1-175

Arrays are indexed ``a[y, x, z(, c)]`` like MATLAB's ``a(y, x, z, c)``.
"""
from __future__ import annotations

import math
import warnings

import numpy as np


def _factor(n):
    """Ascending prime factors (MATLAB ``factor``; factor(1) = [1])."""
    n = int(n)
    if n < 2:
        return [n]
    f, p = [], 2
    while p * p <= n:
        while n % p == 0:
            f.append(p)
            n //= p
        p += 1
    return f + ([n] if n > 1 else [])


def efficient_size(n):
    """SimulationGrid.efficient_size (SimulationGrid.m:64-80): smallest size >= n
    whose largest prime factor is <= 11 and, for 3+ factors, whose second
    largest is <= 5."""
    n = int(n)
    while True:
        f = _factor(n)
        if not (f[-1] > 11 or (len(f) > 2 and f[-2] > 5)):
            return n
        n += 1


def symrange(n):
    """SimulationGrid.symrange (SimulationGrid.m:55-63):
    fftshift((0:N-1) - floor(N/2)), where MATLAB's fftshift is a circular
    shift by floor(N/2).  For odd N this is not the FFT bin order (bin 0 gets
    +1); the reference's value is kept so that results agree with it."""
    r = np.arange(n) - n // 2
    return np.roll(r, n // 2)


def _pad3(v, fill):
    v = list(np.ravel(v))
    return np.array(v + [fill] * (3 - len(v)))


def _pad4(v):
    v = [int(x) for x in np.ravel(v)]
    if len(v) > 4:
        raise ValueError("Position and size vectors can be 4-dimensional at most")
    return np.array(v + [1] * (4 - len(v)), dtype=np.int64)


def as_field(a, ndim=3):
    """NumPy array with MATLAB's shape rules: scalars are 1x1, vectors are
    columns, trailing singleton axes added up to ``ndim``."""
    a = np.asarray(a)
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a[:, None]
    while a.ndim < ndim:
        a = a[..., None]
    return a


class SimulationGrid:
    """SimulationGrid.m:20-52."""

    def __init__(self, min_size, dx, periodic):
        min_size = np.ceil(np.asarray(min_size, dtype=float)).astype(np.int64)
        periodic = np.asarray(periodic, dtype=bool)
        N = np.array([v if p else efficient_size(v) for v, p in zip(min_size, periodic)], dtype=np.int64)
        self.N = N
        self.dx = float(dx)
        self.periodic = periodic
        self.padding = N - min_size
        self.y_range, self.x_range, self.z_range = (np.arange(n) * dx for n in N)
        self.dpy, self.dpx, self.dpz = (2 * np.pi / (dx * n) for n in N)
        self.py_range = self.dpy * symrange(N[0])
        self.px_range = self.dpx * symrange(N[1])
        self.pz_range = self.dpz * symrange(N[2])


class Medium:
    """Medium.m:15-132: e_r = n^2 with replicated edges added as boundary."""

    def __init__(self, refractive_index, options, build_field=True):
        """build_field=False: the checks and the grid geometry only (the
        field set-up then runs on the device, WaveSim option device_setup);
        self.n keeps the ROI's refractive index."""
        n = as_field(refractive_index)
        if np.iscomplexobj(n) and (n.imag < 0).any():
            raise ValueError("Medium cannot have gain, imaginary part of refractive index should be positive")
        self.boundary_type = options.get("boundary_type", "ARL")
        bw = np.ravel(options["boundary_widths"])
        ndims = 3 if n.shape[2] > 1 else 2
        if bw.size < ndims:
            raise ValueError("boundary_widths array is too short")
        if bw.size > 3:
            raise ValueError("boundary_widths array is too long")
        if np.any(np.round(bw) != bw):
            raise ValueError("boundary_widths should be integer numbers")
        sz = np.array(n.shape[:3], dtype=np.int64)
        bw2 = _pad3(bw * 2, 0).astype(np.int64)
        self.grid = SimulationGrid(sz + bw2, options["pixel_size"], bw2 == 0)
        extra = self.grid.N - sz
        self.Bl = (extra + 1) // 2   # ceil
        self.Br = extra // 2         # floor
        self.n = n
        if not build_field:
            self.e_r = None
            return
        e_r = n.astype(complex if np.iscomplexobj(n) else float) ** 2
        self.e_r_min = float(np.real(e_r).min())
        self.e_r_max = float(np.real(e_r).max())
        self.e_r_center = 0.5 * (self.e_r_min + self.e_r_max)
        e_r = np.pad(e_r, [(int(a), int(b)) for a, b in zip(self.Bl, self.Br)], mode="edge")
        if self.boundary_type[:3] == "PBL" and (self.Bl != 0).any():
            e_r = self._pbl(e_r, options)
        self.e_r = e_r

    def _pbl(self, e_r, o):
        """Deprecated polynomial boundary layer, Medium.m:83-123."""
        warnings.warn("PBL boundary conditions are deprecated and may be removed in the future: use ARL")
        k0 = np.sqrt(np.mean(e_r)) * 2 * np.pi / (o["lambda"] / o["pixel_size"])
        c = o["boundary_strength"] * k0 ** 2 / (2 * k0)
        order = {"PBL1": 1, "PBL2": 2, "PBL3": 3, "PBL4": 4, "PBL5": 5}.get(o["boundary_type"])
        if order is None:
            raise ValueError("unknown boundary type" + o["boundary_type"])
        roi = np.array(e_r.shape[:3]) - self.Bl - self.Br
        d = [np.concatenate([np.arange(self.Bl[i], 0, -1), np.zeros(roi[i]), np.arange(1, self.Br[i] + 1)])
             for i in range(3)]
        r = np.sqrt(d[0][:, None, None] ** 2 + d[1][None, :, None] ** 2 + d[2][None, None, :] ** 2)
        # N-th order curve: c^(N+2) r^N ((N+1) + (2ik0 - c) r) / (k0^2 sum_{m=0}^{N+1} (N+1)!/m! (cr)^m)
        N = order
        num = c ** (N + 2) * r ** N * ((N + 1) + (2.0j * k0 - c) * r)
        den = sum(math.factorial(N + 1) // math.factorial(m) * (c * r) ** m for m in range(N + 2))
        curve = num / den / k0 ** 2
        if N == 1:
            curve = curve / k0 ** 2  # Medium.m:111 divides PBL1 by k0^2 once more
        return e_r + curve


class Source:
    """Source.m: a list of (1-based position, value block) pairs."""

    def __init__(self, value=None, position=(1, 1, 1, 1)):
        self.positions, self.values = [], []
        if value is not None:
            self.positions.append(_pad4(position))
            self.values.append(as_field(value, 4))

    def __add__(self, other):
        s = Source()
        s.positions = self.positions + other.positions
        s.values = self.values + other.values
        return s

    def energy(self):
        return float(sum(np.sum(np.abs(v) ** 2) for v in self.values))

    def shift(self, pos):
        s = Source()
        s.positions = [p + _pad4(pos) - 1 for p in self.positions]
        s.values = list(self.values)
        return s

    def crop(self, lo, hi):
        """Keep the parts inside [lo, hi] (1-based, inclusive), Source.m:81-103."""
        s = Source()
        lo, hi = _pad4(lo), _pad4(hi)
        for p, v in zip(self.positions, self.values):
            a = np.maximum(lo, p)
            b = np.minimum(hi, p + np.array(v.shape) - 1)
            if (a > b).any():
                continue
            sl = tuple(slice(int(a[d] - p[d]), int(b[d] - p[d] + 1)) for d in range(4))
            s.positions.append(a)
            s.values.append(v[sl])
        return s


class PlaneWave:
    """A plane-wave source block given by a few numbers instead of values (no
    counterpart in the reference, whose Source holds dense arrays): value at
    offset a from the block corner = amplitude exp(i (phase0 + phase . a)),
    phase = phase advance per pixel along (y, x, z).  size and position as
    the shape and position of Source (1-based, ROI coordinates, 4 entries
    with the polarisation last).  Generated on the device
    (ws_solver_solve_plane_waves)."""

    def __init__(self, size, position=(1, 1, 1, 1), amplitude=1.0, phase=(0.0, 0.0, 0.0)):
        self.size = _pad4(np.maximum(np.asarray(size, dtype=np.int64), 1))
        self.position = _pad4(position)
        self.amplitude = complex(amplitude)
        self.phase = np.asarray(list(phase) + [0.0] * (3 - len(phase)), dtype=float)[:3]
        self.phase0 = 0.0

    def values(self):
        """The dense block (for checks and for the host path)."""
        a = [np.arange(int(n)) for n in self.size]
        ph = (self.phase0 + self.phase[0] * a[0][:, None, None, None] + self.phase[1] * a[1][None, :, None, None]
              + self.phase[2] * a[2][None, None, :, None]) + 0 * a[3][None, None, None, :]
        return self.amplitude * np.exp(1j * ph)

    def placed(self, roi0, N):
        """The block shifted to grid coordinates (by the ROI origin roi0, 1-based)
        and cropped to the grid [1, N]; the phase follows the crop.  None if
        nothing is left."""
        pos = self.position + _pad4(roi0) - 1
        lo = np.maximum(pos, 1)
        hi = np.minimum(pos + self.size - 1, _pad4(N))
        if (lo > hi).any():
            return None
        w = PlaneWave(hi - lo + 1, lo, self.amplitude, self.phase)
        w.phase0 = self.phase0 + float(np.dot(self.phase, (lo - pos)[:3]))
        return w
