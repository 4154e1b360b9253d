"""CPU oracle for the modified Born series (MBS) hot path of IvoVellekoop/wavesim.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` may import this module; the
product (``wavesim_b200``) never does.

This is a NumPy/SciPy restatement, operation by operation, of the MATLAB code of
the reference (paths are relative to the reference project):

* ``Simulation.m``       - option copy, ROI, ``exec``, ``next`` (stop rule), ``energy``
* ``Medium.m``           - e_r = n^2, replicate padding, PBL boundaries
* ``SimulationGrid.m``   - efficient FFT sizes, coordinate and Fourier ranges
* ``WaveSimBase.m``      - epsilon, V, gamma, ARL edge filters, wiggles, the loop
* ``WaveSim.m`` / ``WaveSimVector.m`` - scalar and dyadic propagators
* ``private/*.m``        - f_wiggle, f_g0_scalar, f_g0_vector, f_mix, wiggle_perm
* ``Source.m``           - block sources: shift, crop, energy, add_to

Arrays use NumPy index order ``a[y, x, z(, component)]``, the same subscripts as
MATLAB's ``a(y, x, z, c)``; ``to_matlab_layout`` gives the column-major memory
order that the C-ABI of ``wavesim_b200`` expects.

Precision: ``single_precision=True`` (the reference default,
``Simulation.m:31``) runs the loop in complex64 with ``scipy.fft`` in single
precision, emulating the reference's GPU path; ``False`` runs it in complex128
(the FP64 oracle).  Set-up quantities are computed in float64 and cast as the
reference's ``data_array`` does (``Simulation.m:221-252``).

Parity status: pinned by the reference's own known-answer function
``utilities/homogeneous_medium_analytic_solution.m`` (restated in
``oracle/analytic.py`` and checked in ``tests/test_oracle.py``).  MATLAB is not
installed on this machine, so the restatement is not pinned against MATLAB
execution itself, and MATLAB's ``fftn``/``ifftn`` (FFTW / cuFFT, closed) are
replaced by ``scipy.fft``.
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

ALPHA = 0.7  # private/f_mix.m:3


# ----------------------------------------------------------------------------
# small MATLAB helpers
# ----------------------------------------------------------------------------
def make3(sz, pad):
    """Simulation.m:352-361 - row vector with exactly 3 elements (padded)."""
    sz = list(np.ravel(sz))
    while len(sz) < 3:
        sz.append(pad)
    return np.array(sz)


def make4(sz):
    """Simulation.m:363-379 - 4-element size/position vector, padded with 1."""
    sz = list(np.ravel(sz))
    if len(sz) > 4:
        raise ValueError("Position and size vectors can be 4-dimensional at most")
    while len(sz) < 4:
        sz.append(1)
    return np.array(sz, dtype=np.int64)


def matlab_size4(a):
    """size() of a MATLAB array as a 4-vector (trailing singletons filled)."""
    return make4(np.shape(np.asarray(a)) if np.ndim(a) >= 1 else [1, 1])


def as_matlab_array(a, ndim=3):
    """Give a NumPy array the MATLAB shape convention: at least 2-D, column
    vectors for 1-D input (MATLAB ``ones(N,1)``), trailing singleton axes up
    to ``ndim``."""
    a = np.asarray(a)
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a.reshape(-1, 1)
    while a.ndim < ndim:
        a = a[..., None]
    return a


def prime_factors(n):
    """MATLAB ``factor`` (ascending prime factors; factor(1) == 1)."""
    n = int(n)
    if n <= 1:
        return [n]
    out, p = [], 2
    while p * p <= n:
        while n % p == 0:
            out.append(p)
            n //= p
        p += 1
    if n > 1:
        out.append(n)
    return out


def nuttallwin(n):
    """Symmetric 4-term Blackman-Nuttall window, as MATLAB ``nuttallwin(N)``
    (Nuttall 1981, coefficients a0..a3 below)."""
    a0, a1, a2, a3 = 0.3635819, 0.4891775, 0.1365995, 0.0106411
    if n == 1:
        return np.ones(1)
    k = np.arange(n)
    t = 2.0 * np.pi * k / (n - 1)
    return a0 - a1 * np.cos(t) + a2 * np.cos(2 * t) - a3 * np.cos(3 * t)


def tukeywin(n, r=0.5):
    """MATLAB ``tukeywin(N, r)`` (tapered cosine), used by the Mie example
    (examples/mie_sphere/run_mie_sphere_simulation.m:16-17)."""
    if r <= 0:
        return np.ones(n)
    if r >= 1:
        return 0.5 * (1 - np.cos(2 * np.pi * np.arange(n) / (n - 1)))
    x = np.linspace(0, 1, n)
    w = np.ones(n)
    per = r / 2
    tl = np.floor(per * (n - 1)) + 1
    th = n - tl + 1
    idx = np.arange(n)
    left = idx < tl
    right = idx >= th - 1
    w[left] = 0.5 * (1 + np.cos(np.pi / per * (x[left] - per)))
    w[right] = 0.5 * (1 + np.cos(np.pi / per * (x[right] - 1 + per)))
    return w


def gausswin(n, alpha=2.5):
    """MATLAB ``gausswin(N, alpha)``."""
    k = np.arange(n) - (n - 1) / 2
    return np.exp(-0.5 * (alpha * k / ((n - 1) / 2)) ** 2)


# ----------------------------------------------------------------------------
# SimulationGrid.m
# ----------------------------------------------------------------------------
def symrange(n):
    """SimulationGrid.m:55-63 - fftshift((0:N-1) - floor(N/2))."""
    return np.fft.fftshift(np.arange(n) - n // 2)


def efficient_size(min_size):
    """SimulationGrid.m:64-80 - next size whose prime factors allow a fast FFT:
    largest factor <= 11 and, with more than two factors, second largest <= 5."""
    out = []
    for s in np.ravel(min_size):
        s = int(s)
        f = prime_factors(s)
        while f[-1] > 11 or (len(f) > 2 and f[-2] > 5):
            s += 1
            f = prime_factors(s)
        out.append(s)
    return np.array(out, dtype=np.int64)


@dataclass
class SimulationGrid:
    """SimulationGrid.m:20-52."""

    N: np.ndarray
    dx: float
    periodic: np.ndarray
    padding: np.ndarray = None
    x_range: np.ndarray = None
    y_range: np.ndarray = None
    z_range: np.ndarray = None
    dpx: float = 0.0
    dpy: float = 0.0
    dpz: float = 0.0
    px_range: np.ndarray = None
    py_range: np.ndarray = None
    pz_range: np.ndarray = None

    @classmethod
    def create(cls, min_size, dx, periodic):
        min_size = np.ceil(np.asarray(min_size, dtype=float)).astype(np.int64)  # :34
        periodic = np.asarray(periodic, dtype=bool)
        N = min_size.copy()
        if np.any(~periodic):
            N[~periodic] = efficient_size(min_size[~periodic])  # :37
        g = cls(N=N, dx=float(dx), periodic=periodic)
        g.padding = N - min_size  # :40
        g.x_range = np.arange(N[1]) * dx  # :42
        g.y_range = np.arange(N[0]) * dx
        g.z_range = np.arange(N[2]) * dx
        g.dpx = 2 * np.pi / (dx * N[1])  # :45-47
        g.dpy = 2 * np.pi / (dx * N[0])
        g.dpz = 2 * np.pi / (dx * N[2])
        g.px_range = g.dpx * symrange(N[1])  # :48-50
        g.py_range = g.dpy * symrange(N[0])
        g.pz_range = g.dpz * symrange(N[2])
        return g


# ----------------------------------------------------------------------------
# Medium.m
# ----------------------------------------------------------------------------
def _pbl_curve(kind, c, k0):
    """Medium.m:98-114 - polynomial boundary layer curves (deprecated PBL)."""
    if kind == "PBL5":
        return lambda r: 1 / k0**2 * (c**7 * r**5 * (6.0 + (2.0j * k0 - c) * r)) / (
            720 + 720 * c * r + 360 * c**2 * r**2 + 120 * c**3 * r**3 + 30 * c**4 * r**4
            + 6 * c**5 * r**5 + c**6 * r**6)
    if kind == "PBL4":
        return lambda r: 1 / k0**2 * (c**6 * r**4 * (5.0 + (2.0j * k0 - c) * r)) / (
            120 + 120 * c * r + 60 * c**2 * r**2 + 20 * c**3 * r**3 + 5 * c**4 * r**4 + c**5 * r**5)
    if kind == "PBL3":
        return lambda r: 1 / k0**2 * (c**5 * r**3 * (4.0 + (2.0j * k0 - c) * r)) / (
            24 + 24 * c * r + 12 * c**2 * r**2 + 4 * c**3 * r**3 + c**4 * r**4)
    if kind == "PBL2":
        return lambda r: 1 / k0**2 * (c**4 * r**2 * (3.0 + (2.0j * k0 - c) * r)) / (
            6 + 6 * c * r + 3 * c**2 * r**2 + c**3 * r**3)
    if kind == "PBL1":
        return lambda r: 1 / k0**2 * (c**3 * r * (2.0 + (2.0j * k0 - c) * r)) / (
            2.0 + 2.0 * c * r + c**2 * r**2) / k0**2
    raise ValueError("unknown boundary type" + kind)


@dataclass
class Medium:
    """Medium.m:15-132."""

    boundary_type: str
    e_r: np.ndarray
    e_r_min: float
    e_r_max: float
    e_r_center: float
    Bl: np.ndarray
    Br: np.ndarray

    @classmethod
    def create(cls, refractive_index, opt):
        n = as_matlab_array(refractive_index)
        if np.iscomplexobj(n) and np.min(n.imag) < 0:  # :37-39
            raise ValueError("Medium cannot have gain, imaginary part of refractive index should be positive")
        boundary_type = opt.get("boundary_type", "ARL")  # :42-44
        bw_in = np.ravel(opt["boundary_widths"])
        nd = 3 if (np.ndim(refractive_index) >= 3 and np.shape(refractive_index)[2] > 1) else 2  # MATLAB ndims
        assert bw_in.size >= nd, "boundary_widths array is too short"  # :48
        assert bw_in.size <= 3, "boundary_widths array is too long"  # :49
        assert np.all(np.round(bw_in) == bw_in), "boundary_widths should be integer numbers"  # :50
        e_r = n.astype(np.complex128) ** 2 if np.iscomplexobj(n) else n.astype(np.float64) ** 2  # :53
        e_r_min = float(np.min(np.real(e_r)))  # :54-56
        e_r_max = float(np.max(np.real(e_r)))
        e_r_center = (e_r_min + e_r_max) / 2
        sz = make3(e_r.shape[:3], 1).astype(np.int64)  # :61
        bw = make3(bw_in * 2, 0).astype(np.int64)  # :62
        grid = SimulationGrid.create(sz + bw, opt["pixel_size"], bw == 0)  # :63
        Bl = np.ceil((grid.N - sz) / 2).astype(np.int64)  # :67
        Br = np.floor((grid.N - sz) / 2).astype(np.int64)  # :68
        med = cls(boundary_type, None, e_r_min, e_r_max, e_r_center, Bl, Br)
        med.e_r = med._add_boundary_layer(e_r, opt)  # :71
        return med, grid

    def _add_boundary_layer(self, e_r, opt):
        """Medium.m:75-82."""
        e_r = Medium.extrapolate(e_r, self.Bl, self.Br)
        if self.boundary_type[:3] == "PBL" and np.any(self.Bl != 0):
            e_r = self._polynomial_boundary_layer(e_r, opt)
        return e_r

    def _polynomial_boundary_layer(self, e_r, opt):
        """Medium.m:83-123 (deprecated PBL absorption)."""
        warnings.warn("PBL boundary conditions are deprecated and may be removed in the future: use ARL")
        e_0 = np.mean(e_r)
        k0 = np.sqrt(e_0) * 2 * np.pi / (opt["lambda"] / opt["pixel_size"])
        c = opt["boundary_strength"] * k0**2 / (2 * k0)
        f = _pbl_curve(opt["boundary_type"], c, k0)
        roi_size = make3(e_r.shape[:3], 1) - self.Bl - self.Br
        x = np.concatenate([np.arange(self.Bl[1], 0, -1), np.zeros(roi_size[1]), np.arange(1, self.Br[1] + 1)])
        y = np.concatenate([np.arange(self.Bl[0], 0, -1), np.zeros(roi_size[0]), np.arange(1, self.Br[0] + 1)])
        z = np.concatenate([np.arange(self.Bl[2], 0, -1), np.zeros(roi_size[2]), np.arange(1, self.Br[2] + 1)])
        r = np.sqrt(x[None, :, None] ** 2 + y[:, None, None] ** 2 + z[None, None, :] ** 2)
        return e_r + f(r)

    @staticmethod
    def extrapolate(e_r, Bl, Br):
        """Medium.m:126-132 - padarray(..., 'replicate') pre Bl and post Br."""
        pad = [(int(Bl[d]), int(Br[d])) for d in range(3)]
        return np.pad(e_r, pad, mode="edge")


# ----------------------------------------------------------------------------
# Source.m
# ----------------------------------------------------------------------------
class Source:
    """Source.m:1-175 - list of rectangular source blocks.

    ``positions`` are 1-based 4-vectors (y, x, z, polarization); ``values`` are
    arrays with MATLAB subscripts (y, x, z, c)."""

    def __init__(self, value=None, position=(1, 1, 1, 1)):
        if value is None:  # Source.m:39-44
            self.positions, self.values = [], []
        else:
            self.positions = [make4(position)]
            self.values = [np.asarray(value)]

    def __add__(self, other):  # Source.m:48-55
        c = Source()
        c.positions = self.positions + other.positions
        c.values = self.values + other.values
        return c

    def copy(self):
        c = Source()
        c.positions = [p.copy() for p in self.positions]
        c.values = [v.copy() for v in self.values]
        return c

    @staticmethod
    def _v4(v):
        return as_matlab_array(v, 4)

    def energy(self):
        """Source.m:57-67."""
        return float(sum(np.sum(np.abs(v) ** 2) for v in self.values))

    def shift(self, pos):
        """Source.m:69-79."""
        s = self.copy()
        s.positions = [p + make4(pos) - 1 for p in s.positions]
        return s

    def crop(self, roi):
        """Source.m:81-103; roi = [[1,1,1,1],[Ny,Nx,Nz,Nc]] (1-based inclusive)."""
        roi = np.asarray(roi, dtype=np.int64)
        s = Source()
        for pos, val in zip(self.positions, self.values):
            v4 = self._v4(val)
            sz = make4(v4.shape)
            tlt = np.maximum(roi[0], pos)
            brt = np.minimum(roi[1], pos + sz - 1)
            if np.any(tlt > brt):
                continue
            tls = tlt - pos
            brs = brt - pos + 1
            s.values.append(v4[tls[0]:brs[0], tls[1]:brs[1], tls[2]:brs[2], tls[3]:brs[3]])
            s.positions.append(tlt)
        return s

    def cast(self, dtype):
        s = self.copy()
        s.values = [self._v4(v).astype(dtype) for v in s.values]
        return s

    def add_to(self, E, A):
        """Source.m:139-172 - E(block) = E(block) + A*val (copy, not in place)."""
        E = E.copy()
        E4 = E if E.ndim == 4 else E[..., None]
        for pos, val in zip(self.positions, self.values):
            v4 = self._v4(val)
            t = pos - 1
            b = t + make4(v4.shape)
            E4[t[0]:b[0], t[1]:b[1], t[2]:b[2], t[3]:b[3]] += (A * v4).astype(E.dtype)
        return E

    def dense(self, shape4, dtype=np.complex128):
        """The blocks summed into one dense array of shape ``shape4``."""
        D = np.zeros(shape4, dtype=dtype)
        return self.add_to(D, 1.0)


# ----------------------------------------------------------------------------
# private/*.m element-wise kernels
# ----------------------------------------------------------------------------
def f_wiggle(E, g1, g2, g3):
    """private/f_wiggle.m:5 - E .* g1 .* g2 .* g3."""
    return E * g1 * g2 * g3


def f_g0_scalar(E, pxe2, pye2, pze2k0e):
    """private/f_g0_scalar.m:6 - E ./ (pxe2 + pye2 + pze2k0e)."""
    return E / (pxe2 + pye2 + pze2k0e)


def f_g0_vector(fEx, fEy, fEz, px, py, pz, k0e):
    """private/f_g0_vector.m:4-8 - dyadic Green's function."""
    div = (px * fEx + py * fEy + pz * fEz) / k0e
    g0_k = 1 / (px**2 + py**2 + pz**2 - k0e)
    return g0_k * (fEx - px * div), g0_k * (fEy - py * div), g0_k * (fEz - pz * div)


def f_mix(Ediff, Eprop, gamma):
    """private/f_mix.m:3-4 - (1 - a*gamma) .* Ediff - 1i*a*gamma.^2 .* Eprop."""
    a = ALPHA
    return (1 - a * gamma) * Ediff - 1.0j * a * gamma**2 * Eprop


def wiggle_perm(wiggle_flags):
    """private/wiggle_perm.m:1-28 - all sign combinations of the enabled
    wiggle directions, in the reference's column order."""
    flags = np.asarray(wiggle_flags, dtype=bool).ravel()
    n_dir = flags.size
    n_w = int(flags.sum())
    ws = np.zeros((n_dir, 2**n_w))
    cols = np.arange(1, 2**n_w + 1)
    rows = np.arange(1, n_w + 1)[:, None]
    ws[flags, :] = (-1.0) ** (np.ceil(cols[None, :] / 2.0 ** (rows - 1)) + 1)  # :16
    ind = np.arange(2**n_w)
    if n_w == 2:
        ind = np.array([1, 2, 4, 3]) - 1  # :22
    elif n_w == 3:
        ind = np.array([1, 2, 3, 5, 4, 6, 7, 8]) - 1  # :24
    return ws[:, ind]


# ----------------------------------------------------------------------------
# WaveSimBase.m / WaveSim.m / WaveSimVector.m
# ----------------------------------------------------------------------------
@dataclass
class Wiggle:
    """WaveSimBase.m:300-316 - per-wiggle shifted Fourier coordinates and ramps."""

    wig: np.ndarray
    pxe: np.ndarray  # (Nx,)
    pye: np.ndarray  # (Ny,)
    pze: np.ndarray  # (Nz,)
    gx: np.ndarray
    gy: np.ndarray
    gz: np.ndarray


@dataclass
class State:
    it: int = 1
    max_iterations: float = math.inf
    diff_energy: list = field(default_factory=list)
    last_step_energy: float = math.inf
    calculate_energy: bool = True
    has_next: bool = True
    converged: bool = False
    E: np.ndarray = None
    dE: np.ndarray = None
    source: Source = None
    source_energy: float = 0.0
    fresh_energy: list = field(default_factory=list)


class WaveSim:
    """Scalar MBS solver: WaveSimBase.m + WaveSim.m + Simulation.m restated.

    ``opt`` is the reference's option struct as a dict (``lambda``,
    ``pixel_size``, ``boundary_widths``, ``energy_threshold``, ``max_cycles``,
    ``single_precision``, ``roi``, ``epsilon``, ``ACC``/``wiggle``,
    ``boundary_type``, ``boundary_strength``, ``callback_interval``,
    ``energy_calculation_interval``)."""

    vector = False

    def __init__(self, refractive_index, opt):
        opt = dict(opt)
        if "wiggle" in opt:  # WaveSimBase.m:48-50
            opt["ACC"] = opt["wiggle"]
        # Simulation.m:90-94 property defaults, then option copy
        self.lambda_ = float(opt.get("lambda", 1.0))
        self.single_precision = bool(opt.get("single_precision", True))
        self.callback_interval = opt.get("callback_interval", 50)
        self.energy_threshold = float(opt.get("energy_threshold", 1e-2))
        self.energy_calculation_interval = opt.get("energy_calculation_interval", 8)
        self.max_cycles = opt.get("max_cycles", math.inf)
        self.ACC = opt.get("ACC", True)
        self.epsilonmin = 3
        self.callback = opt.get("callback", None)
        roi_opt = opt.get("roi", None)
        self.rdtype = np.float32 if self.single_precision else np.float64
        self.cdtype = np.complex64 if self.single_precision else np.complex128

        self.sample, self.grid = Medium.create(refractive_index, opt)  # Simulation.m:111
        self.N = np.concatenate([self.grid.N, [1]]).astype(np.int64)  # :114
        default_roi = np.stack([self.sample.Bl + 1, self.grid.N - self.sample.Br])  # :118
        if roi_opt is None:  # :119-124
            self.roi = np.stack([make4(default_roi[0]), make4(default_roi[1])])
        else:
            roi_opt = np.asarray(roi_opt)
            self.roi = np.stack([make4(roi_opt[0]), make4(roi_opt[1])])
            self.roi[:, :3] += default_roi[0] - 1
        self.energy_calculation_interval = min(self.energy_calculation_interval, self.callback_interval)  # :135

        # WaveSimBase.m:58-81
        k0 = 2 * np.pi / self.lambda_
        k0c = np.sqrt(self.sample.e_r_center) * k0
        if "epsilon" in opt:
            eps = float(opt["epsilon"])
        else:
            eps = self.calculate_epsilon(self.sample.e_r, k0, k0c)
        self.iterations_per_cycle = self.lambda_ / (2 * k0c / eps)  # :66
        V = self.sample.e_r * k0**2 - k0c**2 - 1.0j * eps  # :69
        V, self.filters = self.apply_edge_filters(V, opt)  # :70
        self.gamma = (1.0j / eps * V).astype(self.cdtype)  # :73
        self.k02e = self.cdtype(k0c**2 / eps + 1.0j)  # :77
        self.epsilon = self.rdtype(eps)  # :78
        self.k0, self.k0c = k0, k0c
        self.wiggles, self.ACC = self.compute_wiggles()  # :81
        if self.vector:
            if roi_opt is None:  # WaveSimVector.m:14-16
                self.roi[1, 3] = 3
            self.N[3] = 3  # WaveSimVector.m:17

    # --- WaveSimBase.m:201-215
    def calculate_epsilon(self, e_r, k0, k0c):
        V_tot = e_r * k0**2 - k0c**2
        vmax = np.max(np.abs(V_tot)) / 0.95
        return max(float(vmax), self.epsilonmin)

    # --- WaveSimBase.m:217-258
    def apply_edge_filters(self, V, opt):
        filters = [None, None, None]
        if self.sample.boundary_type != "ARL" or np.all(self.sample.Bl == 0):
            return V, filters
        bw = np.ravel(opt["boundary_widths"])
        for dim in range(3):
            bl = int(self.sample.Bl[dim])
            br = int(self.sample.Br[dim])
            roi_size = int(self.grid.N[dim]) - bl - br
            if bl > 0:
                L = int(bw[dim])
                if np.all(self.grid.N > 1):
                    def window(B):
                        return (np.arange(1, B + 1) - 0.21) / (B + 0.66)
                else:
                    def window(B, L=L):
                        return nuttallwin(2 * L - 1)[:B]
                if br == bl:
                    smooth = np.concatenate([[0.0], window(L - 1)])
                else:
                    smooth = window(L)
                filt = np.concatenate([np.zeros(bl - L), smooth, np.ones(roi_size), smooth[::-1], np.zeros(br - L)])
                shape = [1, 1, 1]
                shape[dim] = filt.size
                filters[dim] = filt.reshape(shape)
                V = V * filters[dim]
        return V, filters

    # --- WaveSimBase.m:272-298
    def compute_wiggles(self):
        ACC = np.ravel(np.asarray(self.ACC))
        if ACC.size == 1:
            ACC = ~self.grid.periodic if bool(ACC[0]) else np.zeros(3, dtype=bool)
        ACC = ACC.astype(bool)
        ws = wiggle_perm(ACC)
        return [self.wiggle_descriptor(ws[:, i]) for i in range(ws.shape[1])], ACC

    # --- WaveSimBase.m:300-316
    def wiggle_descriptor(self, wig):
        g = self.grid
        se = np.sqrt(self.epsilon)  # epsilon is already single/double here (:78)
        pxe = ((g.px_range - g.dpx * wig[1] / 4) / se).astype(self.rdtype)
        pye = ((g.py_range - g.dpy * wig[0] / 4) / se).astype(self.rdtype)
        pze = ((g.pz_range - g.dpz * wig[2] / 4) / se).astype(self.rdtype)
        gx = np.exp(1.0j * np.pi / 2 * wig[1] * g.x_range / g.dx / g.x_range.size).astype(self.cdtype)
        gy = np.exp(1.0j * np.pi / 2 * wig[0] * g.y_range / g.dx / g.y_range.size).astype(self.cdtype)
        gz = np.exp(1.0j * np.pi / 2 * wig[2] * g.z_range / g.dx / g.z_range.size).astype(self.cdtype)
        return Wiggle(np.asarray(wig), pxe, pye, pze, gx, gy, gz)

    # --- helpers
    def _fftn(self, E):
        return sfft.fftn(E, axes=(0, 1, 2), workers=-1)

    def _ifftn(self, E):
        return sfft.ifftn(E, axes=(0, 1, 2), workers=-1)

    def _ramp(self, w, conj=False):
        gx, gy, gz = w.gx, w.gy, w.gz
        if conj:
            gx, gy, gz = np.conj(gx), np.conj(gy), np.conj(gz)
        gx = gx.reshape(1, -1, 1)
        gy = gy.reshape(-1, 1, 1)
        gz = gz.reshape(1, 1, -1)
        if self.vector:
            gx, gy, gz = gx[..., None], gy[..., None], gz[..., None]
        return gx, gy, gz

    # --- WaveSim.m:15-59
    def propagate(self, E, w):
        px2 = (w.pxe**2).reshape(1, -1, 1)
        py2 = (w.pye**2).reshape(-1, 1, 1)
        pz2k = (w.pze**2).reshape(1, 1, -1) - self.k02e
        E = f_wiggle(E, *self._ramp(w))
        E = self._fftn(E)
        E = f_g0_scalar(E, px2, py2, pz2k)
        E = self._ifftn(E)
        return f_wiggle(E, *self._ramp(w, conj=True))

    def mix(self, dE, Eprop, gamma):
        """WaveSimBase.m:260-268."""
        if self.vector:
            gamma = gamma[..., None]
        return f_mix(dE, Eprop, gamma)

    def crop_field(self, E):
        """Simulation.m:254-261."""
        r = self.roi
        E4 = E if E.ndim == 4 else E[..., None]
        return E4[r[0, 0] - 1:r[1, 0], r[0, 1] - 1:r[1, 1], r[0, 2] - 1:r[1, 2], r[0, 3] - 1:r[1, 3]]

    @staticmethod
    def energy(E):
        """Simulation.m:265-273 - sum(abs(E(:)).^2)."""
        return float(np.sum(np.abs(E) ** 2, dtype=np.float64))

    def prepare_source(self, source):
        """Simulation.m:154-157 - cast, shift to the ROI origin, crop to the grid."""
        s = source.cast(self.cdtype).shift(self.roi[0]).crop(np.stack([np.ones(4, dtype=np.int64), self.N]))
        return s

    def field_shape(self):
        return tuple(int(v) for v in self.N[:3]) + ((3,) if self.vector else ())

    # --- Simulation.m:193-217
    def next(self, state, can_terminate):
        state.diff_energy.append(state.last_step_energy)
        d = state.diff_energy
        ratio = d[-1] / d[0] if d[0] != 0 else (math.nan if d[-1] == 0 else math.inf)
        if can_terminate and ratio < self.energy_threshold:
            state.has_next = False
            state.converged = True
        elif can_terminate and state.it >= state.max_iterations:
            state.has_next = False
            state.converged = False
        else:
            state.has_next = True
        state.calculate_energy = (state.it - 1) % self.energy_calculation_interval == 0
        if self.callback is not None and (state.it % self.callback_interval == 0 or not state.has_next):
            self.callback(self, state)
        state.it += 1
        return state

    # --- Simulation.m:138-190 (exec) + WaveSimBase.m:157-197 (MATLAB loop)
    def exec(self, source, max_iterations=None, fresh_energy=False):
        """Run the reference loop.  ``max_iterations`` overrides
        ``ceil(max_cycles * iterations_per_cycle)`` (the fixed-iteration
        protocol of examples/mie_sphere/mie_sphere_test.m:20-21).
        ``fresh_energy=True`` records the ROI energy of every iteration in
        ``state.fresh_energy`` as well (the stop rule is unchanged)."""
        state = State()
        state.source = self.prepare_source(source)
        state.source_energy = state.source.energy()
        if state.source_energy == 0:
            warnings.warn("There is no source inside the grid boundaries, expect to get zero field everywhere.")
            return None, state
        state.it = 1
        if max_iterations is not None:
            state.max_iterations = max_iterations
        else:
            state.max_iterations = math.ceil(self.max_cycles * self.iterations_per_cycle) \
                if math.isfinite(self.max_cycles) else math.inf
        shape = self.field_shape()
        state.E = np.zeros(shape, dtype=self.cdtype)
        state.dE = np.zeros(shape, dtype=self.cdtype)
        Nw = len(self.wiggles)
        A = self.cdtype(1.0j / self.epsilon / Nw)
        while state.has_next:
            wig = self.wiggles[(state.it - 1) % Nw]
            if state.it <= Nw:
                Etmp = state.source.add_to(state.dE, A)
            else:
                Etmp = state.dE
            Etmp = self.propagate(Etmp, wig)
            state.dE = self.mix(state.dE, Etmp, self.gamma).astype(self.cdtype)
            state.E = state.E + state.dE
            if state.calculate_energy or fresh_energy:
                e = self.energy(self.crop_field(state.dE))
                if fresh_energy:
                    state.fresh_energy.append(e)
                if state.calculate_energy:
                    state.last_step_energy = e
            can_terminate = state.it % Nw == 0
            state = self.next(state, can_terminate)
        state.E_prime = state.E  # full-grid E' (what RunWaveSimAlgorithmMex returns)
        with np.errstate(divide="ignore", invalid="ignore"):
            Eg = state.E / (self.gamma[..., None] if self.vector else self.gamma)
        E = self.crop_field(Eg)
        if not self.vector:
            E = E[..., 0]
        return E, state


class WaveSimVector(WaveSim):
    """WaveSimVector.m:1-53 - vector (Maxwell) MBS with the dyadic Green's function."""

    vector = True

    def propagate(self, E, w):
        E = f_wiggle(E, *self._ramp(w))
        fEx = self._fftn(E[..., 0])
        fEy = self._fftn(E[..., 1])
        fEz = self._fftn(E[..., 2])
        px = w.pxe.reshape(1, -1, 1)
        py = w.pye.reshape(-1, 1, 1)
        pz = w.pze.reshape(1, 1, -1)
        fEx, fEy, fEz = f_g0_vector(fEx, fEy, fEz, px, py, pz, self.k02e)
        E = np.stack([self._ifftn(fEx), self._ifftn(fEy), self._ifftn(fEz)], axis=-1)
        return f_wiggle(E, *self._ramp(w, conj=True))


def to_matlab_layout(a):
    """Column-major copy: the memory order of a MATLAB array (y fastest)."""
    return np.asfortranarray(a)
