"""Known-answer solutions used to pin the oracle (test infrastructure only).

``homogeneous_1d`` restates utilities/homogeneous_medium_analytic_solution.m:1-37
of the reference: the field of a band-limited (sinc) point source of unit
pixel amplitude on a 1-D grid of spacing ``h`` in a homogeneous medium with
wavenumber ``k``.  MATLAB's ``expint`` (the exponential integral E1 of a
complex argument) is ``scipy.special.exp1``.

``homogeneous_2d`` / ``homogeneous_3d`` are the continuum limits of the same
convention, (nabla^2 + k^2) E = -S with S the pixel amplitudes as a density:
E = h^2 (i/4) H0^(1)(k r) and E = h^3 exp(i k r) / (4 pi r).  They are only
valid a few wavelengths away from the source.
"""
import numpy as np
import scipy.special as sp


def homogeneous_1d(k, h, x):
    """utilities/homogeneous_medium_analytic_solution.m:26-35."""
    x = np.abs(np.asarray(x, dtype=float))
    phi = k * x
    with np.errstate(all="ignore"):
        sol = (1.0j * h / (2 * k) * np.exp(1.0j * phi)
               - h / (4 * np.pi * k) * (
                   np.exp(1.0j * phi) * (sp.exp1(1.0j * (k - np.pi / h) * x) - sp.exp1(1.0j * (k + np.pi / h) * x))
                   - np.exp(-1.0j * phi) * (-sp.exp1(-1.0j * (k - np.pi / h) * x) + sp.exp1(-1.0j * (k + np.pi / h) * x))))
    small = np.abs(k * x) < 1e-10  # :34-35
    sol = np.where(small, 1.0j * h / (2 * k) * (1 + 2.0j * np.arctanh(h * k / np.pi) / np.pi), sol)
    return sol


def homogeneous_2d(k, h, r):
    r = np.asarray(r, dtype=float)
    return h**2 * 0.25j * sp.hankel1(0, k * r)


def homogeneous_3d(k, h, r):
    r = np.asarray(r, dtype=float)
    return h**3 * np.exp(1.0j * k * r) / (4 * np.pi * r)
