"""The Mie restatement (oracle/mie.py) is self-consistent: the tangential
electric field is continuous across the sphere surface, the scattered field
vanishes for an index-matched sphere, and the extinction efficiency agrees
with the optical theorem's small-particle (Rayleigh) limit."""
import numpy as np

from oracle import mie


def _tangential(E, pts):
    rh = pts / np.linalg.norm(pts, axis=-1, keepdims=True)
    return E - np.sum(E * rh, axis=-1, keepdims=True) * rh


def test_tangential_field_is_continuous_at_the_surface():
    rng = np.random.default_rng(0)
    v = rng.standard_normal((200, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    a = 1.0
    Ein = mie.field(v * a * (1 - 1e-7), a, 1.5, 1.33, 0.5)
    Eout = mie.field(v * a * (1 + 1e-7), a, 1.5, 1.33, 0.5)
    ti, to = _tangential(Ein, v), _tangential(Eout, v)
    assert np.abs(ti - to).max() < 1e-5 * np.abs(to).max()
    # normal D = n^2 E continuous too
    ni = np.sum(Ein * v, axis=-1) * 1.5 ** 2
    no = np.sum(Eout * v, axis=-1) * 1.33 ** 2
    assert np.abs(ni - no).max() < 1e-5 * np.abs(no).max()


def test_matched_sphere_does_not_scatter():
    pts = np.array([[0.3, 0.2, 2.0], [1.5, -0.4, 0.1], [0.0, 0.1, -1.2]])
    E = mie.field(pts, 1.0, 1.33, 1.33, 0.5)
    k = 2 * np.pi * 1.33 / 0.5
    want = np.zeros_like(E)
    want[:, 0] = np.exp(1j * k * pts[:, 2])
    assert np.abs(E - want).max() < 1e-9


def test_small_sphere_extinction_matches_rayleigh():
    x, m = 0.05, 1.5
    a, b, c, d = mie.coefficients(x, m, 5)
    qext = 2 / x ** 2 * np.sum((2 * np.arange(1, 6) + 1) * np.real(a + b))
    ray = 8 / 3 * x ** 4 * ((m ** 2 - 1) / (m ** 2 + 2)) ** 2  # non-absorbing: Q_ext = Q_sca
    assert abs(qext - ray) < 0.02 * ray
