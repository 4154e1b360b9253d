"""Mie solution for a sphere in a plane wave (test infrastructure).

Only tests import this.  It restates the published Lorenz-Mie solution as
given by Bohren & Huffman, "Absorption and Scattering of Light by Small
Particles" (Wiley, 1983), chapter 4: the expansion coefficients a_n, b_n
(eq. 4.53) and c_n, d_n (eq. 4.52, mu = mu_1), the vector spherical
harmonics M_o1n, N_e1n (eq. 4.50) with the angular functions pi_n, tau_n
(eq. 4.46-4.47 recurrences), and the fields of an x-polarised plane wave
E0 exp(i k z) along +z (eq. 4.37, 4.40, 4.45): inside
E1 = sum E_n (c_n M_o1n^(1) - i d_n N_e1n^(1)), outside
Es = sum E_n (i a_n N_e1n^(3) - b_n M_o1n^(3)), E_n = i^n E0 (2n+1)/(n(n+1)).
Time dependence exp(-i omega t), outgoing h_n^(1), the same sign convention
as the MBS Green's function (outgoing exp(+i k r)).

The reference's own Mie check (examples/mie_sphere/mie_sphere_test.m) uses
the third-party MatScat package, which the reference does not ship; this
restatement stands in for it.
"""
from __future__ import annotations

import numpy as np
from scipy.special import spherical_jn, spherical_yn


def _bessel(n, rho, kind):
    """z_n(rho) and d/drho z_n for kind 1 (j_n) or 3 (h_n^(1))."""
    j = spherical_jn(n, rho)
    jd = spherical_jn(n, rho, derivative=True)
    if kind == 1:
        return j, jd
    y = spherical_yn(n, rho)
    yd = spherical_yn(n, rho, derivative=True)
    return j + 1j * y, jd + 1j * yd


def coefficients(x, m, nmax):
    """a_n, b_n, c_n, d_n for n = 1..nmax (size parameter x = k a in the host
    medium, relative index m)."""
    n = np.arange(1, nmax + 1)
    mx = m * x
    jx, jdx = _bessel(n, x, 1)
    hx, hdx = _bessel(n, x, 3)
    jm, jdm = _bessel(n, mx, 1)
    psi_x, dpsi_x = x * jx, jx + x * jdx          # psi_n(x), psi_n'(x)
    xi_x, dxi_x = x * hx, hx + x * hdx            # xi_n(x), xi_n'(x)
    psi_m, dpsi_m = mx * jm, jm + mx * jdm        # psi_n(mx), psi_n'(mx)
    a = (m * psi_m * dpsi_x - psi_x * dpsi_m) / (m * psi_m * dxi_x - xi_x * dpsi_m)
    b = (psi_m * dpsi_x - m * psi_x * dpsi_m) / (psi_m * dxi_x - m * xi_x * dpsi_m)
    num = jx * dxi_x - hx * dpsi_x
    c = num / (jm * dxi_x - hx * dpsi_m)
    d = m * num / (m * m * jm * dxi_x - hx * dpsi_m)
    return a, b, c, d


def _angular(nmax, mu):
    """pi_n(mu), tau_n(mu) for n = 1..nmax, arrays of shape (nmax, len(mu))."""
    pi = np.zeros((nmax + 1,) + mu.shape)
    tau = np.zeros_like(pi)
    pi[1] = 1.0
    tau[1] = mu
    for n in range(2, nmax + 1):
        pi[n] = (2 * n - 1) / (n - 1) * mu * pi[n - 1] - n / (n - 1) * pi[n - 2]
        tau[n] = n * mu * pi[n] - (n + 1) * pi[n - 1]
    return pi[1:], tau[1:]


def field(points, radius, n_sphere, n_host, wavelength, E0=1.0, nmax=None):
    """Total electric field (x, y, z components, complex) at points (..., 3)
    relative to the sphere centre, for the incident field E0 exp(i k z) x^
    in the host medium (k = 2 pi n_host / wavelength)."""
    pts = np.asarray(points, dtype=float)
    shp = pts.shape[:-1]
    p = pts.reshape(-1, 3)
    k = 2 * np.pi * n_host / wavelength
    m = n_sphere / n_host
    x = k * radius
    if nmax is None:
        nmax = int(np.round(x + 4 * x ** (1 / 3) + 2))
    a, b, c, d = coefficients(x, m, nmax)
    r = np.linalg.norm(p, axis=1)
    cos_t = np.where(r > 0, p[:, 2] / np.where(r > 0, r, 1), 1.0)
    sin_t = np.sqrt(np.clip(1 - cos_t ** 2, 0, None))
    phi = np.arctan2(p[:, 1], p[:, 0])
    cphi, sphi = np.cos(phi), np.sin(phi)
    pi, tau = _angular(nmax, cos_t)
    n = np.arange(1, nmax + 1)[:, None]
    En = (1j ** n) * E0 * (2 * n + 1) / (n * (n + 1))
    inside = r < radius
    Er = np.zeros(r.shape, complex)
    Et = np.zeros(r.shape, complex)
    Ep = np.zeros(r.shape, complex)
    for region, kind, kk, cm, cn in ((inside, 1, m * k, c, d), (~inside, 3, k, b, a)):
        if not region.any():
            continue
        rho = kk * r[region]
        z, zd = _bessel(n, rho[None, :], kind)
        dz = (z + rho * zd) / rho                          # (rho z_n)' / rho
        zr = z / rho
        pi_r, tau_r = pi[:, region], tau[:, region]
        cp, sp, st = cphi[region], sphi[region], sin_t[region]
        # M_o1n and N_e1n in (r, theta, phi) components
        M_t, M_p = cp * pi_r * z, -sp * tau_r * z
        N_r = cp * n * (n + 1) * st * pi_r * zr
        N_t, N_p = cp * tau_r * dz, -sp * pi_r * dz
        if kind == 1:   # inside: c_n M - i d_n N
            fm, fn = cm[:, None], -1j * cn[:, None]
        else:           # scattered: -b_n M + i a_n N
            fm, fn = -cm[:, None], 1j * cn[:, None]
        Er[region] = np.sum(En * fn * N_r, axis=0)
        Et[region] = np.sum(En * (fm * M_t + fn * N_t), axis=0)
        Ep[region] = np.sum(En * (fm * M_p + fn * N_p), axis=0)
    ct = cos_t
    Ex = Er * sin_t * cphi + Et * ct * cphi - Ep * sphi
    Ey = Er * sin_t * sphi + Et * ct * sphi + Ep * cphi
    Ez = Er * ct - Et * sin_t
    out = np.stack([Ex, Ey, Ez], axis=-1)
    inc = E0 * np.exp(1j * k * p[:, 2])
    out[~inside, 0] += inc[~inside]  # outside: incident + scattered
    return out.reshape(shp + (3,))
