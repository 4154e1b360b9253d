"""Seeded synthetic media and sources for the five benchmark configurations.

No dataset ships with the reference; these generators stand in for it with
the shapes, sizes and value distributions the configurations name (NumPy
PCG64, fixed seeds).  Each returns ``(n, options, source_value, position,
vector)`` in the reference's conventions (positions 1-based in ROI
coordinates, Source.m:24).

* c1: 2-D homogeneous n = 1, 512^2 grid incl. 32-px boundary (ROI 448^2),
      point source at the centre, 4 wiggles.
* c2: 2-D Gaussian random medium, 1024^2 incl. 32-px boundary (ROI 960^2),
      n = clip(1 + 0.3 g, 0.8, 1.6) + 0.01i with g a unit-variance Gaussian
      field of correlation length 1 lambda; Gaussian beam (waist 4 lambda) on
      the left edge.
* c3: 3-D 256^3 incl. 16-px boundary (ROI 224^3): background 1.33 with 2000
      non-overlapping spheres of radius U[0.5, 2] lambda and n = 1.5 placed by
      random sequential addition; plane wave on the z = 1 face.
* c4: 3-D vector, 192^3 x 3 incl. 16-px boundary (ROI 160^3), lambda 0.5,
      pixel lambda/8, one sphere of radius 1.0 and n = 1.5 in 1.33,
      x-polarised plane wave along z.
* c5 helpers: plane waves at angles in +-30 degrees on one medium.
"""
from __future__ import annotations

import numpy as np

PPW = 4  # pixels per wavelength (pixel = lambda / 4)


def gaussian_random_field(shape, corr_px, rng):
    """White noise filtered by a Gaussian of correlation length corr_px
    pixels, normalised to zero mean and unit standard deviation."""
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kk = sum(np.meshgrid(*[ki ** 2 for ki in k], indexing="ij"))
    filt = np.exp(-2 * (np.pi * corr_px) ** 2 * kk)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    g -= g.mean()
    return g / g.std()


def sphere_packing(roi_px, n_spheres, r_min_px, r_max_px, rng, max_tries=2_000_000):
    """Random sequential addition of non-overlapping spheres fully inside a
    cube of roi_px voxels.  Returns (centres, radii) in voxel units."""
    cell = 2 * r_max_px
    ncell = max(1, int(np.ceil(roi_px / cell)))
    buckets = {}
    centres, radii = [], []
    tries = 0
    while len(radii) < n_spheres and tries < max_tries:
        tries += 1
        r = rng.uniform(r_min_px, r_max_px)
        c = rng.uniform(r, roi_px - r, size=3)
        ci = tuple(np.minimum((c // cell).astype(int), ncell - 1))
        ok = True
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    for j in buckets.get((ci[0] + dz, ci[1] + dy, ci[2] + dx), ()):
                        if np.sum((centres[j] - c) ** 2) < (radii[j] + r) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            buckets.setdefault(ci, []).append(len(radii))
            centres.append(c)
            radii.append(r)
    return np.array(centres), np.array(radii)


def rasterise_spheres(shape, centres, radii, n_bg, n_sphere):
    n = np.full(shape, n_bg, dtype=np.float64)
    idx = [np.arange(s) + 0.5 for s in shape]  # voxel centres
    for c, r in zip(centres, radii):
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, shape)
        a = idx[0][lo[0]:hi[0], None, None] - c[0]
        b = idx[1][None, lo[1]:hi[1], None] - c[1]
        d = idx[2][None, None, lo[2]:hi[2]] - c[2]
        inside = a ** 2 + b ** 2 + d ** 2 < r ** 2
        sub = n[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        sub[inside] = n_sphere
    return n


def c1(scale=1):
    roi = 448 // scale
    bw = 32 // scale
    opt = {"lambda": 1.0, "pixel_size": 1.0 / PPW, "boundary_widths": [bw, bw], "energy_threshold": 1e-3}
    return np.ones((roi, roi)), opt, 1.0, [roi // 2 + 1, roi // 2 + 1], False


def c2(scale=1, seed=2):
    rng = np.random.default_rng(seed)
    roi = 960 // scale
    bw = 32 // scale
    g = gaussian_random_field((roi, roi), PPW, rng)
    n = np.clip(1.0 + 0.3 * g, 0.8, 1.6) + 0.01j
    y = np.arange(roi)
    beam = np.exp(-((y - roi / 2) ** 2) / (4 * PPW) ** 2).astype(complex)[:, None]
    opt = {"lambda": 1.0, "pixel_size": 1.0 / PPW, "boundary_widths": [bw, bw], "energy_threshold": 1e-3}
    return n, opt, beam, [1, 1], False


def c3(scale=1, seed=3, n_spheres=2000):
    rng = np.random.default_rng(seed)
    roi = 224 // scale
    bw = 16 // scale
    ns = max(1, n_spheres // scale ** 3)
    cen, rad = sphere_packing(roi, ns, 0.5 * PPW, 2.0 * PPW, rng)
    n = rasterise_spheres((roi, roi, roi), cen, rad, 1.33, 1.5)
    opt = {"lambda": 1.0, "pixel_size": 1.0 / PPW, "boundary_widths": [bw, bw, bw], "energy_threshold": 1e-3}
    return n, opt, np.ones((roi, roi)), [1, 1, 1], False


def c4(scale=1):
    roi = 160 // scale
    bw = 16 // scale
    lam = 0.5
    dx = lam / 8
    r_px = 1.0 / dx / scale
    c = roi / 2
    idx = np.arange(roi) + 0.5 - c
    inside = idx[:, None, None] ** 2 + idx[None, :, None] ** 2 + idx[None, None, :] ** 2 < r_px ** 2
    n = np.where(inside, 1.5, 1.33)
    opt = {"lambda": lam, "pixel_size": dx, "boundary_widths": [bw, bw, bw], "energy_threshold": 1e-3}
    return n, opt, np.ones((roi, roi)), [1, 1, 1, 1], True


def sphere_medium(roi, rng, n_bg=1.33, n_sphere=1.5, spheres_per_224=2000):
    """A roi^3 cube of the c3 sphere distribution (radius U[0.5, 2] lambda at
    4 pixels per wavelength, n_sphere in n_bg) with as many spheres per
    volume as 2000 in a 224^3 cube: the media of the warm-start training set
    and of small test problems."""
    count = max(1, int(round(spheres_per_224 * (roi / 224.0) ** 3)))
    cen, rad = sphere_packing(roi, count, 0.5 * PPW, 2.0 * PPW, rng)
    return rasterise_spheres((roi, roi, roi), cen, rad, n_bg, n_sphere)


def plane_wave_edge(roi_len, angle, pixel_size, lam, n_bg=1.0):
    """exp(i k sin(theta) y) along the entry edge (a column at x = 1)."""
    k = 2 * np.pi / lam * n_bg
    y = np.arange(roi_len) * pixel_size
    return np.exp(1j * k * np.sin(angle) * y)[:, None]


CONFIGS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4}
