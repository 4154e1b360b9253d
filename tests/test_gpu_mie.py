"""Physics check of the vector solver (WaveSimVector) against the Mie
solution (oracle/mie.py, a restatement of Bohren & Huffman ch. 4) for a
dielectric sphere in an x-polarised plane wave - the check
examples/mie_sphere/mie_sphere_test.m makes with the third-party MatScat.

The scattered field is the field with the sphere minus the field of the
same source without it (so the finite source aperture cancels); the Mie
incident amplitude is fitted to the latter around the sphere.  The sphere
is a staircase of 8-pixel radius at lambda/8 pixels, so agreement is at the
level of the discretisation, a few percent, not of the loop's tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_vector_solver_matches_mie(gpu):
    import wavesim_b200 as ws
    from oracle import mie
    lam, h, a, n_s, n_b, roi = 1.0, 0.125, 1.0, 1.5, 1.33, 64
    c = roi / 2
    idx = (np.arange(roi) + 0.5 - c) * h
    Y, X, Z = np.meshgrid(idx, idx, idx, indexing="ij")  # grid axes (y, x, z)
    inside = X ** 2 + Y ** 2 + Z ** 2 < a ** 2
    opt = {"lambda": lam, "pixel_size": h, "boundary_widths": [16, 16, 16], "energy_threshold": 1e-6}
    src = ws.Source(np.ones((roi, roi)), [1, 1, 1, 1])
    E_tot, st = ws.WaveSimVector(np.where(inside, n_s, n_b), opt).exec(src)
    E_inc, _ = ws.WaveSimVector(np.full((roi, roi, roi), n_b), opt).exec(src)
    assert st.converged
    k = 2 * np.pi * n_b / lam
    near = X ** 2 + Y ** 2 + Z ** 2 < (2 * a) ** 2
    # incident amplitude E0 of E0 exp(i k z) x^, fitted around the sphere
    ph = np.exp(1j * k * Z[near])
    E0 = np.vdot(ph, E_inc[..., 0][near]) / np.vdot(ph, ph)
    assert np.abs(E_inc[..., 1:][near]).max() < 1e-3 * abs(E0)  # x-polarised
    pts = np.stack([X[near], Y[near], Z[near]], axis=-1)
    E_m = mie.field(pts, a, n_s, n_b, lam, E0=E0)
    inc = np.zeros_like(E_m)
    inc[:, 0] = E0 * ph
    scat_m = E_m - inc
    scat_n = E_tot[near] - E_inc[near]
    err = np.linalg.norm(scat_n - scat_m) / np.linalg.norm(scat_m)
    err_total = np.linalg.norm(E_tot[near] - E_m) / np.linalg.norm(E_m)
    print(f"Mie: scattered-field error {err:.3f}, total-field error {err_total:.4f}")
    assert err < 0.1, err
    assert err_total < 0.03, err_total
