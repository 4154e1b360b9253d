"""The PSTD restatement (oracle/pstd_oracle.py) against the MBS restatement.

The reference ships no PSTD output, so the time-domain restatement is pinned
by physics: on an absorbing, periodic medium both solvers reach the steady
state of the same Helmholtz equation, (lap + k0^2 e_r) E = -S, and PSTD's
leapfrog is second order in the time step, so its distance to the MBS field
falls as dt^2.
"""
import numpy as np
import pytest

from oracle import mbs_oracle as ref
from oracle.pstd_oracle import PSTD


def _problem():
    L = 48
    rng = np.random.default_rng(1)
    n = 1.0 + 0.1 * rng.random((L, L)) + 0.05j
    return n, ref.Source(np.ones((1, 1)), [L // 2, L // 2, 1, 1])


def test_pstd_converges_to_mbs_as_dt_squared():
    n, src = _problem()
    m = ref.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "energy_threshold": 1e-10,
                        "single_precision": False})
    Em, _ = m.exec(src)
    Em = Em[..., 0]
    err = {}
    for dtr in (0.3, 0.1):
        p = PSTD(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "boundary_type": "ARL",
                     "energy_threshold": 1e-7, "dt_relative": dtr, "single_precision": False})
        Ep, sp = p.exec(src)
        assert sp.converged
        err[dtr] = np.linalg.norm(Ep[..., 0] - Em) / np.linalg.norm(Em)
    assert err[0.1] < 6e-3, err
    assert 6.0 < err[0.3] / err[0.1] < 12.0, err  # second order: (0.3 / 0.1)^2 = 9


def test_pstd_option_checks():
    n, _ = _problem()
    with pytest.raises(ValueError):
        PSTD(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0]})
    with pytest.raises(ValueError):
        PSTD(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "boundary_type": "ARL",
                 "boundary_strength": 0.2})


def test_pstd_time_step_and_coefficients():
    n, _ = _problem()
    p = PSTD(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "boundary_type": "ARL"})
    e_r_min = float(np.min(np.real(n ** 2)))
    assert np.isclose(p.dtmax, 2 / np.sqrt(2) / np.pi * 0.25 * np.sqrt(e_r_min))
    assert np.isclose(p.dt, 0.95 * p.dtmax)
    assert np.isclose(p.iterations_per_cycle, 1.0 / p.dt)
    # lossless points: c1 = -1, c2 = 2 (plain leapfrog); lossy points damp
    q = PSTD(np.ones((8, 8)), {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [0, 0], "boundary_type": "ARL"})
    assert np.allclose(q.c1, -1) and np.allclose(q.c2, 2)
    assert np.all(p.c1 > -1) and np.all(p.c2 < 2)
