"""The register-resident mixed-radix schedule (wavesim_b200/csrc/ws_mixed.cuh,
mixed::stage / mixed::line_fft), replayed on the host for every plan the
library instantiates (the `mixed::Plan<...>` aliases of ws_mbs.cu): P = N/E
threads with E elements each, up to four radices each dividing E, stage 0
from registers (butterfly q of thread p takes v[q + (E/R0) r]), later stages
through the shared line with twiddles W_{Ns R}^{(j mod Ns) r}, the last
stage's outputs reordered so that thread p holds X[p + P m].  The replay must
equal numpy's FFT (MATLAB's fft / ifft * N, which fftn/ifftn in
WaveSimBase.m:118-124 rest on), forward and inverse."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MBS = os.path.join(ROOT, "wavesim_b200", "csrc", "ws_mbs.cu")


def plans():
    """(name, N, E, radices) of every `using X = mixed::Plan<N, E, R0, ...>;`."""
    out = []
    with open(MBS) as f:
        for m in re.finditer(r"using\s+(\w+)\s*=\s*mixed::Plan<([0-9,\s]+)>;", f.read()):
            a = [int(v) for v in m.group(2).split(",")]
            out.append((m.group(1), a[0], a[1], [r for r in a[2:] if r > 1]))
    return out


def replay(x, E, radices, inverse):
    """Thread-by-thread replay of mixed::line_fft: returns X with thread p's
    output v[m] stored at X[p + P m]."""
    N = len(x)
    P = N // E
    sign = 1 if inverse else -1
    tw = np.exp(-2j * np.pi * np.arange(N) / N)
    v = [[x[p + P * r] for r in range(E)] for p in range(P)]
    line = np.zeros(N, complex)
    nst = len(radices)
    for s, R in enumerate(radices):
        Ns = int(np.prod(radices[:s])) if s else 1
        B, NR, TS = E // R, N // R, N // (Ns * R)
        dft = np.exp(sign * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
        new = []
        for p in range(P):
            vv = list(v[p])
            if s == 0 and B > 1:
                vv = [v[p][q + B * r] for q in range(B) for r in range(R)]
            if s > 0:
                for q in range(B):
                    j = p + P * q
                    for r in range(R):
                        vv[q * R + r] = line[j + r * NR]
                    jm = j % Ns
                    for r in range(1, R):
                        w = tw[jm * r * TS]
                        vv[q * R + r] *= np.conj(w) if inverse else w
            for q in range(B):
                vv[q * R:(q + 1) * R] = list(dft @ np.array(vv[q * R:(q + 1) * R]))
            new.append(vv)
        if s < nst - 1:
            # every thread has read the line before any writes it (the stage's barrier)
            written = np.zeros(N, bool)
            for p in range(P):
                for q in range(B):
                    j = p + P * q
                    jm = j % Ns
                    base = (j - jm) * R + jm
                    for r in range(R):
                        idx = base + r * Ns
                        assert 0 <= idx < N and not written[idx]
                        written[idx] = True
                        line[idx] = new[p][q * R + r]
            assert written.all()
            v = new
        else:
            v = [[vv[q * R + r] for m in range(E) for q, r in [(m % B, m // B)]] for vv in new]
    X = np.zeros(N, complex)
    for p in range(P):
        for m in range(E):
            X[p + P * m] = v[p][m]
    return X


PLANS = plans()


def test_plans_found():
    names = {p[0] for p in PLANS}
    assert {"Plan192", "Plan96", "Plan160", "Plan224", "Plan320", "Plan448", "Plan576"} <= names


@pytest.mark.parametrize("name,N,E,radices", PLANS, ids=[p[0] for p in PLANS])
def test_plan_schedule_matches_fft(name, N, E, radices):
    P = N // E
    assert int(np.prod(radices)) == N and N % E == 0
    assert all(E % r == 0 for r in radices), "every radix divides E"
    assert 256 % P == 0 and (P > 32 or 32 % P == 0), "lines of P threads fit the 256-thread blocks"
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    np.testing.assert_allclose(replay(x, E, radices, False), np.fft.fft(x), rtol=0, atol=1e-9 * N)
    np.testing.assert_allclose(replay(x, E, radices, True), np.fft.ifft(x) * N, rtol=0, atol=1e-9 * N)


def test_column_padding_is_the_models_choice():
    """ColPad<N> (ws_mixed.cuh) gives the column passes' exchanges at most 6%
    more shared-memory wavefronts than the best (shift, stride) of the host
    model in wavesim_b200/csrc/colpad_model.py, for every plan it covers."""
    import sys
    csrc = os.path.join(ROOT, "wavesim_b200", "csrc")
    sys.path.insert(0, csrc)
    try:
        import colpad_model as cm
    finally:
        sys.path.pop(0)
    with open(os.path.join(csrc, "ws_mixed.cuh")) as f:
        src = f.read()
    table = {int(m.group(1)): (int(m.group(2)), int(m.group(3))) for m in re.finditer(
        r"struct ColPad<(\d+)> \{ static constexpr int SH = (\d+), CS = (\d+); \};", src)}
    assert table, "ColPad specialisations found"
    for N, E, radices in cm.PLANS:
        SH, CS = table.get(N, (4, N + N // 16 + 1))
        assert CS >= (N - 1) + ((N - 1) >> SH) + 1
        got = cm.wavefronts(N, E, radices, CS, SH)
        best = cm.best(N, E, radices)[0][0]
        assert got <= 1.06 * best, (N, got, best)
