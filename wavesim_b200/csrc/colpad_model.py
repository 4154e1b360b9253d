#!/usr/bin/env python3
"""Host model of the shared-memory wavefronts of the mixed-radix column
passes' exchanges, used to choose ColPad<N> in ws_mixed.cuh.

A column pass holds 256 / P lines of N points per round, P = N / E threads
per line (thread t: line t / P, p = t % P) and element i of a line at
line * CS + i + (i >> SH) (8-byte elements).  Every stage but the first
reads the R inputs j + r N / R of its butterflies j = p + P q, and every
stage but the last writes output r of butterfly j to
(j - j mod Ns) R + j mod Ns + r Ns (the schedule of mixed::stage).  Each such
access is one warp instruction, served half a warp (16 threads, 8-byte
accesses) at a time; a half-warp takes as many wavefronts as the largest
number of distinct addresses that share one of the 16 eight-byte bank
slots.  The model sums these over a block of 256 threads and one transform.

Run:  python colpad_model.py            (prints the best (SH, CS) per plan)
"""
import itertools

# (N, E, radices) of the plans the column passes are instantiated for
PLANS = [(96, 12, (12, 4, 2)), (160, 20, (10, 4, 4)), (192, 12, (12, 4, 4)), (224, 28, (14, 4, 4)),
         (320, 20, (4, 4, 4, 5)), (448, 28, (14, 4, 4, 2)), (576, 36, (12, 12, 4))]
SHIFTS = (3, 4, 5, 6, 31)  # 31: no padding inside a line


def wavefronts(N, E, radices, CS, SH, threads=256):
    P = N // E
    stages, Ns = [], 1
    for s, R in enumerate(radices):
        stages.append((s, R, Ns, E // R, N // R))
        Ns *= R
    last = len(radices) - 1

    def slot(t, idx):
        return ((t // P) * CS + idx + (idx >> SH)) % 16, (t // P) * CS + idx + (idx >> SH)

    total = 0
    for half in range(threads // 16):
        lanes = range(16 * half, 16 * half + 16)
        for s, R, Ns, B, NR in stages:
            accesses = []
            if s > 0:  # reads of the stage's inputs
                accesses += [lambda t, q=q, r=r: (t % P + P * q) + r * NR for q in range(B) for r in range(R)]
            if s < last:  # writes of its outputs
                def w(t, q, r, R=R, Ns=Ns):
                    j = t % P + P * q
                    return (j - j % Ns) * R + j % Ns + r * Ns
                accesses += [lambda t, q=q, r=r, w=w: w(t, q, r) for q in range(B) for r in range(R)]
            for acc in accesses:
                banks = {}
                for t in lanes:
                    b, a = slot(t, acc(t))
                    banks.setdefault(b, set()).add(a)
                total += max(len(v) for v in banks.values())
    return total


def best(N, E, radices, span=16):
    out = []
    for SH in SHIFTS:
        base = (N - 1) + ((N - 1) >> SH) + 1
        for CS in range(base, base + span):
            out.append((wavefronts(N, E, radices, CS, SH), SH, CS))
    return sorted(out)


def main():
    for N, E, radices in PLANS:
        planes = wavefronts(N, E, radices, N + N // 16 + 1, 4)
        w, SH, CS = best(N, E, radices)[0]
        print(f"N = {N:4d}: planes' layout (SH 4, CS {N + N // 16 + 1}) {planes:5d} wavefronts; "
              f"best SH {SH}, CS {CS}: {w}")


if __name__ == "__main__":
    main()
