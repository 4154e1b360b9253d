"""Many solves at once: media of different sizes, or many sources per medium.

No counterpart in the reference, whose ``exec`` runs one solve at a time
(e.g. the angle sweep of examples/pulse2d.m:31-40 calls it in a loop).

* Sources that share a medium go through ``WaveSim.exec_batch``: one batched
  solve, every kernel launch covering all of them.
* Media of different grid sizes cannot share a launch (each size has its own
  FFT plan and kernel shapes).  ``solve_many`` runs them concurrently
  instead: each ``WaveSim`` owns a solver with its own CUDA stream, and
  ``workers`` host threads drive them (the C calls release the interpreter
  lock), so small solves that would leave most SMs idle overlap on the GPU.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor


def solve_many(problems, workers=4, warm_starts=None):
    """problems: list of (sim, source) pairs (sim a WaveSim or WaveSimVector,
    each pair its own medium).  Returns (fields, states, seconds) with the
    results in the order of `problems`; warm_starts (optional) one start per
    problem or None, as WaveSim.exec takes them."""
    starts = warm_starts if warm_starts is not None else [None] * len(problems)
    if len(starts) != len(problems):
        raise ValueError("one warm start per problem")

    def run(i):
        sim, src = problems[i]
        return sim.exec(src, warm_start=starts[i])

    t0 = time.perf_counter()
    if workers <= 1:
        out = [run(i) for i in range(len(problems))]
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            out = list(ex.map(run, range(len(problems))))
    dt = time.perf_counter() - t0
    return [o[0] for o in out], [o[1] for o in out], dt
