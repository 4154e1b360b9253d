"""Runs the oracle (FP32 restatement of the reference loop) on the full 3-D
256^3 disordered-medium workload (config c3) to tolerance 1e-3 and records the
iteration count and energy history in c3_reference_run.json.

This takes several minutes of CPU; it is the reference iteration count that
bench.py --impl reference projects its per-iteration time to, and the GPU
test compares its own count with it.

    python tests/golden/make_c3_reference_run.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle import mbs_oracle as ref  # noqa: E402
from wavesim_b200 import workloads  # noqa: E402


def main():
    n, opt, val, pos, vector = workloads.c3()
    t0 = time.time()
    sim = ref.WaveSim(n, opt)
    t1 = time.time()
    E, st = sim.exec(ref.Source(val, pos), fresh_energy=True)
    t2 = time.time()
    out = {
        "workload": "c3: 3-D 256^3 (ROI 224^3), 2000 spheres n=1.5 in 1.33, plane wave, energy_threshold 1e-3",
        "iterations": st.it - 1,
        "converged": bool(st.converged),
        "diff_energy": [float(v) for v in st.diff_energy],
        "fresh_energy": [float(v) for v in st.fresh_energy],
        "epsilon": float(sim.epsilon),
        "setup_s": t1 - t0,
        "loop_s": t2 - t1,
        "cores": os.cpu_count(),
        "field_roi_l2": float(np.linalg.norm(E)),
        "field_probe": [[float(E[i, j, k].real), float(E[i, j, k].imag)]
                        for (i, j, k) in [(112, 112, 10), (50, 170, 100), (200, 30, 200)]],
    }
    with open(os.path.join(HERE, "c3_reference_run.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out["iterations"], out["converged"], out["loop_s"])


if __name__ == "__main__":
    main()
