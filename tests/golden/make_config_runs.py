"""Full-size oracle runs of the four benchmark configurations (test fixtures).

For each configuration c1..c4 (wavesim_b200/workloads.py: the seeded media
and sources the configurations name) this runs the oracle - the
operation-by-operation restatement of the reference loop in oracle/ - to the
reference tolerance:

* in complex64 (the reference default, single_precision = true) with the
  reference stop rule (Simulation.m:193-217): iteration count, the
  diff_energy history and the ROI energy of every iteration;
* in complex128 for the same number of iterations: the FP64 oracle.

It writes <config>_reference_run.json (iterations, histories, set-up and loop
times) and <config>_digest.npz (a digest of the two ROI fields: the L2 norm of
every z-plane (3-D) or x-column (2-D), and the complex values at 4096 seeded
ROI points).  The GPU tests compare the CUDA loop with these digests; bench.py
reads the iteration count to tolerance.  For c1 (homogeneous n = 1, point
source) it also records the FP64 oracle's error against the analytic 2-D
Green's function more than 8 pixels (2 wavelengths) away from the source.

    python tests/golden/make_config_runs.py [c1 c2 c3 c4]

c3 takes about 3 + 6 minutes on 8 cores, c4 about 2 + 4, c1 and c2 seconds.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle import analytic  # noqa: E402
from oracle import mbs_oracle as ref  # noqa: E402

N_POINTS = 4096
ANALYTIC_MIN_R_PX = 8.0


def _load_workloads():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "ws_workloads", os.path.join(os.path.dirname(os.path.dirname(HERE)), "wavesim_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def plane_norms(E):
    """L2 norm per z-plane of a 3-D ROI field ([y, x, z] or [y, x, z, c]), per
    x-column of a 2-D one ([y, x])."""
    a = np.abs(np.asarray(E, dtype=np.complex128)) ** 2
    if a.ndim == 2:
        return np.sqrt(a.sum(axis=0))
    axes = tuple(i for i in range(a.ndim) if i != 2)
    return np.sqrt(a.sum(axis=axes))


def digest_points(shape, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(int(np.prod(shape)), size=N_POINTS, replace=False)).astype(np.int64)


def run(cfg, workloads):
    n, opt, val, pos, vector = workloads.CONFIGS[cfg]()
    cls = ref.WaveSimVector if vector else ref.WaveSim
    t0 = time.time()
    sim = cls(n, dict(opt, single_precision=True))
    t1 = time.time()
    E32, st = sim.exec(ref.Source(val, pos), fresh_energy=True)
    t2 = time.time()
    iters = st.it - 1
    print(f"{cfg}: fp32 {iters} iterations, converged {st.converged}, {t2 - t1:.1f} s", flush=True)
    sim64 = cls(n, dict(opt, single_precision=False, energy_threshold=0.0))
    t3 = time.time()
    E64, st64 = sim64.exec(ref.Source(val, pos), max_iterations=iters)
    t4 = time.time()
    assert st64.it - 1 == iters, (st64.it, iters)
    print(f"{cfg}: fp64 {st64.it - 1} iterations, {t4 - t3:.1f} s", flush=True)
    E32 = np.asarray(E32)
    E64 = np.asarray(E64)
    if not vector and E32.ndim == 3 and E32.shape[2] == 1:  # 2-D: [y, x]
        E32, E64 = E32[..., 0], E64[..., 0]
    idx = digest_points(E32.shape, 1000 + int(cfg[1]))
    flat32 = E32.reshape(-1, order="F")
    flat64 = E64.reshape(-1, order="F")
    rel = float(np.linalg.norm(flat32 - flat64) / np.linalg.norm(flat64))
    info = {
        "workload": cfg,
        "roi_shape": [int(v) for v in E32.shape],
        "grid": [int(v) for v in sim.N],
        "wiggles": len(sim.wiggles),
        "iterations": iters,
        "converged": bool(st.converged),
        "diff_energy": [float(v) for v in st.diff_energy],
        "fresh_energy": [float(v) for v in st.fresh_energy],
        "epsilon": float(sim.epsilon),
        "field_roi_l2_fp32": float(np.linalg.norm(flat32)),
        "field_roi_l2_fp64": float(np.linalg.norm(flat64)),
        "fp32_vs_fp64_rel_l2": rel,
        "setup_s": t1 - t0, "loop_s": t2 - t1, "loop_fp64_s": t4 - t3, "cores": os.cpu_count(),
    }
    extra = {}
    if cfg == "c1":
        # analytic 2-D Green's function of the point source, away from it
        k = 2 * np.pi / float(opt["lambda"])
        h = float(opt["pixel_size"])
        yy, xx = np.meshgrid(np.arange(E64.shape[0]) + 1, np.arange(E64.shape[1]) + 1, indexing="ij")
        r_px = np.hypot(yy - pos[0], xx - pos[1])
        mask = r_px > ANALYTIC_MIN_R_PX
        Ea = analytic.homogeneous_2d(k, h, r_px * h)
        err = float(np.linalg.norm(E64[mask] - Ea[mask]) / np.linalg.norm(Ea[mask]))
        info.update({"analytic_min_r_px": ANALYTIC_MIN_R_PX, "analytic_rel_l2_fp64": err})
        print(f"c1: FP64 oracle vs analytic 2-D: {err:.3e}")
    with open(os.path.join(HERE, f"{cfg}_reference_run.json"), "w") as f:
        json.dump(info, f, indent=1)
    np.savez_compressed(os.path.join(HERE, f"{cfg}_digest.npz"), idx=idx, v32=flat32[idx].astype(np.complex64),
                        v64=flat64[idx].astype(np.complex128), planes32=plane_norms(E32),
                        planes64=plane_norms(E64), **extra)
    print(f"{cfg}: fp32 vs fp64 rel L2 {rel:.3e}", flush=True)


def main():
    workloads = _load_workloads()
    cfgs = sys.argv[1:] or ["c1", "c2", "c3", "c4"]
    for cfg in cfgs:
        run(cfg, workloads)


if __name__ == "__main__":
    main()
