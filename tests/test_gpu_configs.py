"""Full-size parity on the four benchmark configurations.

Each configuration (wavesim_b200/workloads.py: c1 2-D 512^2 homogeneous
point source, c2 2-D 1024^2 Gaussian random medium with a Gaussian beam, c3
3-D 256^3 with 2000 spheres and a plane wave, c4 3-D 192^3 x 3 vector sphere)
runs through WaveSim.exec to the reference tolerance and is compared with the
oracle's full-size runs (tests/golden/make_config_runs.py, the reference loop
WaveSimBase.m:157-197 with the stop rule of Simulation.m:193-217):

* the same iteration count to tolerance;
* the diff_energy history to 2e-4 relative;
* the ROI field at 4096 seeded points within 1e-4 relative L2 of the FP32
  oracle (the reference's default single precision) and of the FP64 oracle;
* the L2 norm of every z-plane (3-D) or x-column (2-D) within 1e-4;
* c1 also against the analytic 2-D Green's function more than 2 wavelengths
  from the source, within the FP64 oracle's own error there (+2%).

Setting WAVESIM_B200_PARITY_LOG to a file path appends one JSON line of
measured errors per configuration.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-4
HIST_RTOL = 2e-4


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def plane_norms(E):
    a = np.abs(np.asarray(E, dtype=np.complex128)) ** 2
    if a.ndim == 2:
        return np.sqrt(a.sum(axis=0))
    axes = tuple(i for i in range(a.ndim) if i != 2)
    return np.sqrt(a.sum(axis=axes))


def fixture(cfg):
    info = json.load(open(os.path.join(HERE, "golden", f"{cfg}_reference_run.json")))
    dig = np.load(os.path.join(HERE, "golden", f"{cfg}_digest.npz"))
    return info, dig


def log(entry):
    path = os.environ.get("WAVESIM_B200_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(entry) + "\n")


@pytest.mark.parametrize("cfg", ["c1", "c2", "c3", "c4"])
def test_config_matches_oracle(gpu, cfg):
    import wavesim_b200 as ws
    from wavesim_b200 import workloads
    info, dig = fixture(cfg)
    n, opt, val, pos, vector = workloads.CONFIGS[cfg]()
    sim = (ws.WaveSimVector if vector else ws.WaveSim)(n, opt)
    E, st = sim.exec(ws.Source(val, pos))
    sim.close()
    E = np.asarray(E)
    if not vector and E.ndim == 3 and E.shape[2] == 1:
        E = E[..., 0]
    assert list(E.shape) == info["roi_shape"]
    flat = E.reshape(-1, order="F")
    v = flat[dig["idx"]]
    e32 = rel(v, dig["v32"])
    e64 = rel(v, dig["v64"])
    ep = rel(plane_norms(E), dig["planes32"])
    hist_err = float(np.max(np.abs(st.diff_energy - np.asarray(info["diff_energy"]))
                            / np.abs(np.asarray(info["diff_energy"]))))
    entry = {"config": cfg, "iterations": st.it - 1, "oracle_iterations": info["iterations"],
             "rel_l2_vs_fp32_oracle": e32, "rel_l2_vs_fp64_oracle": e64, "plane_norms_rel_l2": ep,
             "history_max_rel": hist_err}
    if cfg == "c1":
        from oracle import analytic
        k = 2 * np.pi / float(opt["lambda"])
        h = float(opt["pixel_size"])
        yy, xx = np.meshgrid(np.arange(E.shape[0]) + 1, np.arange(E.shape[1]) + 1, indexing="ij")
        r_px = np.hypot(yy - pos[0], xx - pos[1])
        mask = r_px > info["analytic_min_r_px"]
        Ea = analytic.homogeneous_2d(k, h, r_px * h)
        entry["analytic_rel_l2"] = rel(E[mask], Ea[mask])
        entry["analytic_rel_l2_fp64_oracle"] = info["analytic_rel_l2_fp64"]
    log(entry)
    assert st.it - 1 == info["iterations"], entry
    assert st.converged == info["converged"]
    assert hist_err < HIST_RTOL, entry
    assert e32 < TOL, entry
    assert e64 < TOL, entry
    assert ep < TOL, entry
    if cfg == "c1":
        assert entry["analytic_rel_l2"] < 1.02 * info["analytic_rel_l2_fp64"], entry
