"""Train the learned warm start on MBS solutions and write its checkpoint.

    python -m wavesim_b200.train_warmstart [--samples 2000] [--sizes 64,96,128] [--steps 4000] [--out PATH]

The defaults are the command that produced the committed checkpoint
(wavesim_b200/data/warmstart_spheres.npz); the checkpoint stores that command,
the training loss and the evaluation below as its provenance
(WarmStart.provenance(path)).

The training set is made by this package's own solver: seeded cubes of the
c3 sphere distribution (radius U[0.5, 2] lambda, n = 1.5 in 1.33, 2000
spheres per 224^3) of sides 64, 96 and 128 (crops of the benchmark's 224^3
medium's distribution, one side drawn per sample), with the c3 plane-wave
source, solved to an energy ratio of 1e-4.  Training runs on the GPU with the
network's own forward and backward kernels (wavesim_b200.warmstart; the
half-resolution network, ROI sides multiples of 16).  The checkpoint stores
bf16 weights (``WarmStart.save(..., bf16=True)``); ``WarmStart.load`` reads it
back.  At the end the script reports, on held-out media of each training size
(seeds apart from the training set's), the prediction error and the
iterations of cold and warm-started solves at energy threshold 1e-3, with
both solves' errors against a converged solve (energy threshold 1e-9).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_spheres.npz")
EVAL_SEED = 12345


def evaluate(model, sides, per_size, boundary=8, seed=EVAL_SEED, tol=1e-3):
    """Cold and warm-started solves of held-out media (seeded apart from the
    training set): per medium the prediction error, the iterations of both
    solves (the warm count includes its cold probe and residual probe
    iterations) and their errors against a converged solve."""
    import wavesim_b200 as ws
    from wavesim_b200.workloads import sphere_medium
    rng = np.random.default_rng(seed)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    out = []
    for roi in sides:
        for _ in range(per_size):
            n = sphere_medium(roi, rng)
            opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [boundary] * 3}
            src = ws.Source(np.ones((roi, roi)), [1, 1, 1])
            ref_sim = ws.WaveSim(n, dict(opt, energy_threshold=1e-9))
            Einf, _ = ref_sim.exec(src)
            ref_sim.close()
            sim = ws.WaveSim(n, dict(opt, energy_threshold=tol))
            E, st = sim.exec(src)
            Ew, sw = sim.exec(src, warm_start=model)
            sim.close()
            out.append({"roi": roi, "pred_err": rel(model.predict(n), Einf), "cold_it": st.it - 1,
                        "warm_it": sw.it - 1 + 2, "discarded": bool(sw.warm_discarded),
                        "residual_ratio": sw.warm_residual_energy / sw.cold_residual_energy,
                        "cold_err": rel(E, Einf), "warm_err": rel(Ew, Einf)})
    return out


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--samples", type=int, default=2000)
    p.add_argument("--sizes", default="64,96,128", help="ROI cube sides of the training media (multiples of 16)")
    p.add_argument("--boundary", type=int, default=8)
    p.add_argument("--steps", type=int, default=4000)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--out", default=DEFAULT_OUT)
    p.add_argument("--eval", type=int, default=3, help="held-out media per evaluation size")
    args = p.parse_args(argv)
    sides = [int(v) for v in args.sizes.split(",")]

    from wavesim_b200 import warmstart as W

    t0 = time.time()
    data = W.make_training_set(args.samples, roi=sides, bw=args.boundary, seed=args.seed, tol=1e-4)
    t_data = time.time() - t0
    model = W.WarmStart()
    t0 = time.time()
    losses = model.train(data, args.steps, lr=args.lr,
                         log=lambda s, l: print(json.dumps({"step": s, "loss": l}), flush=True))
    t_train = time.time() - t0
    del data
    # the command that reproduces these weights (every option but the output path)
    stored = {k: v for k, v in vars(args).items() if k != "out"}
    command = "python -m wavesim_b200.train_warmstart " + " ".join(f"--{k} {v}" for k, v in stored.items())
    report = {"command": command, "args": stored, "params": model.net.nparams, "data_s": t_data, "train_s": t_train,
              "final_loss": float(np.mean(losses[-50:]))}
    report["eval"] = evaluate(model, sides, args.eval, boundary=args.boundary)
    for e in report["eval"]:
        print(json.dumps(e), flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    model.save(args.out, bf16=True, provenance=report)
    print(json.dumps({k: v for k, v in report.items() if k != "eval"}), flush=True)
    return report


if __name__ == "__main__":
    main()
