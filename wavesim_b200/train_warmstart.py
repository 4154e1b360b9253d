"""Train the learned warm start on MBS solutions and write its checkpoint.

    python -m wavesim_b200.train_warmstart [--samples 2000] [--roi 64] [--steps 4000] [--out PATH]

The training set is made by this package's own solver: seeded cubes of the
c3 sphere distribution (radius U[0.5, 2] lambda, n = 1.5 in 1.33, 2000
spheres per 224^3) with the c3 plane-wave source, solved to an energy ratio of
1e-4.  Training runs on the GPU with the network's own forward and backward
kernels (wavesim_b200.warmstart; the half-resolution network, ROI sides
multiples of 16).  The checkpoint stores bf16 weights
(``WarmStart.save(..., bf16=True)``); ``WarmStart.load`` reads it back.
At the end the script reports, on held-out media of the training size and
of twice it, the prediction error and the iterations of cold and
warm-started solves at energy threshold 1e-3.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_spheres.npz")


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--samples", type=int, default=2000)
    p.add_argument("--roi", type=int, default=64)
    p.add_argument("--boundary", type=int, default=8)
    p.add_argument("--steps", type=int, default=4000)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--out", default=DEFAULT_OUT)
    p.add_argument("--eval", type=int, default=3, help="held-out media per evaluation size")
    args = p.parse_args(argv)

    import wavesim_b200 as ws
    from wavesim_b200 import warmstart as W
    from wavesim_b200.workloads import sphere_medium

    t0 = time.time()
    data = W.make_training_set(args.samples, roi=args.roi, bw=args.boundary, seed=args.seed, tol=1e-4)
    t_data = time.time() - t0
    model = W.WarmStart()
    t0 = time.time()
    losses = model.train(data, args.steps, lr=args.lr,
                         log=lambda s, l: print(json.dumps({"step": s, "loss": l}), flush=True))
    t_train = time.time() - t0
    del data
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    model.save(args.out, bf16=True)
    report = {"samples": args.samples, "roi": args.roi, "steps": args.steps, "params": model.net.nparams,
              "data_s": t_data, "train_s": t_train, "final_loss": float(np.mean(losses[-50:])), "eval": []}
    rng = np.random.default_rng(12345)
    for roi in [args.roi] + ([2 * args.roi] if 2 * args.roi <= 128 else []):
        for _ in range(args.eval):
            n = sphere_medium(roi, rng)
            opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [args.boundary] * 3}
            src = ws.Source(np.ones((roi, roi)), [1, 1, 1])
            Einf, _ = ws.WaveSim(n, dict(opt, energy_threshold=1e-9)).exec(src)
            sim = ws.WaveSim(n, dict(opt, energy_threshold=1e-3))
            E, st = sim.exec(src)
            Ew, sw = sim.exec(src, warm_start=model)
            rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
            report["eval"].append({"roi": roi, "pred_err": rel(model.predict(n), Einf), "cold_it": st.it - 1,
                                   "warm_it": sw.it - 1, "discarded": sw.warm_discarded,
                                   "cold_err": rel(E, Einf), "warm_err": rel(Ew, Einf)})
            print(json.dumps(report["eval"][-1]), flush=True)
    print(json.dumps({k: v for k, v in report.items() if k != "eval"}), flush=True)
    return report


if __name__ == "__main__":
    main()
