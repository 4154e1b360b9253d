#!/usr/bin/env python3
"""Benchmark: time-to-tolerance of the modified Born series on a 3-D 256^3
disordered medium (grid incl. 16-px boundary, ROI 224^3, 2000 spheres of
n = 1.5 in n = 1.33, plane-wave source, energy_threshold 1e-3), on B200.

One step = one complete solve to tolerance (the reference's stop rule,
Simulation.m:193-217, decided on the device), inputs resident in HBM.
``value`` is the job-level time per solve in ms (max over ranks of the
timed region / solves done by all ranks); lower is better.  Multi-GPU runs
are independent replicas (each rank solves its own copy), ``scaling`` weak.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``--impl reference`` times the reference algorithm's CPU implementation (the
FP32 restatement in oracle/, scipy.fft on all host cores) on a bounded sample
of iterations of the same workload and projects it to the reference's
iteration count.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D 256³ time-to-tol 1e-3: plain vs warm-start+batched MBS; % B200 HBM peak"
UNIT = "ms"
WORKLOAD = "c3: 3-D scalar 256^3 grid incl. 16-px boundary (ROI 224^3), 2000 seeded spheres n=1.5 in 1.33, " \
           "plane wave on z=1, energy_threshold 1e-3, 8 wiggles"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c4"])
    p.add_argument("--cpu-iters", type=int, default=3, help="iterations in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-warm", action="store_true", help="skip the learned warm-start leg")
    p.add_argument("--batch", type=int, default=4, help="right-hand sides of the batched leg (0: skip)")
    p.add_argument("--media", type=int, default=48, help="media of mixed sizes in the concurrent leg (0: skip)")
    p.add_argument("--angles", type=int, default=128, help="plane-wave angles on the 1024^2 medium (0: skip)")
    p.add_argument("--sweep-batch", type=int, default=8, help="angles per round of the continuation sweep")
    return p.parse_args()


def dist_setup(backend):
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return torch, dist, ws, rank, local


def max_over_ranks(dist, ws, value, device=None):
    if ws == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi sampling during the timed region (SM clock and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic(kernel):
    """DRAM bytes per launch of `kernel` on this workload from the committed ncu
    summary (profiles/*.md, line 'dram_bytes_per_launch[<kernel>]: N'; the
    256^3 workload's kernels are keyed K1/K2/K3, other workloads prefix their
    config, e.g. c4:K3)."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for f in sorted(os.listdir(pdir)):
        if not f.endswith((".md", ".txt")):
            continue
        m = re.search(r"dram_bytes_per_launch\[%s\]:\s*([0-9.eE+]+)" % re.escape(kernel),
                      open(os.path.join(pdir, f)).read())
        if m:
            return float(m.group(1))
    return None


def load_workloads():
    """wavesim_b200/workloads.py loaded on its own (NumPy only): importing it
    through the package would load the CUDA library, which the reference arm
    must never touch."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("ws_bench_workloads",
                                                  os.path.join(ROOT, "wavesim_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def build_problem(config):
    import wavesim_b200 as ws
    n, opt, val, pos, vector = load_workloads().CONFIGS[config]()
    t = time.time()
    sim = (ws.WaveSimVector if vector else ws.WaveSim)(n, dict(opt, device_setup=True))
    return sim, ws.Source(val, pos), time.time() - t, (n, opt, val, pos, vector)


def reference_iterations(config="c3"):
    """Iterations the oracle's restatement of the reference loop needs to reach
    the tolerance on this workload (tests/golden/make_config_runs.py)."""
    try:
        return json.load(open(os.path.join(ROOT, "tests", "golden", f"{config}_reference_run.json")))["iterations"]
    except Exception:
        return None


def config_dict(config, grid, ws):
    """The `config` object of both arms' JSON lines (same keys, same values)."""
    return {"workload": WORKLOAD if config == "c3" else config, "grid": [int(v) for v in grid],
            "stop_rule": "reference (Simulation.next)",
            "l2": "inputs larger than L2 (each 256^3 c64 array is 134 MB > 126 MB L2)",
            "parallelism": f"replicas x{ws}"}


def cpu_sample(spec, iters, sim=None):
    """The FP32 restatement of the reference loop (oracle/) timed for `iters`
    iterations on all host cores; returns ms per iteration and the
    iterations run (the loop ends on a multiple of Nw)."""
    from oracle import mbs_oracle as ref
    n, opt, val, pos, vector = spec
    if sim is None:
        sim = (ref.WaveSimVector if vector else ref.WaveSim)(n, dict(opt, single_precision=True))
    src = ref.Source(val, pos)
    t = time.perf_counter()
    sim.exec(src, max_iterations=iters)
    dt = time.perf_counter() - t
    nw = len(sim.wiggles)
    done = ((iters + nw - 1) // nw) * nw
    return 1e3 * dt / done, done


def run_reference(args):
    """The reference arm: the reference loop's CPU implementation (the FP32
    restatement in oracle/, scipy.fft on every host core) on the same
    workload, built from the seeded generator and the oracle only - no part
    of the CUDA product is imported or run.  A full solve takes minutes on
    the host, so each step times one wiggle cycle (Nw iterations) of the
    solve and the line reports that per-iteration time times the iterations
    the reference loop needs to reach the tolerance (152 for the 256^3
    workload, tests/golden/c3_reference_run.json)."""
    import scipy.fft  # noqa: F401
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
        if rank != 0:
            dist.barrier()
            dist.destroy_process_group()
            return
    from oracle import mbs_oracle as ref
    spec = load_workloads().CONFIGS[args.config]()
    n, opt, val, pos, vector = spec
    sim = (ref.WaveSimVector if vector else ref.WaveSim)(n, dict(opt, single_precision=True))
    iters_tol = reference_iterations(args.config)
    samples, timed = [], 0
    t_all = time.perf_counter()
    for i in range(args.warmup + args.steps):
        ms_it, done = cpu_sample(spec, 1, sim)
        if i >= args.warmup:
            samples.append(ms_it)
            timed += done
    wall_s = time.perf_counter() - t_all
    ms_it = float(np.mean(samples))
    value = ms_it * iters_tol if iters_tol else None
    threads = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32 complex)", "data": "synthetic (seeded)",
        "config": config_dict(args.config, sim.N, ws),
        "value_kind": f"projection: measured ms per iteration x {iters_tol} iterations to tolerance "
                      f"(a full solve is ~{(value or 0) / 1e3:.0f} s on the host)",
        "ms_per_iteration": ms_it, "iterations_timed": timed, "iterations_to_tol": iters_tol,
        "timed_wall_s": wall_s,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} steps of one wiggle cycle ({timed // max(1, args.steps)} "
                                   f"iterations) each of the {args.config} workload, FP32 scipy.fft "
                                   f"restatement of the reference loop on {threads} threads, "
                                   f"{ms_it:.1f} ms per iteration, projected to the reference's "
                                   f"{iters_tol} iterations to tolerance"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_ours(args):
    torch, dist, ws, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from wavesim_b200 import _lib
    sim, source, setup_s, spec = build_problem(args.config)
    sim.device = local
    h = sim.solver()
    stream_ptr = C.c_void_p()
    _lib.check(_lib.lib.ws_solver_buffers(h, None, C.byref(stream_ptr)))
    stream = torch.cuda.ExternalStream(stream_ptr.value, device=dev)

    # device-resident source blocks and output
    s, blocks, keep = sim.source_blocks(source)
    dev_vals = []
    for i, v in enumerate(keep):
        t = torch.from_numpy(np.ascontiguousarray(v.ravel(order="F")).view(np.float32)).to(dev)
        dev_vals.append(t)
        blocks[i].values = t.data_ptr()
    r = sim.roi
    out_n = int(np.prod([r[1, d] - r[0, d] + 1 for d in range(4)]))
    E_dev = torch.empty(out_n * 2, dtype=torch.float32, device=dev)
    opts = _lib.default_options()
    opts.max_iterations = sim.max_iterations()
    opts.energy_threshold = sim.energy_threshold
    opts.energy_interval = sim.energy_calculation_interval
    opts.output = _lib.WS_OUTPUT_FIELD
    n_it = C.c_int64()
    conv = C.c_int()

    def solve():
        _lib.check(_lib.lib.ws_solver_solve(h, len(s.values), blocks, _lib.WS_DEVICE, C.byref(opts),
                                            E_dev.data_ptr(), _lib.WS_DEVICE, None, C.byref(n_it), C.byref(conv)))

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters = []
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            solve()
            iters.append(int(n_it.value))
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
    local_ms = ev0.elapsed_time(ev1)
    if ws > 1:
        dist.barrier()
    total_ms = max_over_ranks(dist, ws, local_ms, dev)
    ms_per_solve_gpu = local_ms / args.steps
    value = total_ms / (args.steps * ws)
    n_iter = iters[-1]
    # K1, K2, K3 (or K2 and K3 fused with the next K1, plus one K1 per solve)
    # and the stop-rule kernel per iteration, the cycle guard per wiggle
    # cycle, state reset, source scatter, finalize
    per_it = _lib.lib.ws_solver_launches_per_iteration(h)
    fused = _lib.lib.ws_solver_fused(h) == 1
    launches_per_solve = (per_it * n_iter + (n_iter // len(sim.wiggles)) + 1 + len(s.values) + 1
                          + (1 if fused else 0))

    # per-kernel device time (CUDA events on the solver's stream) -> roofline
    ms3 = (C.c_float * 3)()
    by3 = (C.c_double * 3)()
    _lib.check(_lib.lib.ws_solver_time_kernels(h, 24, ms3, by3))
    # K1: wiggle + source + inner (y, x) FFT; K2: outer (z) FFT + Green's
    # function + inverse; K3: inverse inner FFT + unwiggle + mix + accumulate
    # + ROI energy (kf_plane_fwd / kf_pencil / kf_plane_inv on the 256^3 grid)
    names = ["K1", "K2", "K3"]
    peaks, peak_kind = measured_peaks()
    peak = float(peaks.get("hbm_gbs", 6650.0))
    kern = []
    for i in range(3):
        gbs = by3[i] / (ms3[i] * 1e-3) / 1e9
        kern.append({"kernel": names[i], "ms": ms3[i], "algorithmic_bytes": by3[i], "achieved_gbs": gbs,
                     "frac": gbs / peak})
    iter_ms = sum(ms3)
    bytes_iter = sum(by3)
    if fused:
        # the loop runs K2 and K3K1 (K3 of an iteration fused with K1 of the
        # next, kf_plane_fused): the separate K1/K3 above are its parts, timed
        # alone for reference; the roofline is taken on the kernels that run
        msf, byf = C.c_float(), C.c_double()
        _lib.check(_lib.lib.ws_solver_time_fused(h, 24, C.byref(msf), C.byref(byf)))
        gbs = byf.value / (msf.value * 1e-3) / 1e9
        for k in kern:
            if k["kernel"] in ("K1", "K3"):
                k["in_loop"] = False
        kern.append({"kernel": "K3K1", "ms": msf.value, "algorithmic_bytes": byf.value, "achieved_gbs": gbs,
                     "frac": gbs / peak, "in_loop": True})
        iter_ms = ms3[1] + msf.value
        bytes_iter = by3[1] + byf.value
        # the split step: its three kernels (inverse x pencils, the column
        # pass, forward x pencils) are the loop's kernels
        ms_s, by_s = (C.c_float * 3)(), (C.c_double * 3)()
        if _lib.lib.ws_solver_time_split(h, 24, ms_s, by_s) == 0:
            kern[-1]["in_loop"] = False
            kern[-1]["kernel"] = "K3K1 (split step, sum)"
            for nm, i in (("Xinv", 0), ("Ycol", 1), ("Xfwd", 2)):
                g_ = by_s[i] / (ms_s[i] * 1e-3) / 1e9
                kern.append({"kernel": nm, "ms": ms_s[i], "algorithmic_bytes": by_s[i], "achieved_gbs": g_,
                             "frac": g_ / peak, "in_loop": True})
    dom = max([k for k in kern if k.get("in_loop", True)], key=lambda k: k["ms"])

    # e2e: the reference-facing one-shot call (ws_run_algorithm, the MEX
    # argument list) with host buffers: set-up upload, solve, E' download
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, sim, s, keep, torch, dev)
        if ws > 1:
            e2e["value"] = max_over_ranks(dist, ws, e2e["value"] * args.steps, dev) / (args.steps * ws)

    # the other side of the metric: batched right-hand sides, learned warm start
    legs = {}
    if ws == 1 and args.config == "c3":
        if args.batch > 0:
            legs["batched"] = run_batched(args, sim, h, stream, torch, dev, value)
            legs["sweep_256"] = run_sweep_256(args, sim, spec, torch, value)
        if not args.no_warm:
            legs["warm_start"] = run_warm(args, sim, h, s, blocks, opts, torch, dev, E_dev, value)
            if args.batch > 0:
                legs["warm_start_batched"] = run_warm_batched(args, sim, torch, dev, value)
            legs["start_quality"] = run_start_quality(sim, h, s, blocks, opts, torch, dev, n_iter)
        if args.media > 0:
            legs["mixed_media"] = run_media(args)
        if args.angles > 0:
            legs["angles_1024"] = run_angles(args)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ms_it, done = cpu_sample(spec, args.cpu_iters)
        cpu = {"value": ms_it * n_iter, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"{done} MBS iterations of the same 256^3 workload with the FP32 restatement of the "
                         f"reference loop (oracle/, scipy.fft, {os.cpu_count()} threads): "
                         f"{ms_it:.1f} ms/iteration, projected to the {n_iter} iterations to tolerance"}

    if rank == 0:
        ref_it = reference_iterations(args.config)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 (fp32 complex)", "data": "synthetic (seeded)",
            "config": config_dict(args.config, sim.N, ws),
            "iterations_to_tol": n_iter, "reference_iterations_to_tol": ref_it, "converged": bool(conv.value),
            "ms_per_solve_per_gpu": ms_per_solve_gpu, "ms_per_iteration": ms_per_solve_gpu / n_iter,
            "iterations_per_s": n_iter / (ms_per_solve_gpu * 1e-3) * ws,
            "effective_hbm_gbs_per_iteration": bytes_iter / (ms_per_solve_gpu / n_iter * 1e-3) / 1e9,
            "kernels": kern,
            "roofline": {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["achieved_gbs"], "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": dom["achieved_gbs"] / peak,
                         "traffic": profile_traffic(dom["kernel"] if args.config == "c3"
                                                    else "%s:%s" % (args.config, dom["kernel"])),
                         "algorithmic_bytes_per_launch": dom["algorithmic_bytes"]},
            "plain_vs_warm_start_batched": dict(legs, plain_ms_per_solve=value),
            "e2e": e2e, "gpu_launches": launches_per_solve * args.steps, "cpu_baseline": cpu,
            "clocks": clk.summary(), "host_setup_s": setup_s,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_batched(args, sim, h, stream, torch, dev, plain_ms):
    """args.batch plane waves at incidence angles spread over +-30 degrees
    (exp(i k n_bg sin(theta) x) on the z = 1 face) on the c3 medium, one
    batched solve with the sources generated on the device
    (ws_solver_solve_plane_waves, every source with its own stop rule);
    time per solve = batch time / batch size."""
    from wavesim_b200 import _lib
    B = args.batch
    r = sim.roi
    ny, nx = int(r[1, 0] - r[0, 0] + 1), int(r[1, 1] - r[0, 1] + 1)
    k = 2 * np.pi / sim.lambda_ * 1.33 * float(sim.options["pixel_size"])
    angles = np.linspace(-30, 30, B) if B > 1 else np.zeros(1)
    waves = (_lib.ws_plane_wave * B)()
    for i, a in enumerate(angles):
        waves[i] = _lib.ws_plane_wave((C.c_int64 * 4)(int(r[0, 0]), int(r[0, 1]), int(r[0, 2]), 1),
                                      (C.c_int64 * 4)(ny, nx, 1, 1), _lib.ws_complex(1.0, 0.0),
                                      (C.c_double * 3)(0.0, k * np.sin(np.radians(a)), 0.0), 0.0)
    opts = _lib.default_options()
    opts.max_iterations = sim.max_iterations()
    opts.energy_threshold = sim.energy_threshold
    opts.output = _lib.WS_OUTPUT_FIELD
    out_n = ny * nx * int(r[1, 2] - r[0, 2] + 1)
    E = torch.empty(B * out_n * 2, dtype=torch.float32, device=dev)
    n_it = (C.c_int64 * B)()
    conv = (C.c_int * B)()

    def solve():
        _lib.check(_lib.lib.ws_solver_solve_plane_waves(h, B, waves, C.byref(opts), E.data_ptr(), _lib.WS_DEVICE,
                                                        None, 0, n_it, conv))
    for _ in range(max(1, args.warmup)):
        solve()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, args.steps // 2)
    ev0.record(stream)
    for _ in range(steps):
        solve()
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    return {"sources": B, "angles_deg": [float(a) for a in angles], "ms_per_batch": ms,
            "ms_per_solve": ms / B, "iterations": [int(v) for v in n_it], "converged": all(bool(c) for c in conv),
            "speedup_vs_plain": plain_ms / (ms / B), "sources_on": "device (plane-wave descriptors)"}


def run_warm(args, sim, h, s, blocks, opts, torch, dev, E_plain, plain_ms):
    """The learned warm start on the c3 problem: network inference on the
    device (features, encoder-decoder, full-grid start) + the warm-started
    solve, timed together; iterations, discard and the difference from the
    plain answer.  Needs the committed checkpoint of the training script."""
    from wavesim_b200 import _lib, warmstart
    from wavesim_b200.train_warmstart import DEFAULT_OUT
    if not os.path.exists(DEFAULT_OUT):
        return {"unavailable": "no trained checkpoint (python -m wavesim_b200.train_warmstart)"}
    model = warmstart.WarmStart.load(DEFAULT_OUT, device=dev.index or 0)
    n_roi = torch.from_numpy(np.ascontiguousarray(sim.roi_medium().ravel(order="F"))).to(dev)
    n_roi = n_roi.reshape(tuple(int(v) for v in sim.roi_medium().shape))
    E_ref = E_plain.clone()
    E_w = torch.empty_like(E_plain)
    o = _lib.ws_solve_options()
    C.pointer(o)[0] = opts
    o.warm_discard_ratio = sim.warm_discard_ratio
    o.initial_memory = _lib.WS_DEVICE
    n_it, conv = C.c_int64(), C.c_int()

    cold, warm, disc = C.c_double(), C.c_double(), C.c_int()
    rc, rw = C.c_double(), C.c_double()

    def step():
        psi = model.predict_grid(sim, n_roi)
        o.initial_field = psi.data_ptr()
        _lib.check(_lib.lib.ws_solver_solve(h, len(s.values), blocks, _lib.WS_DEVICE, C.byref(o), E_w.data_ptr(),
                                            _lib.WS_DEVICE, None, C.byref(n_it), C.byref(conv)))
        _lib.check(_lib.lib.ws_solver_warm_report(h, 0, C.byref(cold), C.byref(warm), C.byref(disc)))
        _lib.check(_lib.lib.ws_solver_warm_residual(h, 0, C.byref(rc), C.byref(rw)))
        if disc.value:  # given up after one cycle: the cold solve decides
            _lib.check(_lib.lib.ws_solver_solve(h, len(s.values), blocks, _lib.WS_DEVICE, C.byref(opts),
                                                E_w.data_ptr(), _lib.WS_DEVICE, None, C.byref(n_it), C.byref(conv)))
        return psi
    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    steps = max(1, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / steps
    t0 = time.perf_counter()
    for _ in range(steps):
        model.predict_grid(sim, n_roi)
    torch.cuda.synchronize()
    ms_pred = (time.perf_counter() - t0) * 1e3 / steps
    o.initial_field = None
    diff = float((E_w - E_ref).norm() / E_ref.norm())
    return {"ms_per_solve": ms, "ms_inference": ms_pred,
            "iterations": int(n_it.value) + (0 if disc.value else 1),
            "note_iterations": "loop iterations plus the cold probe iteration of a warm start",
            "discarded": bool(disc.value), "first_cycle_energy_ratio": warm.value / cold.value,
            "initial_residual_ratio": (rw.value / rc.value) if rc.value > 0 else None,
            "rel_l2_vs_plain": diff, "speedup_vs_plain": plain_ms / ms, "checkpoint": os.path.relpath(DEFAULT_OUT, ROOT)}


def _tilt(sim, angle_deg, n_bg=1.33):
    """exp(i k n_bg sin(theta) x) over the ROI (y, x, z), and along x: the
    phase of a plane wave tilted in the x-z plane, at the source plane."""
    r = sim.roi
    ny, nx, nz = (int(r[1, d] - r[0, d] + 1) for d in range(3))
    k = 2 * np.pi / sim.lambda_ * n_bg * float(sim.options["pixel_size"])
    ph = np.exp(1j * k * np.sin(np.radians(angle_deg)) * np.arange(nx))
    return np.broadcast_to(ph[None, :, None], (ny, nx, nz)), ph


def run_sweep_256(args, sim, spec, torch, plain_ms):
    """The continuation start on the 256^3 medium: 16 plane waves on the z = 1
    face at incidence angles 0.5 degrees apart (exp(i k n_bg sin(theta) x),
    n_bg 1.33), solved by wavesim_b200.batch.solve_sweep in rounds of 2
    (round 0 cold, every later angle started from its neighbour's field
    tilted on the device) against the same rounds solved cold; both through
    the Python API with the fields copied to the host.  Accuracy of one
    continued field and its cold counterpart against a tight solve
    (threshold 1e-7)."""
    import wavesim_b200 as ws
    from wavesim_b200.batch import solve_sweep
    r = sim.roi
    ny, nx = int(r[1, 0] - r[0, 0] + 1), int(r[1, 1] - r[0, 1] + 1)
    k = 2 * np.pi / sim.lambda_ * 1.33 * float(sim.options["pixel_size"])
    angles = -3.75 + 0.5 * np.arange(16)
    waves = [ws.PlaneWave((ny, nx, 1), [1, 1, 1], phase=(0.0, k * np.sin(np.radians(a)), 0.0)) for a in angles]
    B = 2
    rounds = -(-len(waves) // B)
    solve_sweep(sim, waves[:2 * B], batch=B)  # warm-up: graphs, staging
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Ec, sc = [None] * len(waves), [None] * len(waves)
    for j in range(rounds):
        E, st = sim.exec_batch(waves[j::rounds])
        for i, e, s_ in zip(range(j, len(waves), rounds), E, st):
            Ec[i], sc[i] = e, s_
    torch.cuda.synchronize()
    t_cold = time.perf_counter() - t0
    Ew, sw, t_w = solve_sweep(sim, waves, batch=B)
    torch.cuda.synchronize()
    i = len(waves) // 2 + 1
    tight = ws.WaveSim(spec[0], dict(spec[1], device_setup=True, energy_threshold=1e-7))
    Et, _ = tight.exec_batch([waves[i]])
    tight.close()
    ref = Et[0]
    nr = float(np.linalg.norm(ref))
    n = len(waves)
    return {"angles_deg": [float(a) for a in angles], "batch": B, "rounds": rounds,
            "ms_per_solve": t_w * 1e3 / n, "ms_per_solve_same_rounds_cold": t_cold * 1e3 / n,
            "iterations": [s_.it - 1 for s_ in sw], "iterations_cold": [s_.it - 1 for s_ in sc],
            "discarded": int(sum(bool(getattr(s_, "warm_discarded", False)) for s_ in sw)),
            "speedup_vs_same_rounds_cold": t_cold / t_w,
            "rel_l2_vs_tight_solve": {"angle_deg": float(angles[i]), "cold": float(np.linalg.norm(Ec[i] - ref)) / nr,
                                      "continuation": float(np.linalg.norm(Ew[i] - ref)) / nr},
            "timing": "host wall clock, fields copied to the host included (both sides)"}


def run_warm_batched(args, sim, torch, dev, plain_ms):
    """The two sides together: args.batch plane waves at angles over +-30
    degrees on the c3 medium in one batched solve (exec_batch), each
    warm-started from the network's prediction for normal incidence times the
    tilt's phase across the ROI; the time covers inference and the batched
    solve (and any cold rerun of a discarded start).  Per-solve time against
    the plain single solve."""
    import wavesim_b200 as ws
    from wavesim_b200 import warmstart
    from wavesim_b200.train_warmstart import DEFAULT_OUT
    if not os.path.exists(DEFAULT_OUT):
        return {"unavailable": "no trained checkpoint (python -m wavesim_b200.train_warmstart)"}
    model = warmstart.WarmStart.load(DEFAULT_OUT, device=dev.index or 0)
    B = args.batch
    angles = np.linspace(-30, 30, B) if B > 1 else np.zeros(1)
    r = sim.roi
    ny, nx = int(r[1, 0] - r[0, 0] + 1), int(r[1, 1] - r[0, 1] + 1)
    n_roi = sim.roi_medium()
    srcs = [ws.Source(np.broadcast_to(_tilt(sim, a)[1][None, :], (ny, nx)).copy(), [1, 1, 1]) for a in angles]

    # the tilt of each start over the whole grid (x measured from the ROI's
    # first column, as the sources' phase), applied on the device
    N = [int(v) for v in sim.N[:3]]
    kk = 2 * np.pi / sim.lambda_ * 1.33 * float(sim.options["pixel_size"])
    xg = np.arange(N[1]) - (int(r[0, 1]) - 1)
    tilts = torch.from_numpy(np.stack([np.exp(1j * kk * np.sin(np.radians(a)) * xg)
                                       for a in angles]).astype(np.complex64)).to(dev)

    def step():
        base = model.predict_grid(sim, n_roi).view(N[2], N[1], N[0])  # [z, x, y]: column-major
        starts = (base[None] * tilts[:, None, :, None]).reshape(len(angles), -1)
        return sim.exec_batch(srcs, warm_starts=starts)
    step()
    torch.cuda.synchronize()
    steps = max(1, args.steps // 4)
    t0 = time.perf_counter()
    for _ in range(steps):
        Es, sts = step()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / steps
    return {"sources": B, "angles_deg": [float(a) for a in angles], "ms_per_batch": ms, "ms_per_solve": ms / B,
            "iterations": [int(st.it - 1) for st in sts],
            "discarded": [bool(getattr(st, "warm_discarded", False)) for st in sts],
            "initial_residual_ratio": [float(st.warm_residual_energy / st.cold_residual_energy) for st in sts],
            "speedup_vs_plain": plain_ms / (ms / B),
            "timing": "host wall clock: inference, the starts built on the device, the batched warm solve and "
                      "one batched cold rerun of the discarded starts"}


def run_start_quality(sim, h, s, blocks, opts, torch, dev, plain_it):
    """How good a start must be: the c3 solve warm-started from the converged
    field (energy threshold 1e-7) plus smooth complex noise of relative
    amplitude a, for several a: total iterations (loop + the two probe
    iterations) and the speed-up over the plain solve that a start of that
    quality would give at zero inference cost."""
    from wavesim_b200 import _lib
    r = sim.roi
    shape = tuple(int(r[1, d] - r[0, d] + 1) for d in range(3))
    n_out = int(np.prod(shape))
    E_out = torch.empty(2 * n_out, dtype=torch.float32, device=dev)
    o = _lib.ws_solve_options()
    C.pointer(o)[0] = opts
    o.energy_threshold = 1e-7
    n_it, conv = C.c_int64(), C.c_int()
    _lib.check(_lib.lib.ws_solver_solve(h, len(s.values), blocks, _lib.WS_DEVICE, C.byref(o), E_out.data_ptr(),
                                        _lib.WS_DEVICE, None, C.byref(n_it), C.byref(conv)))
    Einf = E_out.cpu().numpy().view(np.complex64).reshape(shape, order="F")
    tight_it = int(n_it.value)
    rng = np.random.default_rng(5)
    k = [np.fft.fftfreq(n).astype(np.float32) for n in shape]
    lp = np.exp(-(k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2)
                * (2 * np.pi * 2) ** 2 / 2)
    z = np.fft.ifftn(np.fft.fftn(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * lp)
    z *= np.linalg.norm(Einf) / np.linalg.norm(z)
    o2 = _lib.ws_solve_options()
    C.pointer(o2)[0] = opts
    o2.warm_discard_ratio = sim.warm_discard_ratio
    o2.initial_memory = _lib.WS_HOST
    out = []
    for a in (0.02, 0.05, 0.1, 0.2, 0.4):
        u = sim.initial_field((Einf + a * z).astype(np.complex64))
        o2.initial_field = u.ctypes.data
        _lib.check(_lib.lib.ws_solver_solve(h, len(s.values), blocks, _lib.WS_DEVICE, C.byref(o2), E_out.data_ptr(),
                                            _lib.WS_DEVICE, None, C.byref(n_it), C.byref(conv)))
        disc = C.c_int()
        rc_, rw_ = C.c_double(), C.c_double()
        _lib.check(_lib.lib.ws_solver_warm_report(h, 0, None, None, C.byref(disc)))
        _lib.check(_lib.lib.ws_solver_warm_residual(h, 0, C.byref(rc_), C.byref(rw_)))
        # a discarded start stops after the two probe iterations and is rerun cold
        it = int(n_it.value) + 2 + (plain_it if disc.value else 0)
        out.append({"start_error": a, "iterations": it, "discarded": bool(disc.value),
                    "initial_residual_ratio": rw_.value / rc_.value if rc_.value > 0 else None,
                    "speedup_at_zero_inference": plain_it / it})
    o2.initial_field = None
    return {"converged_field_iterations": tight_it, "plain_iterations": plain_it, "curve": out,
            "note": "start = converged field (threshold 1e-7) + smooth noise of relative L2 amplitude start_error; "
                    "speed-up = plain iterations / (warm loop iterations + 2 probe iterations, + the cold "
                    "rerun of a discarded start)"}


def run_media(args):
    """args.media seeded media of mixed sizes (2-D 256^2-1024^2 Gaussian
    random media with a Gaussian-beam edge source, 3-D 64^3-192^3 cubes of the
    sphere distribution with a plane wave), set up on the device, solved
    (1) one at a time, (2) concurrently (wavesim_b200.batch.solve_many, one
    solver stream per medium, 4 host threads) and (3) grouped
    (wavesim_b200.batch.solve_media: the media of each size in one batched
    solve, one launch per kernel for the whole group, the groups on 4 host
    threads); solves/s of each, and the largest difference of a grouped field
    from the medium's own solve."""
    import wavesim_b200 as ws
    from wavesim_b200.batch import group_media, solve_many, solve_media
    from wavesim_b200.workloads import PPW, gaussian_random_field, sphere_medium
    rng = np.random.default_rng(48)
    probs, sizes = [], []
    t0 = time.perf_counter()
    for i in range(args.media):
        if i % 2 == 0:
            side = int(rng.choice([256, 384, 512, 768, 1024]))
            n = np.clip(1.0 + 0.3 * gaussian_random_field((side, side), PPW, rng), 0.8, 1.6) + 0.01j
            opt = {"lambda": 1.0, "pixel_size": 1.0 / PPW, "boundary_widths": [32, 32], "energy_threshold": 1e-3,
                   "device_setup": True}
            y = np.arange(side)
            src = ws.Source(np.exp(-((y - side / 2) ** 2) / (4 * PPW) ** 2)[:, None], [1, 1])
            sizes.append(f"2d {side}^2")
        else:
            side = int(rng.choice([64, 96, 128, 160, 192]))
            n = sphere_medium(side, rng)
            opt = {"lambda": 1.0, "pixel_size": 1.0 / PPW, "boundary_widths": [16, 16, 16], "energy_threshold": 1e-3,
                   "device_setup": True}
            src = ws.Source(np.ones((side, side)), [1, 1, 1])
            sizes.append(f"3d {side}^3")
        probs.append((ws.WaveSim(n, opt), src))
    setup_s = time.perf_counter() - t0
    solve_many(probs, workers=1)  # warm-up: solvers, graphs
    E_seq, st_seq, t_seq = solve_many(probs, workers=1)
    _, st_par, t_par = solve_many(probs, workers=4)
    _, _, _, batches = solve_media(probs, workers=4)  # warm-up: media solvers, graphs
    E_grp, st_grp, t_grp, _ = solve_media(probs, workers=4, batches=batches)
    diff = max(float(np.max(np.abs(a - b))) for a, b in zip(E_grp, E_seq))
    same_it = all(a.it == b.it for a, b in zip(st_grp, st_seq))
    groups = group_media(probs)
    for b in batches:
        if b is not None:
            b.close()
    for sim, _ in probs:
        sim.close()
    return {"media": sizes, "groups": [len(g) for g in groups], "host_setup_s": setup_s,
            "iterations": [s.it - 1 for s in st_seq],
            "sequential_solves_per_s": len(probs) / t_seq, "concurrent_solves_per_s": len(probs) / t_par,
            "grouped_solves_per_s": len(probs) / t_grp, "speedup": t_seq / t_par,
            "grouped_speedup": t_seq / t_grp, "grouped_max_abs_diff": diff, "grouped_same_iterations": same_it,
            "timing": "host wall clock around the solves (set-up excluded)"}


def run_angles(args):
    """C5's angle sweep: args.angles plane waves at incidence angles uniform in
    +-30 degrees on the c2 medium (2-D 1024^2, Gaussian random field), one
    batched solve (sources generated on the device) against single solves of
    a sample of 8 of the angles; then the continuation sweep
    (wavesim_b200.batch.solve_sweep: rounds of args.sweep_batch angles, each
    later angle warm-started from its neighbour's tilted field) against the
    same rounds cold, and the accuracy of cold and continued fields against
    tight solves at three angles."""
    import torch
    import wavesim_b200 as ws
    n, opt, _, _, _ = load_workloads().CONFIGS["c2"]()
    sim = ws.WaveSim(n, dict(opt, device_setup=True))
    r = sim.roi
    ny = int(r[1, 0] - r[0, 0] + 1)
    k = 2 * np.pi / sim.lambda_ * float(opt["pixel_size"])
    angles = np.linspace(-30, 30, args.angles)
    waves = [ws.PlaneWave((ny, 1), [1, 1], amplitude=1.0, phase=(k * np.sin(np.radians(a)), 0.0)) for a in angles]
    sim.exec_batch(waves)  # warm-up: graph, and the pinned output staging at the batch's size
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Eb, sb = sim.exec_batch(waves)
    torch.cuda.synchronize()
    t_b = time.perf_counter() - t0
    sample = waves[:: max(1, len(waves) // 8)][:8]
    sim.exec_batch(sample[:1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its = []
    for w in sample:
        _, st = sim.exec_batch([w])
        its.append(st[0].it - 1)
    torch.cuda.synchronize()
    t_s = (time.perf_counter() - t0) / len(sample)
    # continuation: rounds of args.sweep_batch angles, each angle after the
    # first round warm-started from its neighbour's field tilted to its angle
    from wavesim_b200.batch import solve_sweep
    solve_sweep(sim, waves[:2 * args.sweep_batch], batch=args.sweep_batch)  # warm-up: the warm graph
    torch.cuda.synchronize()
    # the same rounds cold, to separate the starts' gain from the batch size
    rounds = -(-len(waves) // args.sweep_batch)
    t0 = time.perf_counter()
    cold_it = []
    for j in range(rounds):
        _, st = sim.exec_batch(waves[j::rounds])
        cold_it += [x.it - 1 for x in st]
    torch.cuda.synchronize()
    t_rc = time.perf_counter() - t0
    Ew, sw, t_w = solve_sweep(sim, waves, batch=args.sweep_batch)
    torch.cuda.synchronize()
    # accuracy of both against tight solves (threshold 1e-9) at a few angles
    simt = ws.WaveSim(n, dict(opt, device_setup=True, energy_threshold=1e-9))
    errs = []
    for i in (len(waves) // 4 + 1, len(waves) // 2 + 1, 3 * len(waves) // 4 + 1):
        Et, _ = simt.exec_batch([waves[i]])
        ref = Et[0]
        nr = float(np.linalg.norm(ref))
        errs.append({"angle_deg": float(angles[i]), "cold": float(np.linalg.norm(Eb[i] - ref)) / nr,
                     "continuation": float(np.linalg.norm(Ew[i] - ref)) / nr})
    simt.close()
    sim.close()
    warm_it = [x.it - 1 for x in sw]
    round_max = [max(warm_it[j::rounds]) for j in range(rounds)]
    return {"angles": len(waves), "grid": [int(v) for v in sim.N[:2]], "ms_batch": t_b * 1e3,
            "ms_per_solve_batched": t_b * 1e3 / len(waves), "ms_per_solve_single": t_s * 1e3,
            "speedup": t_s * len(waves) / t_b, "iterations": [s.it - 1 for s in sb][:: max(1, len(waves) // 8)],
            "single_iterations": its,
            "continuation": {"rounds": rounds, "batch": args.sweep_batch,
                             "ms_per_solve": t_w * 1e3 / len(waves),
                             "ms_per_solve_same_rounds_cold": t_rc * 1e3 / len(waves),
                             "mean_iterations": float(np.mean(warm_it)),
                             "mean_iterations_cold": float(np.mean(cold_it)),
                             "round_max_iterations": round_max,
                             "iterations_sample": warm_it[:: max(1, len(waves) // 16)],
                             "discarded": int(sum(bool(getattr(x, "warm_discarded", False)) for x in sw)),
                             "speedup_vs_single": t_s * len(waves) / t_w,
                             "speedup_vs_batched_cold": t_b / t_w,
                             "rel_l2_vs_tight_solve": errs,
                             "note": "round 0 cold; every later angle starts from its neighbour's field "
                                     "times the tilt between the two plane waves (wavesim_b200.batch.solve_sweep)"},
            "timing": "host wall clock, fields copied to the host included"}


def run_e2e(args, sim, s, keep, torch, dev):
    """ws_run_algorithm on pinned host buffers: H2D of gamma, wiggles and source,
    the solve, D2H of E' and the energy history, every step."""
    from wavesim_b200 import _lib
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    gamma = pin(np.asfortranarray(sim.gamma).ravel(order="F"))
    wkeep = []
    wig = (_lib.ws_wiggle * len(sim.wiggles))()
    for i, w in enumerate(sim.wiggles):
        parts = [pin(a) for a in (w.pxe, w.pye, w.pze, w.gx, w.gy, w.gz)]
        wkeep.extend(parts)
        wig[i] = _lib.ws_wiggle(*[p.ctypes.data for p in parts])
    blocks = (_lib.ws_source_block * len(keep))()
    vkeep = []
    for i, (p, v) in enumerate(zip(s.positions, keep)):
        pv = pin(np.asfortranarray(v).ravel(order="F"))
        vkeep.append(pv)
        blocks[i] = _lib.ws_source_block((C.c_int64 * 4)(*[int(a) for a in p]),
                                         (C.c_int64 * 4)(*[int(a) for a in v.shape]), pv.ctypes.data)
    npts_c = int(np.prod(sim.N))
    E = pin(np.zeros(npts_c, np.complex64))
    maxit = sim.max_iterations()
    hist = pin(np.zeros(maxit + 64))
    N = (C.c_int64 * 4)(*[int(v) for v in sim.N])
    n_it = C.c_int64()

    def call():
        _lib.check(_lib.lib.ws_run_algorithm(
            N, gamma.ctypes.data, len(sim.wiggles), wig, len(keep), blocks, C.c_float(sim.epsilon),
            _lib.ws_complex(sim.k02e.real, sim.k02e.imag), sim._roi8(), maxit, sim.energy_threshold,
            b"NoCallback", sim.callback_interval, _lib.CALLBACK(), None, _lib.WS_HOST, E.ctypes.data,
            hist.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n_it)))

    call()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        call()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t) * 1e3 / args.steps
    h2d = gamma.nbytes + sum(a.nbytes for a in wkeep) + sum(a.nbytes for a in vkeep)
    d2h = E.nbytes + 8 * int(n_it.value)
    return {"value": ms, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "api": "ws_run_algorithm (RunWaveSimAlgorithmMex argument list), host pinned buffers, "
                   "host wall clock around the blocking call"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
