"""The fused loop (K3 of each iteration and K1 of the next: on 3-D planes the
split step - x pencils, the column pass, x pencils - or with
WAVESIM_B200_STEP=cluster one kernel on a cluster; on 2-D grids the column
pass alone) against the three separate kernels (WAVESIM_B200_FUSE=0).  Both do
the same arithmetic in the same order, so the fields must agree bit for bit:
cold, warm, batched, with the host loop and with the CUDA graph."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solve(fuse, fn, env=None):
    import wavesim_b200 as ws
    env = dict(env or {})
    env["WAVESIM_B200_FUSE"] = None if fuse else "0"
    old = {k: os.environ.get(k) for k in env}
    try:
        for k, v in env.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        return fn(ws)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def medium(shape, seed=3):
    rng = np.random.default_rng(seed)
    return 1.3 + 0.15 * rng.random(shape) + 0.002j


CLUSTER = {"WAVESIM_B200_STEP": "cluster"}
CASES = {
    # power-of-two planes: the split step (x pencils, column pass, x pencils)
    "64_split": ((32, 32, 32), [16, 16, 16], None),
    "128_split": ((96, 96, 96), [16, 16, 16], None),
    "256_split": ((224, 224, 16), [16, 16, 8], None),
    "256_split_x16": ((224, 224, 16), [16, 16, 8], {"WAVESIM_B200_XTY": "16"}),
    "256_split_vector": ((224, 224, 8), [16, 16, 4], "vector"),
    # 2-D: K2 and the column pass (kc_col_step2d)
    "2d_256": ((224, 224), [16, 16], None),
    "2d_1024": ((960, 960), [32, 32], None),
    "2d_512x120": ((448, 100), [32, 10], None),
    # 2-D on mixed-radix lines (kmc_col_step2d), with a partial last block
    "2d_320": ((256, 256), [32, 32], None),
    "2d_576": ((512, 512), [32, 32], None),
    "2d_320x100": ((256, 68), [32, 16], None),
    # the one-kernel step with the cluster exchange
    "128_cluster2": ((96, 96, 96), [16, 16, 16], CLUSTER),
    "256_cluster8": ((224, 224, 16), [16, 16, 8], CLUSTER),
    # 16-block clusters: K1's half of the exchange pushed (kf_plane_fused_push)
    "256_cluster16": ((224, 224, 16), [16, 16, 8], dict(CLUSTER, WAVESIM_B200_CLUSTER="16")),
    # mixed-radix planes, split step (kt_xpencil_m, kmc_col_step): 192, scalar and vector, and 96
    "192_split": ((160, 160, 8), [16, 16, 4], None),
    "192_split_vector": ((160, 160, 4), [16, 16, 2], "vector"),
    "192_split_x16": ((160, 160, 8), [16, 16, 4], {"WAVESIM_B200_XTY": "16"}),
    "96_split": ((64, 64, 32), [16, 16, 16], None),
    "160_split": ((128, 128, 8), [16, 16, 4], None),
    "224_split": ((192, 192, 8), [16, 16, 4], None),
    # 192-point planes on 6 blocks (km_plane_fused), scalar
    "192_cluster6": ((160, 160, 8), [16, 16, 4], CLUSTER),
    "192_cluster6_vector": ((160, 160, 4), [16, 16, 2], ("vector", CLUSTER)),
    # 160- and 224-point planes on clusters of 5 and 7 blocks
    "160_cluster5": ((128, 128, 8), [16, 16, 4], CLUSTER),
    "224_cluster7": ((192, 192, 8), [16, 16, 4], CLUSTER),
    # K3's rows by per-thread loads instead of one tensor copy (kf_plane_fused)
    "128_cluster2_loads": ((96, 96, 96), [16, 16, 16], dict(CLUSTER, WAVESIM_B200_FUSED_TMA="0")),
    "256_cluster8_loads": ((224, 224, 16), [16, 16, 8], dict(CLUSTER, WAVESIM_B200_FUSED_TMA="0")),
    # 96^2 planes on one block (km_plane_fused with a cluster of 1)
    "96_one_block": ((64, 64, 32), [16, 16, 16], CLUSTER),
    "192_cluster6_loads": ((160, 160, 8), [16, 16, 4], dict(CLUSTER, WAVESIM_B200_FUSED_TMA="0")),
    "96_one_block_loads": ((64, 64, 32), [16, 16, 16], dict(CLUSTER, WAVESIM_B200_FUSED_TMA="0")),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("use_graph", [True, False])
def test_fused_loop_is_bit_identical(gpu, name, use_graph):
    shape, bw, env = CASES[name]
    vector = env == "vector" or (isinstance(env, tuple) and env[0] == "vector")
    env = env[1] if isinstance(env, tuple) else (None if vector else env)
    n = medium(shape)
    opt = {"lambda": 1.0, "pixel_size": 0.125 if vector else 0.25, "boundary_widths": bw,
           "energy_threshold": 1e-3, "max_iterations": 48, "use_graph": use_graph}
    val = np.ones(shape[:2]) + 0.3j
    pos = [1, 1, 1, 2] if vector else [1, 1, 1]

    def run(ws):
        sim = (ws.WaveSimVector if vector else ws.WaveSim)(n, opt)
        from wavesim_b200 import _lib
        fused = _lib.lib.ws_solver_fused(sim.solver()) == 1
        E, st = sim.exec(ws.Source(val, pos))
        sim.close()
        return E, st, fused

    Ef, sf, fused = solve(True, run, env)
    Eu, su, unfused = solve(False, run, env)
    assert fused and not unfused
    assert sf.it == su.it
    np.testing.assert_array_equal(sf.diff_energy, su.diff_energy)
    np.testing.assert_array_equal(Ef, Eu)


def test_fused_warm_and_batched(gpu):
    shape, bw, _ = CASES["128_cluster2"]
    n = medium(shape, 5)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-3,
           "max_iterations": 64}
    rng = np.random.default_rng(9)
    start = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64) * 0.05

    def run(ws):
        sim = ws.WaveSim(n, opt)
        src = ws.Source(np.ones(shape[:2]), [1, 1, 1])
        Ew, sw = sim.exec(src, warm_start=start)
        Eb, sb = sim.exec_batch([src, ws.Source(np.ones((8, 8)), [40, 40, 30])])
        sim.close()
        return Ew, sw, Eb, sb

    Ewf, swf, Ebf, sbf = solve(True, run)
    Ewu, swu, Ebu, sbu = solve(False, run)
    assert swf.it == swu.it and swf.warm_discarded == swu.warm_discarded
    np.testing.assert_array_equal(Ewf, Ewu)
    for a, b in zip(Ebf, Ebu):
        np.testing.assert_array_equal(a, b)
    assert [s.it for s in sbf] == [s.it for s in sbu]


@pytest.mark.parametrize("name", ["256_split", "192_split", "2d_1024", "2d_320"])
@pytest.mark.parametrize("var", ["WAVESIM_B200_PDL", "WAVESIM_B200_FIN"])
def test_loop_variants_are_bit_identical(gpu, name, var):
    """WAVESIM_B200_PDL=1 (the loop's kernels launched with programmatic
    dependent launch, each waiting for the one before it) and
    WAVESIM_B200_FIN=1 (the column pass's last block runs the stop rule, no
    k_finish_iteration) give the same fields and histories as the default."""
    shape, bw, env = CASES[name]
    n = medium(shape)
    opt = {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": bw, "energy_threshold": 1e-3, "max_iterations": 48}
    val = np.ones(shape[:2]) + 0.3j
    pos = [1] * len(shape)

    def run(ws):
        sim = ws.WaveSim(n, opt)
        E, st = sim.exec(ws.Source(val, pos))
        sim.close()
        return E, st

    Ep, sp = solve(True, run, dict(env or {}, **{var: "1"}))
    Eq, sq = solve(True, run, dict(env or {}, **{var: "0"}))
    assert sp.it == sq.it
    np.testing.assert_array_equal(sp.diff_energy, sq.diff_energy)
    np.testing.assert_array_equal(Ep, Eq)
