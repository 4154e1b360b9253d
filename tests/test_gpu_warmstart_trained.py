"""What the trained warm-start network gains over the method without it.

The committed checkpoint (wavesim_b200/data/warmstart_spheres.npz, made by
python -m wavesim_b200.train_warmstart with the command stored in it) is
loaded and used on held-out media of its training distribution (seeds apart
from the training set's): every medium is solved cold - the reference loop,
the method without the network - and warm-started from the network's
prediction, both to the same energy tolerance.  The warm solve must take
fewer iterations in total (its loop plus the cold probe and residual probe
iterations) and end at least about as close to the converged field
(energy threshold 1e-9) as the cold solve.
"""
import os

import pytest

pytestmark = pytest.mark.gpu


def test_checkpoint_records_its_training_command(gpu):
    from wavesim_b200.train_warmstart import DEFAULT_OUT
    from wavesim_b200.warmstart import WarmStart
    prov = WarmStart.provenance(DEFAULT_OUT)
    assert prov is not None and prov["command"].startswith("python -m wavesim_b200.train_warmstart")
    assert prov["args"]["samples"] >= 1000 and prov["eval"]


def test_trained_network_saves_iterations(gpu):
    from wavesim_b200.train_warmstart import DEFAULT_OUT, evaluate
    from wavesim_b200.warmstart import WarmStart
    assert os.path.exists(DEFAULT_OUT)
    model = WarmStart.load(DEFAULT_OUT, device=0)
    rows = evaluate(model, [64], 3, seed=777)
    cold = sum(r["cold_it"] for r in rows)
    warm = sum(r["warm_it"] for r in rows)
    for r in rows:
        assert not r["discarded"], r
        assert r["residual_ratio"] < 1.0, r
        assert r["warm_err"] <= 1.5 * r["cold_err"] + 1e-4, r
    assert warm < cold, rows
