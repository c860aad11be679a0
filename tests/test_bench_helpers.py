"""bench.py's host-side arithmetic and its CPU sample (no device)."""

from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    sys.path.insert(0, str(ROOT))
    return importlib.import_module("bench")


def test_nn_query_rates():
    bench = _bench()
    # this rank: 1e9 queries in a 500 ms ladder stage; all ranks: 2e9 queries in a 2 s step
    r = bench.nn_query_rates({"ladder": 48.0e9}, {"ladder": 500.0}, 2000.0, 2.0e9)
    assert r["ladder_queries_per_step"] == 2.0e9
    assert r["nn_queries_per_s"] == 2.0e9
    assert r["nn_queries_per_s_whole_step"] == 1.0e9
    assert bench.nn_query_rates({"ladder": 0.0}, {}, 0.0, 0.0)["nn_queries_per_s"] is None


def test_oracle_sample_is_even_and_deterministic():
    bench = _bench()

    class W:
        n_items = 99840

    a = bench.oracle_sample(W(), 512)
    assert len(a) == 512 and a[0] == 0 and a[-1] == 99839
    assert np.all(np.diff(a) > 0)
    assert np.array_equal(a, bench.oracle_sample(W(), 512))

    class Small:
        n_items = 5

    assert np.array_equal(bench.oracle_sample(Small(), 512), np.arange(5))


def test_both_arms_describe_the_workload_alike(monkeypatch):
    """The reference arm and the CUDA arm print the same config dictionary."""
    bench = _bench()
    synth = importlib.import_module("sherd-refit_b200.synth")
    wl = synth.make("slab", 0)

    class Args:
        config = "slab"
        sched = "batched"

    monkeypatch.setenv("WORLD_SIZE", "1")
    a = bench._config_dict(wl, Args())
    b = bench._config_dict(wl, Args())
    assert a == b and a["items"] == 16 and "strong scaling" in a["parallelism"]
