"""bench.py's host-side arithmetic (no device)."""

from __future__ import annotations

import importlib
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_nn_query_rates():
    sys.path.insert(0, str(ROOT))
    bench = importlib.import_module("bench")
    r = bench.nn_query_rates({"ladder": 48.0e9}, {"ladder": 500.0}, 2000.0, 2)
    assert r["ladder_queries_per_step"] == 1.0e9
    assert r["nn_queries_per_s"] == 2.0e9
    assert r["nn_queries_per_s_whole_step"] == 1.0e9
    assert bench.nn_query_rates({"ladder": 0.0}, {}, 0.0, 1)["nn_queries_per_s"] is None
