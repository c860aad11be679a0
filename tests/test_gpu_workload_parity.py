"""The target's parity condition on the synthetic workloads, through the C ABI (-m gpu).

Every (pair, start) item of the slab workload (two fragments, 16 starts) and of two pot pairs
(one adjacent, one not; 64 starts each) goes through the batched CUDA path and through the
oracle. Per item: the same status, the same accept/reject verdict, and the final transform within
1e-4 t (at the moving cloud and at the origin) and 1e-5 rad of the oracle's f64 answer. An item
outside that bound is excused only when the oracle's own ladder is not a function of its input
(the twelve one-ULP neighbours of its start move the oracle's answer out of the bound or flip its
verdict, crates/sherd-gpu/src/crosscheck.rs:197-246), and at most 0.4 of a pair's items may be
excused (crosscheck.rs:76-78).
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(sherd, gpu_ctx, oracle, config, pairs=None):
    synth = importlib.import_module("sherd-refit_b200.synth")
    workload = importlib.import_module("sherd-refit_b200.workload")
    parity = importlib.import_module("oracle.parity")
    wl = synth.make(config, 0)
    params = sherd.default_params()
    dev = workload.to_device(gpu_ctx, wl, params, pairs=pairs)
    got = sherd.candidates(gpu_ctx.ladder_verify_batch(dev.pairs, dev.items, params)).copy()
    got["pair"] = np.asarray(dev.pair_index)[got["pair"].astype(np.int64)]
    opairs, keep = oracle.collection(wl)
    arrays = workload.item_arrays(wl)
    pair, start, inits = arrays
    idx = np.asarray(dev.item_index, np.int64)
    ref, _ = oracle.ladder_verify_items(opairs, oracle.work_items_from(pair[idx], start[idx],
                                                                       inits[idx]),
                                        oracle.default_params())
    ref = np.ctypeslib.as_array(ref)[: len(idx)].copy()
    t, c = parity.item_scale(wl, pair[idx])
    probe = parity.collection_probe(oracle, opairs, oracle.default_params(), arrays, idx, ref, t,
                                    c)
    res = parity.compare(got, ref, t, c, pair_ids=pair[idx], probe=probe)
    print(config, res)
    assert res["items"] == len(idx) > 0
    assert res["determined_status_mismatch"] == 0, res
    assert res["determined_verdict_mismatch"] == 0, res
    assert res["determined_past_bound"] == 0, res
    assert res["chaotic_share_worst_pair"] is not None, res
    assert res["chaotic_share_worst_pair"] <= parity.CHAOTIC_S2, res
    assert res["ok"], res
    del keep
    return res


def test_slab_workload_matches_the_oracle(sherd, gpu_ctx, oracle):
    """The slab workload (config 1's shape): one pair, all 16 starts."""
    res = _check(sherd, gpu_ctx, oracle, "slab")
    assert res["items"] == 16


def test_pot_pairs_match_the_oracle(sherd, gpu_ctx, oracle):
    """Two pairs of the pot workload (config 2's shape), 64 starts each: pair 0 is adjacent
    (starts around the true join), pair 1 is not (starts bring the fracture clouds together)."""
    res = _check(sherd, gpu_ctx, oracle, "pot", pairs=[0, 1])
    assert res["items"] == 128
