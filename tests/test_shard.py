"""The multi-rank host logic of the batched path, on two gloo ranks on the CPU.

Each rank verifies its own start set for the same pairs (weak scaling); the job's step time
is the maximum over ranks; results travel as fixed-size records in one all-gather. No GPU is
needed: the collectives run on gloo with world size 2.
"""

from __future__ import annotations

import importlib
import os
import socket
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        synth = importlib.import_module("sherd-refit_b200.synth")
        shard = importlib.import_module("sherd-refit_b200.shard")
        backend = importlib.import_module("sherd-refit_b200.backend")
        workload = importlib.import_module("sherd-refit_b200.workload")
        base = synth.make("slab", 0)
        wl = shard.rank_workload(base, rank, 0)
        assert [(p.a, p.b) for p in wl.pairs] == [(p.a, p.b) for p in base.pairs]
        items = np.frombuffer(bytes(backend.work_item_array(*workload.item_arrays(wl))),
                              backend.WORK_ITEM)
        assert len(items) == base.n_items
        everyone = shard.gather_records(items)
        assert len(everyone) == world and np.array_equal(everyone[rank], items)
        assert np.array_equal(everyone[0]["init"], np.frombuffer(bytes(backend.work_item_array(
            *workload.item_arrays(base))), backend.WORK_ITEM)["init"])
        for other in range(world):
            if other != rank:
                assert not np.array_equal(everyone[other]["init"], items["init"])
        ragged = shard.gather_records(items[:rank + 1])
        assert [len(r) for r in ragged] == [r + 1 for r in range(world)]
        assert shard.max_over_ranks(1.5 + rank) == 1.5 + (world - 1)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_starts_and_gather_the_records():
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(2, _free_port()), nprocs=2, join=True)


def test_partition_pairs_balances_and_covers():
    shard = importlib.import_module("sherd-refit_b200.shard")
    parts = shard.partition_pairs([5, 1, 4, 2, 3, 3], 2)
    assert sorted(k for p in parts for k in p) == list(range(6))
    assert parts == [[0, 1, 5], [2, 3, 4]]          # longest first: loads 9 and 9
    assert shard.partition_pairs([1, 1], 3) == [[0], [1], []]


def _rank_match(rank, world, port):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    try:
        oracle = importlib.import_module("oracle")
        sherd = importlib.import_module("sherd-refit_b200")
        shard = importlib.import_module("sherd-refit_b200.shard")
        pm = importlib.import_module("sherd-refit_b200.pair")
        from _slab import piece
        from test_pair import _OracleCollectionDevice, _params
        with np.load(ROOT / "tests" / "golden" / "slab.npz") as z:
            slab = {k: z[k] for k in z.files}
        frags = []
        for name in ("pieceA", "pieceB"):
            p = piece(slab, name)
            frags.append(pm.FragmentInput(p["V"], p["F"], p["frac"], float(p["thick_t"]),
                                          float(p["res"]), bool(p["watertight"])))
        dev = _OracleCollectionDevice(oracle)
        pairs = [(0, 1), (0, 1), (0, 1)]
        out = shard.match_collection_sharded(dev, frags, pairs, _params(sherd, slab))
        assert [len(o) for o in out] == [5, 5, 5]
        for o in out:                                   # every rank's copy of the same pair
            assert bytes(o[0]["rungs"]) == bytes(out[0][0]["rungs"]) and o[0]["accepted"] == 1
            s = [r["scores"]["seam"] * r["scores"]["tight"] for r in o]
            assert all(x >= y for x, y in zip(s, s[1:]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_pairs_of_a_collection():
    import torch.multiprocessing as mp
    mp.spawn(_rank_match, args=(2, _free_port()), nprocs=2, join=True)
