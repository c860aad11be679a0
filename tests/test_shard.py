"""The multi-rank host logic of the batched path, on two gloo ranks on the CPU.

A collection is split by pairs over the ranks by estimated cost (the survey's collection plan,
crates/sherd-core/src/pipeline.rs:1615-1690); each rank holds only the fragments its pairs touch
and verifies its pairs' items; one all-gather of fixed-size candidate records gives every rank
every item's candidate. The job's step time is the maximum over ranks. No GPU is needed: the
collectives run on gloo with world size 2, and the verification runs on an oracle-backed stand-in
for the device context.
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


class _OracleContext:
    """The constructors workload.to_device calls and the batched call, answered by the oracle."""

    def __init__(self, oracle):
        self.o = oracle

    def mesh(self, v, f):
        return self.o.Mesh(v, f)

    def surfaces(self, fracture, mesh, watertight, frac_area, pf, s, brk_p, brk_ns, margin_p,
                 margin_n):
        return self.o.Surfaces(fracture, mesh, watertight, frac_area, pf, s, brk_p, brk_ns,
                               margin_p, margin_n)

    def cloud(self, p, n):
        return self.o.Cloud(p, n)

    def pair(self, a, b, reg_t, frac_t, reg_p, frac_p, scales):
        return self.o.Pair(a, b, reg_t, frac_t, reg_p, frac_p,
                           self.o.Scales.from_buffer_copy(scales))

    def ladder_verify_batch(self, pairs, items, params, sched=0):
        out, _ = self.o.ladder_verify_items(pairs, items, self.o.Params.from_buffer_copy(params))
        return out


def small_collection():
    """Six pairs of the pot workload (seven fragments), two starts each."""
    synth = importlib.import_module("sherd-refit_b200.synth")
    wl = synth.make("pot", 0)
    return synth.Workload(name="pot6", fragments=wl.fragments, pairs=wl.pairs[:6],
                          starts=[s[:2] for s in wl.starts[:6]], seed=0)


def _rank_main(rank, world, port):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=300))
    try:
        oracle = importlib.import_module("oracle")
        shard = importlib.import_module("sherd-refit_b200.shard")
        backend = importlib.import_module("sherd-refit_b200.backend")
        workload = importlib.import_module("sherd-refit_b200.workload")
        wl = small_collection()
        ctx = _OracleContext(oracle)
        params = backend.default_params()
        parts = shard.partition_pairs(shard.pair_costs(wl), world)
        assert all(parts) and sorted(k for p in parts for k in p) == list(range(len(wl.pairs)))
        mine = shard.rank_pairs(wl, rank, world)
        assert mine == parts[rank]
        dev = workload.to_device(ctx, wl, params, pairs=mine)
        touched = {f for k in mine for f in (wl.pairs[k].a, wl.pairs[k].b)}
        assert len(dev.meshes) == len(touched) < len(wl.fragments)
        assert dev.n_items == sum(len(wl.starts[k]) for k in mine)
        got = backend.candidates(ctx.ladder_verify_batch(dev.pairs, dev.items, params))
        full = shard.gather_candidates(wl, dev, got)
        # one rank over the whole collection, byte for byte
        one = workload.to_device(ctx, wl, params)
        want = backend.candidates(ctx.ladder_verify_batch(one.pairs, one.items, params))
        assert full.tobytes() == want[: wl.n_items].tobytes()
        assert np.array_equal(full["pair"], workload.item_arrays(wl)[0])
        assert shard.max_over_ranks(1.5 + rank) == 1.5 + (world - 1)
        assert shard.sum_over_ranks(1.0 + rank) == world * (world + 1) / 2
        ragged = shard.gather_records(np.asarray(got)[:rank + 1])
        assert [len(r) for r in ragged] == [r + 1 for r in range(world)]
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_a_collection_by_pairs_and_gather_every_candidate():
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(2, _free_port()), nprocs=2, join=True)


def test_one_rank_gather_is_the_candidates_themselves():
    """Without a process group, a device collection that holds every pair and item in the
    workload's order gathers to the candidates array itself (nothing to move); one that holds
    them in another order goes through the general path and comes back in the workload's
    order with the workload's pair indices."""
    from types import SimpleNamespace
    oracle = importlib.import_module("oracle")
    shard = importlib.import_module("sherd-refit_b200.shard")
    backend = importlib.import_module("sherd-refit_b200.backend")
    workload = importlib.import_module("sherd-refit_b200.workload")
    wl = small_collection()
    ctx = _OracleContext(oracle)
    params = backend.default_params()
    dev = workload.to_device(ctx, wl, params)
    got = backend.candidates(ctx.ladder_verify_batch(dev.pairs, dev.items, params))[:wl.n_items]
    assert shard.gather_candidates(wl, dev, got) is got
    # The same candidates as a rank that holds the pairs reversed (device pair k is the
    # workload's pair n - 1 - k) and its items in reverse order.
    n_pairs = len(wl.pairs)
    flipped = got[::-1].copy()
    flipped["pair"] = n_pairs - 1 - flipped["pair"].astype(np.int64)
    fake = SimpleNamespace(pair_index=np.arange(n_pairs)[::-1].copy(),
                           item_index=np.arange(wl.n_items)[::-1].copy())
    back = shard.gather_candidates(wl, fake, flipped)
    assert back is not flipped and back.tobytes() == got.tobytes()


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
        # The swapped pair is a different question (B fixed, A moving), so the ranks' shares
        # differ: two pairs on rank 0, one on rank 1.
        pairs = [(0, 1), (1, 0), (0, 1)]
        assert shard.partition_pairs([1, 1, 1], world) == [[0, 2], [1]]
        params = _params(sherd, slab)
        out = shard.match_collection_sharded(dev, frags, pairs, params)
        assert [len(o) for o in out] == [5, 5, 5]
        for o in out:
            s = [r["scores"]["seam"] * r["scores"]["tight"] for r in o]
            assert all(x >= y for x, y in zip(s, s[1:]))
        assert out[0][0]["accepted"] == 1
        # Against one process matching the whole pair list: the same records, byte for byte.
        whole = pm.match_collection(dev, frags, pairs, params)
        for k, (o, w) in enumerate(zip(out, whole)):
            assert len(o) == len(w.candidates)
            for rec, c in zip(o, w.candidates):
                want = np.frombuffer(bytes(c), rec.dtype).copy()
                want["pair"] = k
                assert rec.tobytes() == want.tobytes()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_pairs_of_a_collection():
    import torch.multiprocessing as mp
    mp.spawn(_rank_match, args=(2, _free_port()), nprocs=2, join=True)
