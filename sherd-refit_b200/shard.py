"""One process per GPU: how the batched stage-2 path is spread over ranks.

(pair, start) items are independent, so the path shards without a collective on its data
path. Rank r verifies its own start set for every pair of the collection: the same fragments
and pairs, starts drawn from the seed (seed, r), so each rank carries one collection's worth of
work and the whole job grows with the rank count (weak scaling). Around that:
  * `max_over_ranks`, the job's step time (a one-element MAX all-reduce);
  * `gather_records`, one all-gather of fixed-size result records (sherd_candidate, 808 B) in
    rank order, for a caller that wants every rank's candidates on every rank.
Nothing here reads peer memory; the collectives go through torch.distributed (NCCL on GPUs,
gloo on the CPU).
"""

from __future__ import annotations

import numpy as np

from . import synth


def rank_workload(wl, rank: int, seed: int):
    """The workload rank `rank` verifies: wl itself on rank 0, else the same fragments and pairs
    with starts drawn from the seed (seed, rank)."""
    if rank == 0:
        return wl
    n_starts = len(wl.starts[0]) if wl.starts else 0
    rng = np.random.default_rng((seed, rank))
    pairs, starts = synth._pairs_and_starts(rng, wl.fragments, n_starts,
                                            all_pairs=len(wl.pairs) == _all_pairs(wl))
    assert [(p.a, p.b) for p in pairs] == [(p.a, p.b) for p in wl.pairs]
    return synth.Workload(name=wl.name, fragments=wl.fragments, pairs=pairs, starts=starts,
                          seed=wl.seed)


def _all_pairs(wl):
    n = len(wl.fragments)
    return n * (n - 1) // 2


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_records(records: np.ndarray, device=None) -> list:
    """Every rank's fixed-size records (a structured numpy array, any length per rank), in rank
    order, on every rank: one all-gather of the counts, one of the zero-padded bytes."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [records]
    world = dist.get_world_size()
    item = records.dtype.itemsize
    n = torch.tensor([len(records)], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    counts = [int(c.item()) for c in counts]
    longest = max(counts) * item
    buf = torch.zeros(max(longest, 1), dtype=torch.uint8, device=device)
    raw = np.frombuffer(records.tobytes(), np.uint8)
    buf[:len(raw)] = torch.from_numpy(raw.copy()).to(buf.device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf)
    return [np.frombuffer(b.cpu().numpy()[:c * item].tobytes(), records.dtype)
            for b, c in zip(bufs, counts)]


def partition_pairs(cost, world: int) -> list:
    """Pairs over ranks by estimated cost, longest first onto the least-loaded rank (ties to the
    lower rank): a list per rank of pair indices, ascending. Deterministic, so every rank
    computes the same partition without talking to the others."""
    load = [0.0] * max(int(world), 1)
    out = [[] for _ in load]
    for k in sorted(range(len(cost)), key=lambda k: (-float(cost[k]), k)):
        r = min(range(len(load)), key=lambda r: (load[r], r))
        load[r] += float(cost[k])
        out[r].append(k)
    return [sorted(o) for o in out]


def match_collection_sharded(ctx, fragments, pairs, params, keep: int = 5, seed: int = 0,
                             stage1_floor: float = 0.0, device=None) -> list:
    """pair.match_collection with the pairs shared out over the ranks by estimated cost (the
    fragments' face counts): each rank builds the arrays of only the fragments its pairs touch,
    matches its pairs, and one all-gather of fixed-size candidate records (sherd_candidate, the
    pair field rewritten to the collection's pair index) hands every rank every pair's ranked
    candidates. Returns, per pair, its candidate records in R 5.7's order."""
    import torch.distributed as dist

    from . import pair as pair_mod
    from .backend import CANDIDATE
    on = dist.is_available() and dist.is_initialized()
    rank, world = (dist.get_rank(), dist.get_world_size()) if on else (0, 1)
    cost = [len(fragments[a].f) + len(fragments[b].f) for a, b in pairs]
    mine = partition_pairs(cost, world)[rank]
    res = pair_mod.match_collection(ctx, fragments, [pairs[k] for k in mine], params, keep, seed,
                                    stage1_floor)
    recs = []
    for k, r in zip(mine, res):
        for c in r.candidates:
            rec = np.frombuffer(bytes(c), CANDIDATE).copy()
            rec["pair"] = k
            recs.append(rec)
    mine_recs = np.concatenate(recs) if recs else np.zeros(0, CANDIDATE)
    out = [[] for _ in pairs]
    for part in gather_records(mine_recs, device):
        for rec in part:
            out[int(rec["pair"])].append(rec)
    return out
