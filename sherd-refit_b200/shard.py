"""One process per GPU: how the batched stage-2 path is spread over ranks.

(pair, start) items are independent, so the path shards without a collective on its data path
(the collection plan of the reference's matching stage, crates/sherd-core/src/pipeline.rs:1615-1690,
`match_all` over blocks of pairs). A collection is split by pairs:
  * `pair_costs` estimates each pair's device time from its point and sample counts;
  * `partition_pairs` shares the pairs out, longest first onto the least-loaded rank, the same
    on every rank without a message;
  * each rank makes resident only the fragments its pairs touch (workload.to_device with
    `pairs`) and runs one batched call over its pairs' items;
  * `gather_candidates` ends the job with one all-gather of fixed-size candidate records
    (sherd_candidate, 808 B) rewritten to the collection's pair indices, which puts every item's
    candidate, in the collection's item order, on every rank.
Around that, `max_over_ranks` gives the job's step time (a one-element MAX all-reduce). The
total work is fixed whatever the rank count (strong scaling). Nothing here reads peer memory;
the collectives go through torch.distributed (NCCL on GPUs, gloo on the CPU).
"""

from __future__ import annotations

import numpy as np

# Device seconds per algorithmic byte of the two halves of an item, from the batched path on the
# 40-fragment collection: the ICP ladder moves about 800 GB/s of its 48 B point-iterations, the
# penetration wavefront about 60 GB/s of its 24 B surface-sample queries. Only the ratio matters.
LADDER_S_PER_BYTE = 1.0 / 800e9
PEN_S_PER_BYTE = 1.0 / 60e9
PASSES_PER_RUNG = 12.0


def pair_costs(wl) -> np.ndarray:
    """Estimated device seconds of each pair's items: per start, the four rungs over B's
    registration and fracture clouds (PASSES_PER_RUNG passes of 48 B per point) and the
    penetration queries of both sides' surface samples (24 B each)."""
    out = np.empty(len(wl.pairs))
    for k, (p, st) in enumerate(zip(wl.pairs, wl.starts)):
        a, b = wl.fragments[p.a], wl.fragments[p.b]
        ladder = 2.0 * (len(b.reg_p) + len(b.pf)) * PASSES_PER_RUNG * 48.0
        pen = (len(a.s) + len(b.s)) * 24.0
        out[k] = len(st) * (ladder * LADDER_S_PER_BYTE + pen * PEN_S_PER_BYTE)
    return out


def rank_pairs(wl, rank: int, world: int) -> list:
    """The pairs (indices into wl.pairs, ascending) rank `rank` of `world` verifies."""
    return partition_pairs(pair_costs(wl), world)[rank]


def gather_candidates(wl, dev, cands, device=None) -> np.ndarray:
    """Every item's candidate in the collection's item order, on every rank: this rank's
    candidates (a structured sherd_candidate array over dev's items) get the collection's pair
    index and travel with their item index in one all-gather of fixed-size records."""
    import torch.distributed as dist
    from .backend import CANDIDATE
    cands = np.asarray(cands)
    alone = not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1
    if alone and len(cands) == wl.n_items and _identity(dev.item_index) \
            and _identity(dev.pair_index):
        return cands  # one rank holding the whole collection in its own order: nothing to move
    mine = cands.copy()
    mine["pair"] = np.asarray(dev.pair_index, np.int64)[cands["pair"].astype(np.int64)]
    rec = np.dtype([("item", np.uint64), ("cand", CANDIDATE)])
    recs = np.zeros(len(mine), rec)
    recs["item"] = np.asarray(dev.item_index, np.uint64)
    recs["cand"] = mine
    out = np.zeros(wl.n_items, CANDIDATE)
    seen = np.zeros(wl.n_items, bool)
    for part in gather_records(recs, device):
        idx = part["item"].astype(np.int64)
        out[idx] = part["cand"]
        seen[idx] = True
    if not seen.all():
        raise RuntimeError(f"{int((~seen).sum())} items were verified by no rank")
    return out


def _identity(index) -> bool:
    """Whether an index array is 0, 1, ..., len - 1 (no array: the identity)."""
    if index is None:
        return True
    index = np.asarray(index)
    return bool(np.array_equal(index, np.arange(len(index), dtype=index.dtype)))


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    """The sum of x over all ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
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
