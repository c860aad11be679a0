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
