"""Candidate-by-candidate comparison of a batch of (pair, start) results with the oracle's.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's CPU-baseline leg, where it is the
checker of the CUDA backend's candidates. The product package never imports it.

What is compared, per (pair, start) item, is what the target condition names: the status, the
accept/reject verdict (identical), and the final transform (the last rung's pose, the one the
verification ran at) against the oracle's f64 answer, within 1e-4 t and 1e-5 rad. The pose gap is
measured as the reference's cross-check measures it (crates/sherd-core/src/matching/icp.rs:799-880,
`pose_gap`):

* rotation: the Frobenius form ||R - R'||_F = 2 sqrt(2) |sin(theta / 2)| (icp.rs:840-849),
  exactly zero for identical bits, reported here in radians;
* translation at the moving cloud: how far the centroid of the moving fracture cloud travels
  between the two poses, in wall thicknesses (icp.rs:871-880, `cloud_t`), the row the
  reference's cross-check gates (crates/sherd-gpu/src/crosscheck.rs:927-960);
* translation at the origin: |tau - tau'| / t (icp.rs:858-864, `origin_t`), D 10.2's own form,
  reported beside it and counted against the same bound.

An item whose pose or verdict is outside the bound is then probed for chaos, as the reference's
cross-check does (crosscheck.rs:197-246, `determined_batch`): the oracle re-climbs the ladder
from the twelve initial poses one ULP away from the item's own (each entry of the 3x4 block moved
to its next representable neighbour, one at a time). The item is *determined* when all twelve
answers land within the bound of the oracle's unperturbed answer with the same verdict; otherwise
its ladder is not a function of its input at double precision, and a difference there measures
the ladder's chaos, not the kernel. Chaotic items are counted and excluded from the bound; the
reference bounds their share per pair at 0.4 (crosscheck.rs:76-78, `CHAOTIC_S2`).
"""

from __future__ import annotations

import numpy as np

TOL_T = 1e-4       # final transforms within 1e-4 t of the FP64 oracle
TOL_RAD = 1e-5     # and 1e-5 rad
CHAOTIC_S2 = 0.4   # crosscheck.rs:76-78: the share of a pair's items the bound may excuse
PAIR_MIN_ITEMS = 8  # the fewest items of a pair over which its chaotic share is taken


def _as_struct(cands) -> np.ndarray:
    if isinstance(cands, np.ndarray):
        return cands
    return np.ctypeslib.as_array(cands)


def final_poses(cands) -> np.ndarray:
    """(n, 4, 4) final transforms: the last rung's pose of each candidate."""
    c = _as_struct(cands)
    return np.asarray(c["rungs"]["transform"][:, 3], np.float64).reshape(-1, 4, 4)


def frobenius_rad(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """pose_gap::frobenius_deg (icp.rs:840-849) in radians, over stacks of 4x4 poses."""
    d = a[..., :3, :3] - b[..., :3, :3]
    fro = np.sqrt(np.sum(d * d, axis=(-2, -1)))
    half = np.clip(fro / (2.0 * np.sqrt(2.0)), -1.0, 1.0)
    return 2.0 * np.arcsin(half)


def origin_t(a: np.ndarray, b: np.ndarray, t) -> np.ndarray:
    """pose_gap::origin_t (icp.rs:858-864): |tau - tau'| / t."""
    d = a[..., :3, 3] - b[..., :3, 3]
    return np.sqrt(np.sum(d * d, axis=-1)) / t


def cloud_t(a: np.ndarray, b: np.ndarray, centre: np.ndarray, t) -> np.ndarray:
    """pose_gap::cloud_t (icp.rs:871-880): the travel of `centre` (source frame) between the two
    poses, in wall thicknesses."""
    delta = (a[..., :3, 3] - b[..., :3, 3]) + np.einsum(
        "...ij,...j->...i", a[..., :3, :3] - b[..., :3, :3], centre)
    return np.sqrt(np.sum(delta * delta, axis=-1)) / t


def next_up(x: float) -> float:
    """f64::next_up: the next representable value towards +infinity."""
    return float(np.nextafter(np.float64(x), np.float64(np.inf)))


def nudged_inits(init: np.ndarray) -> np.ndarray:
    """The twelve one-ULP neighbours of a 4x4 initial pose (crosscheck.rs:231-238): each entry of
    the 3x4 block moved to its next representable neighbour, one at a time."""
    out = np.repeat(np.asarray(init, np.float64).reshape(1, 4, 4), 12, axis=0)
    k = 0
    for i in range(3):
        for j in range(4):
            out[k, i, j] = next_up(out[k, i, j])
            k += 1
    return out


def _stats(x: np.ndarray) -> dict:
    if len(x) == 0:
        return {"max": None, "median": None}
    return {"max": float(np.max(x)), "median": float(np.median(x))}


def determined(oracle, pairs, params, items, base, t, centre) -> np.ndarray:
    """Per item (pair index, start id, init 4x4 in `items`), whether the oracle's own ladder is a
    function of its input: the twelve one-ULP neighbours of its initial pose land within the bound
    of its unperturbed answer `base` (a Candidate row per item) with the same verdict
    (crosscheck.rs:209-246)."""
    n = len(items["pair"])
    if n == 0:
        return np.zeros(0, bool)
    pair = np.repeat(np.asarray(items["pair"], np.uint32), 12)
    start = np.repeat(np.asarray(items["start"], np.uint32), 12)
    inits = np.concatenate([nudged_inits(x) for x in np.asarray(items["init"])]).reshape(-1, 16)
    wi = oracle.work_items_from(pair, start, inits)
    got, _ = oracle.ladder_verify_items(pairs, wi, params, 0)
    got = _as_struct(got)[: 12 * n]
    gp = final_poses(got).reshape(n, 12, 4, 4)
    bp = final_poses(base)[:, None]
    tt = np.asarray(t, np.float64)[:, None]
    cc = np.asarray(centre, np.float64)[:, None]
    within = ((frobenius_rad(gp, bp) <= TOL_RAD) & (cloud_t(gp, bp, cc, tt) <= TOL_T)
              & (origin_t(gp, bp, tt) <= TOL_T))
    same = got["accepted"].reshape(n, 12) == _as_struct(base)["accepted"][:, None]
    return np.all(within & same, axis=1)


def compare(gpu, ref, t, centre, pair_ids=None, probe=None) -> dict:
    """The parity summary of a batch: `gpu` and `ref` are Candidate arrays over the same items in
    the same order, `t` the pair's wall thickness per item and `centre` the moving fracture
    cloud's centroid (source frame) per item. `probe(mask)` returns, for the items selected by
    `mask`, whether each is determined (`determined` bound to the oracle's objects); without it
    every out-of-bound item counts as determined, the strict reading."""
    g, r = _as_struct(gpu), _as_struct(ref)
    n = len(g)
    assert len(r) == n
    t = np.asarray(t, np.float64)
    centre = np.asarray(centre, np.float64).reshape(n, 3)
    gp, rp = final_poses(g), final_poses(r)
    rot = frobenius_rad(gp, rp)
    ct = cloud_t(gp, rp, centre, t)
    ot = origin_t(gp, rp, t)
    status_bad = g["status"] != r["status"]
    verdict_bad = g["accepted"] != r["accepted"]
    past = (rot > TOL_RAD) | (ct > TOL_T) | (ot > TOL_T) | ~np.isfinite(rot) | ~np.isfinite(ct)
    off = past | verdict_bad | status_bad
    det = np.ones(n, bool)
    if probe is not None and off.any():
        det[off] = probe(off)
    chaotic = off & ~det
    acc = r["accepted"] != 0
    bits = np.array([bytes(memoryview(g[k : k + 1])) == bytes(memoryview(r[k : k + 1]))
                     for k in range(n)]) if n else np.zeros(0, bool)
    out = {
        "items": int(n),
        "bound": {"cloud_t": TOL_T, "origin_t": TOL_T, "rot_rad": TOL_RAD},
        "status_mismatch": int(status_bad.sum()),
        "verdict_mismatch": int(verdict_bad.sum()),
        "accepted_gpu": int((g["accepted"] != 0).sum()),
        "accepted_oracle": int(acc.sum()),
        "bit_identical_candidates": int(bits.sum()),
        "rot_rad": _stats(rot), "cloud_t": _stats(ct), "origin_t": _stats(ot),
        "accepted_rot_rad": _stats(rot[acc]), "accepted_cloud_t": _stats(ct[acc]),
        "accepted_origin_t": _stats(ot[acc]),
        "past_bound": int(past.sum()),
        "chaotic": int(chaotic.sum()),
        "determined_past_bound": int((past & det).sum()),
        "determined_verdict_mismatch": int((verdict_bad & det).sum()),
        "determined_status_mismatch": int((status_bad & det).sum()),
        "chaos_probe": ("twelve one-ULP neighbours of each out-of-bound item's initial pose, "
                        "re-climbed by the oracle" if probe is not None else "not run"),
    }
    if probe is not None and off.any():
        out["chaotic_rot_rad"] = _stats(rot[chaotic])
        out["chaotic_cloud_t"] = _stats(ct[chaotic])
    out["chaotic_share"] = float(chaotic.sum()) / n if n else 0.0
    out["chaotic_share_bound"] = CHAOTIC_S2
    worst = None
    if pair_ids is not None:
        # The reference states its bound over a pair's candidates; a share over one or two
        # sampled items of a pair says nothing, so it is taken over pairs with PAIR_MIN_ITEMS
        # or more items in the comparison.
        pair_ids = np.asarray(pair_ids)
        shares = []
        for p in np.unique(pair_ids):
            m = pair_ids == p
            if m.sum() >= PAIR_MIN_ITEMS:
                shares.append(float(chaotic[m].sum()) / float(m.sum()))
        worst = max(shares) if shares else None
        out["pairs_with_share"] = len(shares)
    out["chaotic_share_worst_pair"] = worst
    out["ok"] = bool(out["determined_past_bound"] == 0 and out["determined_verdict_mismatch"] == 0
                     and out["determined_status_mismatch"] == 0
                     and out["chaotic_share"] <= CHAOTIC_S2
                     and (worst is None or worst <= CHAOTIC_S2))
    return out


def collection_probe(oracle, pairs, params, items_all, idx, ref, t, centre):
    """A `probe` for `compare` over the items `idx` of a workload (item arrays `items_all` =
    (pair, start, inits) as workload.item_arrays gives them) whose oracle answers are `ref`."""
    pair, start, inits = items_all
    r = _as_struct(ref)

    def probe(mask):
        sel = np.flatnonzero(mask)
        it = {"pair": pair[idx[sel]], "start": start[idx[sel]], "init": inits[idx[sel]]}
        return determined(oracle, pairs, params, it, r[sel], np.asarray(t)[sel],
                          np.asarray(centre)[sel])
    return probe


def item_scale(wl, pair_index) -> tuple[np.ndarray, np.ndarray]:
    """Per item: the pair's wall thickness (t_pair = min t, scales.rs:94-96) and the centroid of
    the moving fracture cloud (B's pc_frac, B's frame)."""
    t = np.array([min(wl.fragments[p.a].t, wl.fragments[p.b].t) for p in wl.pairs])
    c = np.stack([wl.fragments[p.b].pf.mean(0) for p in wl.pairs])
    pi = np.asarray(pair_index, np.int64)
    return t[pi], c[pi]


__all__ = ["TOL_T", "TOL_RAD", "CHAOTIC_S2", "compare", "determined", "collection_probe",
           "item_scale", "frobenius_rad", "cloud_t", "origin_t", "nudged_inits", "final_poses"]

