"""A synthetic collection (synth.Workload) made resident on the device.

Per fragment: the working-mesh LBVH, the fracture-face LBVH (RayScene::of_subset), the R 6
Surfaces and the two ICP targets (pc_reg, pc_frac with normals). Per pair (A fixed, B moving,
R 0's convention): B's two moving clouds, both Surfaces and the pair's Scales
(Scales::for_fragments, matching/scales.rs:94-96: t_pair = min t, res_pair = max res).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi as A
from .backend import Context, default_params, scales_for_pair, work_item_array


@dataclass
class DeviceCollection:
    ctx: Context
    meshes: list
    fractures: list
    surfaces: list
    reg_targets: list
    frac_targets: list
    pairs: list
    scales: list
    items: object          # ctypes WorkItem array (pair = index into `pairs`)
    n_src: np.ndarray      # (n_pairs, 2): |pc_reg of B|, |pc_frac of B|
    pair_index: np.ndarray | None = None  # per device pair, its index in the workload's pairs
    item_index: np.ndarray | None = None  # per work item, its index in the workload's item list

    @property
    def n_items(self):
        return len(self.items)


def pair_scales(wl, params=None):
    params = params or default_params()
    out = []
    for p in wl.pairs:
        a, b = wl.fragments[p.a], wl.fragments[p.b]
        out.append(scales_for_pair(params, min(a.t, b.t), max(a.res, b.res)))
    return out


def item_arrays(wl):
    """(pair index, start id, init poses) of every work item, pair-major."""
    pair = np.concatenate([np.full(len(s), k, np.uint32) for k, s in enumerate(wl.starts)])
    start = np.concatenate([np.arange(len(s), dtype=np.uint32) for s in wl.starts])
    inits = np.concatenate([s.reshape(-1, 16) for s in wl.starts])
    return pair, start, inits


def to_device(ctx: Context, wl, params: A.Params | None = None, pairs=None) -> DeviceCollection:
    """The workload made resident through `ctx`. `pairs` (indices into wl.pairs, ascending)
    restricts it to those pairs' items and to the fragments they touch, as one rank of a
    cost-partitioned collection holds them; the device pair index of a work item is then its
    position in `pairs`, and `item_index` maps each work item back to the workload's item list."""
    keep = np.arange(len(wl.pairs)) if pairs is None else np.asarray(pairs, np.int64)
    used = sorted({f for k in keep for f in (wl.pairs[k].a, wl.pairs[k].b)})
    meshes, fractures, surfaces, reg_t, frac_t = ({}, {}, {}, {}, {})
    for i in used:
        fr = wl.fragments[i]
        m = ctx.mesh(fr.v, fr.f)
        fm = m.subset(fr.frac)
        meshes[i] = m
        fractures[i] = fm
        surfaces[i] = ctx.surfaces(fm, m, True, fr.frac_area, fr.pf, fr.s, fr.brk_p, fr.brk_ns,
                                   fr.margin_p, fr.margin_n)
        reg_t[i] = ctx.cloud(fr.reg_p, fr.reg_n)
        frac_t[i] = ctx.cloud(fr.pf, fr.pf_n)
    all_scales = pair_scales(wl, params)
    scales = [all_scales[k] for k in keep]
    dev_pairs = []
    n_src = np.zeros((len(keep), 2), np.int64)
    for j, k in enumerate(keep):
        p = wl.pairs[k]
        b = wl.fragments[p.b]
        dev_pairs.append(ctx.pair(surfaces[p.a], surfaces[p.b], reg_t[p.a], frac_t[p.a], b.reg_p,
                                  b.pf, all_scales[k]))
        n_src[j] = (len(b.reg_p), len(b.pf))
    pair, start, inits = item_arrays(wl)
    if pairs is None:
        sel = np.arange(len(pair))
        local = pair
    else:
        where = np.full(len(wl.pairs), -1, np.int64)
        where[keep] = np.arange(len(keep))
        sel = np.flatnonzero(where[pair] >= 0)
        local = where[pair[sel]].astype(np.uint32)
    items = work_item_array(local, start[sel], inits[sel])
    order = lambda d: [d[i] for i in used]
    return DeviceCollection(ctx, order(meshes), order(fractures), order(surfaces), order(reg_t),
                            order(frac_t), dev_pairs, scales, items, n_src, keep, sel)


def pair_n_src(wl) -> np.ndarray:
    """(n_pairs, 2): |pc_reg of B|, |pc_frac of B| of every pair of the workload."""
    return np.array([(len(wl.fragments[p.b].reg_p), len(wl.fragments[p.b].pf)) for p in wl.pairs],
                    np.int64).reshape(-1, 2)


def stage_bytes(wl, cands, n_src=None):
    """Compulsory bytes of each stage of the batched path over the units in `cands` (their pair
    field indexing wl.pairs, and n_src by default that of every workload pair):
    ladder: 48 B per ICP point-iteration (16 B source point, 32 B matched target point and
    normal) over the passes each rung ran (iterations + 1); verify: 24 B per query of
    |Pf_A| + |Pf_B| + |brk_A| + |Pm_B|; pen_inside: 24 B per surface sample |S_A| + |S_B|;
    pen_min: 24 B per surface sample of the items whose two sides had nothing inside
    (pen_depth <= 0; a lower bound of the points that pass scans)."""
    if n_src is None:
        n_src = pair_n_src(wl)
    pair = cands["pair"].astype(np.int64)
    passes = cands["rungs"]["iterations"].astype(np.int64) + 1
    src = np.stack([n_src[pair, 0], n_src[pair, 0], n_src[pair, 1], n_src[pair, 1]], axis=1)
    fr = wl.fragments
    ver = np.array([len(fr[p.a].pf) + len(fr[p.b].pf) + len(fr[p.a].brk_p) + len(fr[p.b].margin_p)
                    for p in wl.pairs], np.float64)
    surf = np.array([len(fr[p.a].s) + len(fr[p.b].s) for p in wl.pairs], np.float64)
    none_inside = cands["scores"]["pen_depth"] <= 0.0
    return {"ladder": float(np.sum(passes * src) * 48), "verify": float(np.sum(ver[pair]) * 24),
            "pen_inside": float(np.sum(surf[pair]) * 24),
            "pen_min": float(np.sum(surf[pair][none_inside]) * 24), "finalize": 0.0}


def algorithmic_bytes(wl, cands, n_src):
    """Compulsory bytes of the verification units in `cands` (structured Candidate array):
    ICP: 48 B per point-iteration (16 B source point, 32 B matched target point + normal) over
    the passes each rung actually ran (iterations + 1); verification: 24 B per query of
    |Pf_A| + |Pf_B| + |S_A| + |S_B| + |brk_A| + |Pm_B|. Returns (icp bytes, verify bytes)."""
    pair = cands["pair"].astype(np.int64)
    passes = cands["rungs"]["iterations"].astype(np.int64) + 1  # (n, 4)
    src = np.stack([n_src[pair, 0], n_src[pair, 0], n_src[pair, 1], n_src[pair, 1]], axis=1)
    icp = float(np.sum(passes * src) * 48)
    per_pair = np.array([
        len(wl.fragments[p.a].pf) + len(wl.fragments[p.b].pf) + len(wl.fragments[p.a].s) +
        len(wl.fragments[p.b].s) + len(wl.fragments[p.a].brk_p) + len(wl.fragments[p.b].margin_p)
        for p in wl.pairs], np.float64)
    ver = float(np.sum(per_pair[pair]) * 24)
    return icp, ver


def perturbed_group_poses(wl, n_poses, seed=0, rot_deg=0.5, trans_t=0.2):
    """The assembled world poses of a workload's fragments (fragment frame -> world, the
    inverse of each Fragment.pose) and n_poses seeded perturbations of all of them: each
    fragment turned by rot_deg about a uniform axis through its fracture centroid and moved by
    trans_t * t in a uniform direction. Returns (truth (G, 4, 4), poses (P, G, 4, 4))."""
    rng = np.random.default_rng(seed)
    truth = np.stack([np.linalg.inv(fr.pose) for fr in wl.fragments])
    g = len(truth)
    out = np.empty((n_poses, g, 4, 4))
    for k, fr in enumerate(wl.fragments):
        c = truth[k, :3, :3] @ fr.pf.mean(0) + truth[k, :3, 3]
        axis = rng.normal(size=(n_poses, 3))
        axis /= np.linalg.norm(axis, axis=1, keepdims=True)
        ang = np.radians(rot_deg)
        kx = np.zeros((n_poses, 3, 3))
        kx[:, 0, 1], kx[:, 0, 2], kx[:, 1, 2] = -axis[:, 2], axis[:, 1], -axis[:, 0]
        kx -= kx.transpose(0, 2, 1)
        r = np.eye(3) + np.sin(ang) * kx + (1.0 - np.cos(ang)) * (kx @ kx)
        step = rng.normal(size=(n_poses, 3))
        step *= trans_t * fr.t / np.linalg.norm(step, axis=1, keepdims=True)
        d = np.tile(np.eye(4), (n_poses, 1, 1))
        d[:, :3, :3] = r
        d[:, :3, 3] = c - (r @ c) + step
        out[:, k] = d @ truth[k]
    return truth, out


def assembled_group(dev: DeviceCollection, wl, opts=None):
    """The adjacent pairs of a device collection as the edges of one assembled group."""
    from .adjoint import Group
    keep = [k for k, p in enumerate(wl.pairs) if p.adjacent]
    opts = opts or A.AdjointOptions(0.2, 0.01, 30.0)
    return Group(ctx=dev.ctx, edges=[dev.pairs[k] for k in keep],
                 a=np.array([wl.pairs[k].a for k in keep], np.int64),
                 b=np.array([wl.pairs[k].b for k in keep], np.int64),
                 n_fragments=len(wl.fragments),
                 n_source=np.array([len(wl.fragments[wl.pairs[k].b].pf) for k in keep], np.int64),
                 t=np.array([dev.scales[k].t for k in keep]), opts=opts,
                 centroid=np.stack([fr.pf.mean(0) for fr in wl.fragments]),
                 rho=np.array([np.sqrt(((fr.pf - fr.pf.mean(0)) ** 2).sum(1).mean())
                               for fr in wl.fragments]))
