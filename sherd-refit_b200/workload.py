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
    items: object          # ctypes WorkItem array
    n_src: np.ndarray      # (n_pairs, 2): |pc_reg of B|, |pc_frac of B|

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


def to_device(ctx: Context, wl, params: A.Params | None = None) -> DeviceCollection:
    meshes, fractures, surfaces, reg_t, frac_t = [], [], [], [], []
    for fr in wl.fragments:
        m = ctx.mesh(fr.v, fr.f)
        fm = m.subset(fr.frac)
        meshes.append(m)
        fractures.append(fm)
        surfaces.append(ctx.surfaces(fm, m, True, fr.frac_area, fr.pf, fr.s, fr.brk_p, fr.brk_ns,
                                     fr.margin_p, fr.margin_n))
        reg_t.append(ctx.cloud(fr.reg_p, fr.reg_n))
        frac_t.append(ctx.cloud(fr.pf, fr.pf_n))
    scales = pair_scales(wl, params)
    pairs = []
    n_src = np.zeros((len(wl.pairs), 2), np.int64)
    for k, (p, sc) in enumerate(zip(wl.pairs, scales)):
        b = wl.fragments[p.b]
        pairs.append(ctx.pair(surfaces[p.a], surfaces[p.b], reg_t[p.a], frac_t[p.a], b.reg_p, b.pf,
                              sc))
        n_src[k] = (len(b.reg_p), len(b.pf))
    items = work_item_array(*item_arrays(wl))
    return DeviceCollection(ctx, meshes, fractures, surfaces, reg_t, frac_t, pairs, scales, items,
                            n_src)


def stage_bytes(wl, cands, n_src):
    """Compulsory bytes of each stage of the batched path over the units in `cands`:
    ladder: 48 B per ICP point-iteration (16 B source point, 32 B matched target point and
    normal) over the passes each rung ran (iterations + 1); verify: 24 B per query of
    |Pf_A| + |Pf_B| + |brk_A| + |Pm_B|; pen_inside: 24 B per surface sample |S_A| + |S_B|;
    pen_min: 24 B per surface sample of the items whose two sides had nothing inside
    (pen_depth <= 0; a lower bound of the points that pass scans)."""
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
