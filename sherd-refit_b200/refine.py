"""R 9, full-resolution join refinement (crates/sherd-core/src/refine.rs), on the device.

After assembly every join the assembly used is registered once more, on the ORIGINAL meshes'
fracture vertices, and the correction is carried along each group's spanning walk: starting
from the group's first fragment, the first join in `used` order with exactly one endpoint
placed is taken next, its placed end stays fixed and the other end's pose becomes
rung2 . pose (refine.rs:282-318). Each join is two point-to-plane rungs at icp_dist(0.05) and
icp_dist(0.02), 40 iterations each, from the identity (refine.rs:334-386).

What runs where:
  * the vertex normals (Open3D's ComputeVertexNormals, refine.rs:121-151): sherd_vertex_normals,
    bit-identical to the reference's face-order loop;
  * each vertex's nearest working-mesh centroid (refine.rs:161-178): the bounded nearest
    neighbour of Cloud.nearest_below over the centroids' LBVH, which returns the unbounded
    nearest whenever it is within the radius (spatial/kdtree.rs:182-190);
  * each join's placement and two rungs: sherd_refine_join, one pose spread over every SM;
  * on the host: the walk, the selection mask and, above 150 000 candidates, the cap's draw.
"""

from __future__ import annotations

import logging
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .backend import Context, default_params, scales_for_pair

log = logging.getLogger(__name__)

MAX_POINTS = 150_000    # refine.rs:56
CAP_SEED = 0            # refine.rs:64
SELECT_T = 0.15         # refine.rs:66
SELECT_RES = 1.5        # refine.rs:68
RUNGS = (0.05, 0.02)    # refine.rs:70
ITERATIONS = 40         # refine.rs:72
_MISS = 0xFFFFFFFF


@dataclass
class FractureCloud:
    """refine::FractureCloud (refine.rs:78-113). `idx` indexes the original mesh's vertices in the
    order the ICP reads them; points and normals are those vertices'."""
    idx: np.ndarray
    points: np.ndarray
    normals: np.ndarray

    def __len__(self) -> int:
        return len(self.points)


@dataclass
class RefinePiece:
    """refine::RefinePiece (refine.rs:236-244): R 3.2's thickness, R 3.3's res and the cloud
    (None when the fragment has none)."""
    thick: float
    res: float
    cloud: FractureCloud | None


@dataclass
class RefinedJoin:
    """refine::RefinedJoin (refine.rs:247-262), the fields of the fixture's refine/joins.json."""
    fixed: int
    moving: int
    dist: list
    rungs: list
    fitness: float
    rmse_t: float
    registrations: list = field(default_factory=list, repr=False)


@dataclass
class Refinement:
    """refine::Refinement (refine.rs:265-271)."""
    poses: list
    joins: list


def vertex_normals(ctx: Context, v, f) -> np.ndarray:
    """refine::vertex_normals (refine.rs:121-151) on the device."""
    return ctx.vertex_normals(v, f)


def select_candidates(ctx: Context, v, centroids, fracture, thick, res) -> np.ndarray:
    """refine::select_candidates (refine.rs:161-178): the vertices whose nearest working-mesh
    centroid is a fracture face and lies strictly closer than max(0.15 t, 1.5 res), ascending."""
    v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
    centroids = np.ascontiguousarray(centroids, np.float64).reshape(-1, 3)
    fracture = np.asarray(fracture).astype(bool).reshape(-1)
    if len(centroids) != len(fracture):
        raise A.SherdError(A.E_INVALID, "one fracture label per centroid")
    if len(centroids) == 0 or len(v) == 0:
        return np.zeros(0, np.uint32)
    radius = max(SELECT_T * float(thick), SELECT_RES * float(res))
    j, _ = ctx.cloud(centroids).nearest_below(v, radius)
    keep = j != _MISS
    keep[keep] = fracture[j[keep]]
    return np.flatnonzero(keep).astype(np.uint32)


def cap_selection(idx, max_points: int = MAX_POINTS, seed: int = CAP_SEED) -> np.ndarray:
    """refine::cap_selection (refine.rs:186-193): above `max_points`, a draw of that many
    without replacement whose order is the ICP's summation order; under it, `idx` untouched. The
    draw is numpy's default_rng(seed).choice(idx, max_points, replace=False), the one
    refine.rs:30-37 describes (the reference draws from its own seeded stream there, so above
    the cap the two select different vertices)."""
    idx = np.asarray(idx, np.uint32)
    if len(idx) > max_points:
        idx = np.random.default_rng(seed).choice(idx, max_points, replace=False).astype(np.uint32)
    return idx


def select_vertices(ctx: Context, v, centroids, fracture, thick, res,
                    max_points: int = MAX_POINTS, seed: int = CAP_SEED) -> np.ndarray:
    """refine::select_vertices (refine.rs:196-205): the predicate, then the cap."""
    return cap_selection(select_candidates(ctx, v, centroids, fracture, thick, res), max_points,
                         seed)


def cloud_from_indices(v, normals, idx) -> FractureCloud:
    """refine::cloud_from_indices (refine.rs:208-214)."""
    idx = np.asarray(idx, np.uint32)
    take = idx.astype(np.int64)
    return FractureCloud(idx, np.ascontiguousarray(np.asarray(v, np.float64).reshape(-1, 3)[take]),
                         np.ascontiguousarray(np.asarray(normals, np.float64).reshape(-1, 3)[take]))


def fracture_cloud(ctx: Context, v, f, centroids, fracture, thick, res,
                   seed: int = CAP_SEED) -> FractureCloud:
    """refine::fracture_cloud (refine.rs:217-227): the original mesh (v, f) in, its cloud out.
    One device call (sherd_fracture_cloud) uploads the mesh once and returns only the selected
    vertices with their points and normals; the cap's draw (cap_selection) then picks among
    them on the host."""
    if len(centroids) != len(np.asarray(fracture).reshape(-1)):
        raise A.SherdError(A.E_INVALID, "one fracture label per centroid")
    radius = max(SELECT_T * float(thick), SELECT_RES * float(res))
    idx, pts, nrm = ctx.fracture_cloud(v, f, centroids, fracture, radius)
    capped = cap_selection(idx, MAX_POINTS, seed)
    if len(capped) != len(idx):
        at = np.searchsorted(idx, capped)
        idx, pts, nrm = capped, pts[at], nrm[at]
    return FractureCloud(np.asarray(idx, np.uint32), np.ascontiguousarray(pts),
                         np.ascontiguousarray(nrm))


def matmul4(a, b) -> np.ndarray:
    """A 4x4 product summed k = 0..3 left to right, with no fused multiply-add."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return ((a[:, 0:1] * b[0] + a[:, 1:2] * b[1]) + a[:, 2:3] * b[2]) + a[:, 3:4] * b[3]


def refine_one(ctx: Context, pieces, poses, fixed: int, moving: int,
               params: A.Params) -> RefinedJoin | None:
    """refine::refine_one (refine.rs:334-386): the pair's scales at min(t) and max(res), then the
    two rungs of sherd_refine_join. None when either side has no cloud."""
    target_piece, source_piece = pieces[fixed], pieces[moving]
    if target_piece.cloud is None or source_piece.cloud is None:
        return None
    sc = scales_for_pair(params, min(target_piece.thick, source_piece.thick),
                         max(target_piece.res, source_piece.res))
    dist = [k * sc.t * sc.icp for k in RUNGS]   # Scales::icp_dist (scales.rs:100-102)
    regs = ctx.refine_join(source_piece.cloud.points, target_piece.cloud.points,
                           target_piece.cloud.normals, poses[fixed], poses[moving], dist,
                           ITERATIONS)
    rungs = [np.array(r.transform[:]).reshape(4, 4) for r in regs]
    return RefinedJoin(fixed, moving, dist, rungs, regs[1].fitness, regs[1].inlier_rmse / sc.t,
                       regs)


def refine_joins(ctx: Context, pieces, poses, groups, used, params: A.Params | None = None,
                 ) -> Refinement:
    """refine::refine_joins (refine.rs:282-318) over every group, in group order. `used` is the
    assembly's joins as (a, b) fragment ids in the order it took them; a group of one is
    skipped, and so is a join one side of which has no cloud (its pose is left as it is)."""
    params = params or default_params()
    out = [np.array(p, np.float64).reshape(4, 4) for p in poses]
    joins = []
    for group in groups:
        if len(group) < 2:
            continue
        done = [group[0]]
        members = set(group)
        edges = [(a, b) for a, b in used if a in members and b in members]
        while True:
            step = next((i for i, (a, b) in enumerate(edges) if (a in done) != (b in done)), None)
            if step is None:
                break
            a, b = edges.pop(step)
            fixed, moving = (a, b) if a in done else (b, a)
            join = refine_one(ctx, pieces, out, fixed, moving, params)
            if join is not None:
                out[moving] = matmul4(join.rungs[1], out[moving])
                joins.append(join)
            else:
                log.warning("no full-resolution fracture cloud for one side of join %d-%d; "
                            "pose left as it is", fixed, moving)
            done.append(moving)
    return Refinement(out, joins)
