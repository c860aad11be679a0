"""Stage 1 of pair matching (R 5.1-5.5) on the device: hypotheses, coarse score, suppression,
the breakline ladder and its re-score, and the second suppression that yields stage 2's starts.

The chain is pair.rs:375-440's up to `suppress_stage1`, each step the reference's:
  * R 5.1 (hypotheses.rs:139-211): every complementary pair of breakline frames is a pose;
  * R 5.2 (coarse.rs:113-133): each pose's coarse score over a 60-point probe of B;
  * R 5.3 (pair.rs:183-187, nms.rs): suppression over the best 5000, at most `stage1` kept;
  * R 5.4 (pair.rs:200-238, ladder.rs:131-186): two point-to-point rungs of B's breakline subset
    against A's whole breakline (0.2 and 0.08 t.icp, 20 iterations each), then the re-score
    over B's whole subset at `scales.stage1`;
  * R 5.5 (ladder.rs:191-215): suppression of the refined poses, at most `stage2` kept.

R 5.1 and R 5.2 are one device call (sherd_hypotheses_coarse): the poses go from the frames
straight into the score without leaving HBM. The ladder and the re-score are the batched
sherd_icp_rung and sherd_coarse_scores; the two suppressions are the library's host code
(sherd_order_by_score, sherd_nms). The probe is drawn as the reference's Python pipeline draws
it, numpy.random.default_rng(seed).choice(B.brk_sub, 60, replace=False) (the fixture's
coarse.idx); the Rust reference draws from its own seeded stream there (coarse.rs:88-95).
Walk orders are descending by score with ties to the lower index (nms.rs:46-59); the
reference's Python pipeline used an unstable sort (nms.rs:26-36), so an order can be passed in
to reproduce its choices exactly.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi as A
from .backend import ALL, Context, nms, order_by_score

DIHEDRAL_TOL = 25.0        # params.rs:143
COARSE_POINTS = 60         # params.rs:145
STAGE1 = 250               # params.rs:146
STAGE2 = 10                # params.rs:147
NORMAL_AGREE = 0.7         # coarse.rs:42
COARSE_ORDER_LIMIT = 5000  # pair.rs:50
COARSE_FLOOR = 0.1         # pair.rs:52
STAGE1_RUNGS = (0.2, 0.08)  # ladder.rs:51
STAGE1_ITERATIONS = 20     # ladder.rs:53
STAGE1_FLOOR = 0.05        # ladder.rs:61


@dataclass
class Frames:
    """hypotheses::Frames (hypotheses.rs:53-82): breakline points, shell macro-normals, in-plane
    axes (f64, (n, 3)), dihedrals in degrees and R 3.5.5's subset."""
    p: np.ndarray
    ns: np.ndarray
    f: np.ndarray
    dih: np.ndarray
    sub: np.ndarray

    @property
    def tangent(self) -> np.ndarray:
        """ns x f (breakline.rs:180-182)."""
        ns, f = self.ns, self.f
        return np.stack([ns[:, 1] * f[:, 2] - ns[:, 2] * f[:, 1],
                         ns[:, 2] * f[:, 0] - ns[:, 0] * f[:, 2],
                         ns[:, 0] * f[:, 1] - ns[:, 1] * f[:, 0]], axis=1)


@dataclass
class Hypotheses:
    """hypotheses::Hypotheses (hypotheses.rs:101-136): positions into the two subsets and the
    poses (row-major 4x4: R and tau)."""
    pa: np.ndarray
    pb: np.ndarray
    poses: np.ndarray

    def __len__(self) -> int:
        return len(self.pa)


@dataclass
class Stage1Result:
    """What R 5.1-5.5 produced for one pair."""
    hypotheses: Hypotheses
    coarse: np.ndarray          # R 5.2 score per hypothesis
    kept: np.ndarray            # R 5.3: hypotheses refined, in keeping order
    transforms: np.ndarray      # R 5.4: the refined pose of each kept hypothesis
    scores: np.ndarray          # R 5.4: its re-score
    kept2: np.ndarray           # R 5.5: positions into `kept`, in keeping order

    @property
    def starts(self) -> np.ndarray:
        """Stage 2's inits, transforms[kept2]."""
        return self.transforms[self.kept2]

    @property
    def best(self) -> float:
        """The pair's best stage-1 score (brk_best), or 0 with nothing refined."""
        return float(self.scores.max()) if len(self.scores) else 0.0


def probe_draw(pool, points: int = COARSE_POINTS, seed: int = 0) -> np.ndarray:
    """R 5.2's probe: min(points, |pool|) distinct entries of B's subset, in draw order."""
    pool = np.asarray(pool)
    return np.random.default_rng(seed).choice(pool, min(points, len(pool)), replace=False)


class PairStage1:
    """One pair's stage 1 on the device: A's whole breakline as one device cloud (the coarse
    target and the ladder's target, kd_brk / pc_brk_full) and B's subset (pc_brk)."""

    def __init__(self, ctx: Context, a: Frames, b: Frames, scales: A.Scales):
        self.ctx, self.a, self.b, self.scales = ctx, a, b, scales
        self.target = ctx.cloud(a.p, a.ns) if len(a.p) else None
        sub = np.asarray(b.sub, np.int64)
        self.brk_points = np.ascontiguousarray(b.p[sub])
        self.brk_normals = np.ascontiguousarray(b.ns[sub])

    def hypotheses_coarse(self, probe_idx, dihedral_tol: float = DIHEDRAL_TOL):
        """R 5.1 over the two subsets and R 5.2 with the probe B.p[probe_idx]."""
        if self.target is None or not len(self.a.sub) or not len(self.b.sub):
            return Hypotheses(np.zeros(0, np.uint32), np.zeros(0, np.uint32),
                              np.zeros((0, 4, 4))), np.zeros(0)
        idx = np.asarray(probe_idx, np.int64)
        pa, pb, poses, cs = self.ctx.hypotheses_coarse(
            self.a, self.b, self.a.sub, self.b.sub, dihedral_tol, self.target, self.b.p[idx],
            self.b.ns[idx], self.scales.coarse, NORMAL_AGREE)
        return Hypotheses(pa, pb, poses), cs

    def suppress(self, hyp: Hypotheses, cs, stage1: int = STAGE1, order=None) -> np.ndarray:
        """R 5.3 (pair.rs:183-187): NMS over the best COARSE_ORDER_LIMIT, floor 0.1."""
        if order is None:
            order = order_by_score(cs, COARSE_ORDER_LIMIT)
        return nms(order, hyp.poses, cs, self.scales.nms, stage1, COARSE_FLOOR)

    def stage1(self, hyp: Hypotheses, kept):
        """R 5.4 (pair.rs:200-238): the two point-to-point rungs from each kept hypothesis, then
        the re-score at scales.stage1 over B's whole subset. Returns (transforms, scores)."""
        kept = np.asarray(kept, np.int64)
        if self.target is None or not len(kept):
            return np.zeros((0, 4, 4)), np.zeros(0)
        poses = hyp.poses[kept]
        for k in STAGE1_RUNGS:
            regs = self.ctx.icp_rung_array(self.brk_points, self.target, poses,
                                           k * self.scales.t * self.scales.icp, STAGE1_ITERATIONS,
                                           estimation=A.POINT_TO_POINT)
            poses = np.ascontiguousarray(regs["transform"]).reshape(-1, 4, 4)
        scores = self.ctx.coarse_scores(self.target, self.brk_points, self.brk_normals, poses,
                                        self.scales.stage1, NORMAL_AGREE)
        return poses, np.asarray(scores, np.float64)

    def suppress_stage1(self, transforms, scores, stage2: int = STAGE2,
                        order=None) -> np.ndarray:
        """R 5.5 (ladder.rs:191-215): NMS over every refined pose, floor 0.05."""
        if order is None:
            order = order_by_score(scores, ALL)
        return nms(order, transforms, scores, self.scales.nms, stage2, STAGE1_FLOOR)

    def run(self, seed: int = 0, stage1: int = STAGE1, stage2: int = STAGE2,
            probe_idx=None, order1=None, order2=None) -> Stage1Result:
        """The chain R 5.1-5.5 (pair.rs:399-425 up to the second suppression)."""
        if probe_idx is None:
            probe_idx = probe_draw(self.b.sub, COARSE_POINTS, seed)
        hyp, cs = self.hypotheses_coarse(probe_idx)
        if not len(hyp):
            return Stage1Result(hyp, cs, np.zeros(0, np.uint32), np.zeros((0, 4, 4)),
                                np.zeros(0), np.zeros(0, np.uint32))
        kept = self.suppress(hyp, cs, stage1, order1)
        transforms, scores = self.stage1(hyp, kept)
        kept2 = (self.suppress_stage1(transforms, scores, stage2, order2) if len(scores)
                 else np.zeros(0, np.uint32))
        return Stage1Result(hyp, cs, kept, transforms, scores, kept2)
