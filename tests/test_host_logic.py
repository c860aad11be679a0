"""Edge cases of the package's host logic (stage1.py, pair.py, refine.py, preprocess.py) over an
oracle-backed context: the early exits the reference takes (pair.rs:399-412, refine.rs:282-318,
samples.rs:391-440) come out the same here.
"""

from __future__ import annotations

import importlib

import numpy as np

from _slab import piece


def _mod(name):
    return importlib.import_module(f"sherd-refit_b200.{name}")


class _Device:
    def __init__(self, oracle):
        self.o = oracle

    def cloud(self, p, n=None):
        return self.o.Cloud(p, n)

    def face_geometry(self, v, f):
        return self.o.face_geometry(v, f)

    def breaklines(self, v, f, frac, t, macro_inner=0.15, macro_outer=0.6, brk_voxel=0.5):
        return self.o.breaklines(v, f, frac, t, macro_inner, macro_outer, brk_voxel)

    def hypotheses_coarse(self, fa, fb, ia, ib, tol, target, q, qn, delta, agree=0.7):
        d = lambda fr: {"p": fr.p, "ns": fr.ns, "f": fr.f, "dih": fr.dih}
        pa, pb, poses = self.o.hypotheses(d(fa), d(fb), ia, ib, tol)
        return pa, pb, poses, self.o.coarse_scores(target, q, qn, poses, delta, agree)

    def icp_rung(self, *a, **k):
        raise AssertionError("no rung should run")

    def coarse_scores(self, *a, **k):
        raise AssertionError("no re-score should run")

    def ladder_verify_batch(self, *a, **k):
        raise AssertionError("no stage-2 item should run")


def _frames(slab, name):
    st = _mod("stage1")
    p = piece(slab, name)
    return st.Frames(p=p["brk_P"], ns=p["brk_ns"], f=p["brk_f"], dih=p["brk_dih"], sub=p["brk_sub"])


def test_a_pair_without_hypotheses_returns_nothing(sherd, oracle, slab):
    """R 5.1's empty return: an empty subset on one side, or dihedrals that never complement."""
    st, pm = _mod("stage1"), _mod("pair")
    dev = _Device(oracle)
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    a, b = _frames(slab, "pieceA"), _frames(slab, "pieceB")
    b.sub = np.zeros(0, np.uint32)
    res = pm.match_pair(dev, None, st.PairStage1(dev, a, b, scales), sherd.default_params())
    assert res.candidates == [] and len(res.stage1.hypotheses) == 0
    assert res.stage1.starts.shape == (0, 4, 4) and res.stage1.best == 0.0
    b = _frames(slab, "pieceB")
    b.dih = np.full(len(b.dih), 10.0)      # 90 + 10 - 180 = -80: no pair within 25 deg
    a.dih = np.full(len(a.dih), 90.0)
    res = pm.match_pair(dev, None, st.PairStage1(dev, a, b, scales), sherd.default_params())
    assert res.candidates == []


def test_a_pair_whose_coarse_scores_stay_under_the_floor_keeps_nothing(sherd, oracle, slab):
    """R 5.3's floor (0.1): with a coarse radius of 1e-9 only a hypothesis's own anchor point can
    land on A's breakline, so no score reaches 1/60 < 0.1; the suppression keeps nothing and
    stage 1 refines nothing."""
    st = _mod("stage1")
    dev = _Device(oracle)
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    scales.coarse = 1e-9
    a, b = _frames(slab, "pieceA"), _frames(slab, "pieceB")
    res = st.PairStage1(dev, a, b, scales).run(seed=0)
    assert len(res.hypotheses) > 0 and np.all(res.coarse <= 1.0 / 60.0)
    assert len(res.kept) == 0 and len(res.kept2) == 0


def test_refine_walk_skips_singletons_and_joins_outside_the_group(oracle):
    """refine.rs:282-318: a group of one is skipped; a join with an endpoint outside the group is
    not walked; a join whose both ends are already placed is not walked either."""
    rf = _mod("refine")

    class Dev:
        calls = []

        def refine_join(self, source, target, target_normals, pose_fixed, pose_moving, dist,
                        max_iteration=40):
            Dev.calls.append(len(source))
            A = importlib.import_module("sherd-refit_b200._abi")
            regs = [A.Registration(), A.Registration()]
            for r in regs:
                r.transform[:] = np.eye(4).reshape(16).tolist()
            return regs

    cloud = rf.FractureCloud(np.arange(3, dtype=np.uint32), np.eye(3), np.eye(3))
    pieces = [rf.RefinePiece(1.0, 0.1, cloud) for _ in range(4)]
    out = rf.refine_joins(Dev(), pieces, [np.eye(4)] * 4, [[3], [0, 1, 2]],
                          [(0, 3), (1, 2), (0, 1), (0, 2)])
    assert [(j.fixed, j.moving) for j in out.joins] == [(0, 1), (1, 2)]
    assert len(Dev.calls) == 2


def test_samples_without_a_breakline_have_no_margin(sherd, oracle, slab):
    """samples.rs:391-440: d_brk is +inf everywhere without a breakline, so the margin is empty."""
    pre = _mod("preprocess")
    p = piece(slab, "pieceB")
    s = pre.samples(_Device(oracle), p["V"], p["F"], p["frac"], np.zeros((0, 3)), 30.0, 0)
    assert len(s.s) == 20000 and len(s.margin_idx) == 0
    md = pre.match_data(_Device(oracle), p["V"], p["F"], np.ones(len(p["F"]), bool), 30.0, 0)
    assert len(md.brk) == 0 and len(md.samples.margin_idx) == 0
    assert len(md.samples.pf) == 12000      # every face is fracture: the count hits the cap
