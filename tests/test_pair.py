"""R 5's whole pair chain (pair.rs:375-440, `match_pair`): stage 1, the batched stage-2 ladder and
verification, R 5.7's ranking and cut, against the slab fixture's `result.candidates.json`.

With the fixture's own walk orders the chain must return the fixture's five candidates in its
order (sherd-parity/src/stages/candidates.rs:1-20's injected row: the ranking, the count, each
verdict and brk_best), each pose within stage 2's 0.05 deg / 0.01 t. On the CPU the package's host
code runs over an oracle-backed context (every device call answered by the oracle); on the GPU it
runs on the device.
"""

from __future__ import annotations

import ctypes as C
import importlib

import numpy as np
import pytest

from _slab import oracle_pair, origin_t, piece, slab_params, trace_deg

ROT_DEG, TRANS_T, SCORE = 0.05, 0.01, 0.02


def _frames(st, slab, name):
    p = piece(slab, name)
    return st.Frames(p=p["brk_P"], ns=p["brk_ns"], f=p["brk_f"], dih=p["brk_dih"], sub=p["brk_sub"])


def _params(sherd, slab):
    p = sherd.default_params()
    for k, v in zip(("min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n"), slab["params"]):
        setattr(p, k, float(v))
    return p


class _OracleDevice:
    """The Context calls pair.py and stage1.py make, answered by the oracle."""

    def __init__(self, oracle):
        self.o = oracle
        self.A = importlib.import_module("sherd-refit_b200._abi")

    def cloud(self, p, n=None):
        return self.o.Cloud(p, n)

    def hypotheses_coarse(self, fa, fb, ia, ib, tol, target, q, qn, delta, agree=0.7):
        d = lambda f: {"p": f.p, "ns": f.ns, "f": f.f, "dih": f.dih}
        pa, pb, poses = self.o.hypotheses(d(fa), d(fb), ia, ib, tol)
        return pa, pb, poses, self.o.coarse_scores(target, q, qn, poses, delta, agree)

    def icp_rung(self, source, target, inits, distance, max_iteration=30, estimation=1):
        regs = self.o.icp_rung(source, target, inits, distance, max_iteration,
                               point_to_point=estimation == self.A.POINT_TO_POINT)
        return [self.A.Registration.from_buffer_copy(r) for r in regs]

    def icp_rung_array(self, *a, **k):
        regs = self.icp_rung(*a, **k)
        rec = importlib.import_module("sherd-refit_b200.backend").REGISTRATION
        return np.frombuffer(b"".join(bytes(r) for r in regs), rec)

    def coarse_scores(self, target, points, normals, poses, radius, normal_agree=0.7):
        return self.o.coarse_scores(target, points, normals, poses, radius, normal_agree)

    def ladder_verify_batch(self, pairs, items, params, sched=0):
        w = [self.o.WorkItem(p, s, (C.c_double * 16)(*np.ravel(t))) for p, s, t in items]
        out, _ = self.o.ladder_verify_batch(pairs, w, self.o.Params.from_buffer_copy(params))
        return [self.A.Candidate.from_buffer_copy(c) for c in out]


def _check_against_fixture(res, slab):
    t = float(slab["scales"][0])
    assert len(res.candidates) == len(slab["result_T"]) == 5
    for k, c in enumerate(res.candidates):
        mine = np.array(c.rungs[3].transform[:]).reshape(4, 4)
        theirs = slab["result_T"][k]
        assert trace_deg(mine, theirs) <= ROT_DEG and origin_t(mine, theirs, t) <= TRANS_T, k
        assert bool(c.accepted) == bool(slab["result_accepted"][k]), k
        assert abs(c.scores.brk - slab["result_brk"][k, 0]) <= SCORE
        assert abs(c.scores.brk_best - slab["result_brk"][k, 1]) <= SCORE
        assert abs(c.scores.seam - slab["result_seam_tight"][k, 0]) <= 0.34     # verify.rs row
        assert abs(c.scores.tight - slab["result_seam_tight"][k, 1]) <= 0.01
    # R 5.7's order: seam * tight descending.
    s = [c.scores.seam * c.scores.tight for c in res.candidates]
    assert all(x >= y for x, y in zip(s, s[1:]))


def test_match_pair_on_the_oracle_reproduces_the_fixture(sherd, oracle, slab):
    st = importlib.import_module("sherd-refit_b200.stage1")
    pair_mod = importlib.import_module("sherd-refit_b200.pair")
    dev = _OracleDevice(oracle)
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    stage1 = st.PairStage1(dev, _frames(st, slab, "pieceA"), _frames(st, slab, "pieceB"), scales)
    op = oracle_pair(oracle, slab)
    res = pair_mod.match_pair(dev, op["pair"], stage1, _params(sherd, slab), seed=0,
                              order1=slab["nms1_order"], order2=slab["nms2_order"])
    _check_against_fixture(res, slab)


def test_a_pair_under_the_stage1_floor_returns_its_best_pose_partial(sherd, oracle, slab):
    st = importlib.import_module("sherd-refit_b200.stage1")
    pair_mod = importlib.import_module("sherd-refit_b200.pair")
    dev = _OracleDevice(oracle)
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    stage1 = st.PairStage1(dev, _frames(st, slab, "pieceA"), _frames(st, slab, "pieceB"), scales)
    res = pair_mod.match_pair(dev, None, stage1, _params(sherd, slab), seed=0, stage1_floor=0.5,
                              order1=slab["nms1_order"])
    (c,) = res.candidates
    assert c.scores.partial == 1 and c.accepted == 0
    assert c.scores.brk == c.scores.brk_best == res.stage1.best
    k = int(np.argmax(res.stage1.scores))
    assert np.array_equal(np.array(c.rungs[3].transform[:]).reshape(4, 4), res.stage1.transforms[k])
    assert c.scores.gap_limit == scales.gap / scales.t


@pytest.mark.gpu
def test_match_pair_on_the_device_reproduces_the_fixture(sherd, gpu_ctx, gpu_slab, slab):
    st = importlib.import_module("sherd-refit_b200.stage1")
    pair_mod = importlib.import_module("sherd-refit_b200.pair")
    stage1 = st.PairStage1(gpu_ctx, _frames(st, slab, "pieceA"), _frames(st, slab, "pieceB"),
                           gpu_slab["scales"])
    res = pair_mod.match_pair(gpu_ctx, gpu_slab["pair"], stage1, _params(sherd, slab), seed=0,
                              order1=slab["nms1_order"], order2=slab["nms2_order"])
    _check_against_fixture(res, slab)
    # On its own walk orders: the fixture's accepted join is still the best candidate.
    own = pair_mod.match_pair(gpu_ctx, gpu_slab["pair"], stage1, _params(sherd, slab), seed=0)
    best = np.array(own.candidates[0].rungs[3].transform[:]).reshape(4, 4)
    assert own.candidates[0].accepted == 1
    assert trace_deg(best, slab["result_T"][0]) <= 0.2


class _OracleCollectionDevice(_OracleDevice):
    """_OracleDevice plus the object constructors match_collection uses, on the oracle."""

    def face_geometry(self, v, f):
        return self.o.face_geometry(v, f)

    def breaklines(self, v, f, frac, t, macro_inner=0.15, macro_outer=0.6, brk_voxel=0.5):
        return self.o.breaklines(v, f, frac, t, macro_inner, macro_outer, brk_voxel)

    def mesh(self, v, f):
        return self.o.Mesh(v, f)

    def surfaces(self, fracture, mesh, watertight, frac_area, pf, s, brk_p, brk_ns, margin_p,
                 margin_n):
        return self.o.Surfaces(fracture, mesh, watertight, frac_area, pf, s, brk_p, brk_ns,
                               margin_p, margin_n)

    def pair(self, a, b, reg_t, frac_t, reg_p, frac_p, scales):
        return self.o.Pair(a, b, reg_t, frac_t, reg_p, frac_p,
                           self.o.Scales.from_buffer_copy(scales))


def test_match_collection_is_match_pair_per_pair(sherd, oracle, slab):
    """The collection form (one batched stage 2 over every pair's starts) gives each pair what
    match_pair gives it, and on the slab the fixture's accepted join first."""
    pm = importlib.import_module("sherd-refit_b200.pair")
    pre = importlib.import_module("sherd-refit_b200.preprocess")
    st = importlib.import_module("sherd-refit_b200.stage1")
    dev = _OracleCollectionDevice(oracle)
    params = _params(sherd, slab)
    frags = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        frags.append(pm.FragmentInput(p["V"], p["F"], p["frac"], float(p["thick_t"]),
                                      float(p["res"]), bool(p["watertight"])))
    timings = {}
    (res,) = pm.match_collection(dev, frags, [(0, 1)], params, timings=timings)
    assert set(timings) == {"preprocess", "stage1", "stage2", "rank"}
    sc = sherd.scales_for_pair(params, min(f.t for f in frags), max(f.res for f in frags))
    assert np.array_equal(np.array([getattr(sc, k) for k, _ in sc._fields_]), slab["scales"])
    mds = [pre.match_data(dev, f.v, f.f, f.frac, sc.t, 0) for f in frags]
    surf = []
    for f, md in zip(frags, mds):
        mesh = oracle.Mesh(f.v, f.f)
        fm = mesh.subset(f.frac)
        surf.append((mesh, fm, oracle.Surfaces(fm, mesh, int(f.watertight), md.frac_area,
                                               md.samples.pf, md.samples.s, md.brk.p, md.brk.ns,
                                               md.margin_p, md.margin_n)))
    a, b = mds
    pair = oracle.Pair(surf[0][2], surf[1][2], oracle.Cloud(a.reg_p, a.reg_n),
                       oracle.Cloud(a.samples.pf, a.pf_n), b.reg_p, b.samples.pf,
                       oracle.Scales.from_buffer_copy(sc))
    want = pm.match_pair(dev, pair, st.PairStage1(dev, a.frames, b.frames, sc), params)
    assert len(res.candidates) == len(want.candidates) == 5
    for g, w in zip(res.candidates, want.candidates):
        assert bytes(g.rungs) == bytes(w.rungs) and g.accepted == w.accepted
        assert g.scores.brk == w.scores.brk and g.scores.brk_best == w.scores.brk_best
    best = np.array(res.candidates[0].rungs[3].transform[:]).reshape(4, 4)
    assert res.candidates[0].accepted == 1 and trace_deg(best, slab["result_T"][0]) <= 0.05


def test_match_collection_under_the_stage1_floor(sherd, oracle, slab):
    """match_collection's stage1_floor branch is match_pair's: the best stage-1 pose alone,
    partial and refused, and no stage-2 item."""
    pm = importlib.import_module("sherd-refit_b200.pair")

    class NoStage2(_OracleCollectionDevice):
        def ladder_verify_batch(self, *a, **k):
            raise AssertionError("no stage-2 item should run under the floor")

    frags = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        frags.append(pm.FragmentInput(p["V"], p["F"], p["frac"], float(p["thick_t"]),
                                      float(p["res"]), bool(p["watertight"])))
    (res,) = pm.match_collection(NoStage2(oracle), frags, [(0, 1)], _params(sherd, slab),
                                 stage1_floor=0.9)
    (c,) = res.candidates
    assert c.scores.partial == 1 and c.accepted == 0 and c.scores.brk == res.stage1.best
