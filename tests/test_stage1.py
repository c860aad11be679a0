"""Stage 1 of pair matching (R 5.1-5.5): hypotheses, coarse score, suppression, the breakline
ladder with its re-score, and the second suppression, pinned to the slab fixture.

The fixture's pair carries every boundary of the chain: the subsets and kept frame pairs
(hyp.ia/ib/pa/pb), the probe (coarse.idx) and all 16 337 coarse scores (coarse.cs), both
suppressions' walk orders and kept lists (nms1.*, nms2.*), the refined poses (s1.T) and their
re-scores (s1.score). The oracle reproduces each exactly, the ladder within
sherd-parity/src/stages/stage1.rs:55-63's injected rows (0.05 deg, 0.01 t, score 0.02). The
library's host suppression is checked here on the CPU; the device half on the GPU: hypotheses,
poses and scores bit-identical, the chain within the same rows.
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest

from _slab import origin_t, piece, trace_deg

ROT_DEG, TRANS_T, SCORE = 0.05, 0.01, 0.02   # stage1.rs:55-59 (injected)


def _stage1():
    return importlib.import_module("sherd-refit_b200.stage1")


def _frames(slab, name):
    p = piece(slab, name)
    return {"p": p["brk_P"], "ns": p["brk_ns"], "f": p["brk_f"], "dih": p["brk_dih"],
            "sub": p["brk_sub"]}


def _scales(oracle, slab):
    return oracle.scales_from(slab["scales"])


@pytest.fixture(scope="module")
def hyp(oracle, slab):
    a, b = _frames(slab, "pieceA"), _frames(slab, "pieceB")
    return oracle.hypotheses(a, b, a["sub"], b["sub"])


# ---- the oracle, pinned ---------------------------------------------------------------------


def test_hypotheses_are_the_fixtures(oracle, slab, hyp):
    a, b = _frames(slab, "pieceA"), _frames(slab, "pieceB")
    assert np.array_equal(slab["hyp_ia"], a["sub"]) and np.array_equal(slab["hyp_ib"], b["sub"])
    pa, pb, poses = hyp
    assert np.array_equal(pa, slab["hyp_pa"]) and np.array_equal(pb, slab["hyp_pb"])
    r = poses[:, :3, :3]
    assert np.abs(np.einsum("nij,nkj->nik", r, r) - np.eye(3)).max() < 1e-12


def test_a_matching_frame_pair_is_the_identity(oracle):
    """hypotheses.rs:225-260: two halves of a wall broken along y, shells up, A's fracture facing
    +x (its outward in-plane axis -x) and B's facing -x: one hypothesis, the identity."""
    a = {"p": np.zeros((1, 3)), "ns": np.array([[0.0, 0, 1]]), "f": np.array([[-1.0, 0, 0]]),
         "dih": np.array([90.0])}
    b = {"p": np.zeros((1, 3)), "ns": np.array([[0.0, 0, 1]]), "f": np.array([[1.0, 0, 0]]),
         "dih": np.array([90.0])}
    pa, pb, poses = oracle.hypotheses(a, b, [0], [0])
    assert list(pa) == [0] and list(pb) == [0]
    assert np.array_equal(poses[0], np.eye(4))
    b["dih"] = np.array([120.0])          # |90 + 120 - 180| = 30 >= 25: no hypothesis
    assert len(oracle.hypotheses(a, b, [0], [0])[0]) == 0


def test_probe_draw_is_the_fixture_probe(slab):
    b = _frames(slab, "pieceB")
    assert np.array_equal(_stage1().probe_draw(b["sub"], 60, 0), slab["coarse_idx"])


def test_oracle_coarse_scores_are_the_fixtures(oracle, slab, hyp):
    a, b = _frames(slab, "pieceA"), _frames(slab, "pieceB")
    idx = slab["coarse_idx"].astype(np.int64)
    cs = oracle.coarse_scores(oracle.Cloud(a["p"], a["ns"]), b["p"][idx], b["ns"][idx], hyp[2],
                              _scales(oracle, slab).coarse)
    assert np.array_equal(cs, slab["coarse_cs"])


def test_oracle_suppressions_are_the_fixtures(oracle, slab, hyp):
    sc = _scales(oracle, slab)
    kept = oracle.nms(slab["nms1_order"], hyp[2], slab["coarse_cs"], sc.nms, 250,
                      oracle.COARSE_FLOOR)
    assert np.array_equal(kept, slab["nms1_kept"])
    kept2 = oracle.nms(slab["nms2_order"], slab["s1_T"], slab["s1_score"], sc.nms, 10,
                       oracle.STAGE1_FLOOR)
    assert np.array_equal(kept2, slab["nms2_kept"])


def test_oracle_ladder_and_rescore_reach_the_fixture(oracle, slab, hyp):
    """From the kept hypotheses' own poses: both point-to-point rungs within the injected rows of
    s1.T, and the re-score at scales.stage1 equal to s1.score."""
    sc = _scales(oracle, slab)
    a, b = _frames(slab, "pieceA"), _frames(slab, "pieceB")
    sub = b["sub"].astype(np.int64)
    target = oracle.Cloud(a["p"], a["ns"])
    poses = oracle.stage1_ladder(b["p"][sub], target, hyp[2][slab["nms1_kept"].astype(np.int64)],
                                 sc)
    for mine, theirs in zip(poses, slab["s1_T"]):
        assert trace_deg(mine, theirs) <= ROT_DEG and origin_t(mine, theirs, sc.t) <= TRANS_T
    rescore = oracle.coarse_scores(target, b["p"][sub], b["ns"][sub], poses, sc.stage1)
    assert np.abs(rescore - slab["s1_score"]).max() <= SCORE
    assert np.mean(rescore == slab["s1_score"]) >= 0.99


# ---- the library's host suppression (no device) -------------------------------------------------


def test_order_by_score_ties_go_to_the_lower_index(sherd, oracle):
    """nms.rs:125-132's case, and the oracle's order on the fixture's coarse scores."""
    be = importlib.import_module("sherd-refit_b200.backend")
    s = [0.1, 0.5, 0.5, 0.2, 0.5]
    assert list(be.order_by_score(s)) == [1, 2, 4, 3, 0]
    assert list(be.order_by_score(s, 3)) == [1, 2, 4]
    assert len(be.order_by_score([], 10)) == 0
    assert list(be.order_by_score([0.0, -0.0, np.nan, 1.0])) == [2, 3, 0, 1]   # total order


def test_library_nms_is_the_fixtures_and_the_oracles(sherd, oracle, slab, hyp):
    be = importlib.import_module("sherd-refit_b200.backend")
    sc = _scales(oracle, slab)
    cs = slab["coarse_cs"]
    kept = be.nms(slab["nms1_order"], hyp[2], cs, sc.nms, 250, 0.1)
    assert np.array_equal(kept, slab["nms1_kept"])
    own = be.order_by_score(cs, 5000)
    assert np.array_equal(own, oracle.order_by_score(cs, 5000))
    assert np.array_equal(be.nms(own, hyp[2], cs, sc.nms, 250, 0.1),
                          oracle.nms(own, hyp[2], cs, sc.nms, 250, 0.1))
    kept2 = be.nms(slab["nms2_order"], slab["s1_T"], slab["s1_score"], sc.nms, 10, 0.05)
    assert np.array_equal(kept2, slab["nms2_kept"])


def test_nms_rules(sherd):
    """A cluster collapses to its best; a pose far enough away, or turned by more than about
    18.2 deg (trace <= 2.9), survives; the walk breaks at the floor; topk = 0 keeps one."""
    be = importlib.import_module("sherd-refit_b200.backend")

    def pose(deg, x):
        a = np.radians(deg)
        t = np.eye(4)
        t[:2, :2] = [[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]]
        t[0, 3] = x
        return t

    poses = np.stack([pose(0, 0), pose(5, 0.1), pose(0, 3.0), pose(20, 0.0), pose(0, 0.2)])
    score = np.array([0.9, 0.8, 0.7, 0.6, 0.05])
    order = be.order_by_score(score)
    assert list(be.nms(order, poses, score, 1.0, 10, 0.1)) == [0, 2, 3]
    assert list(be.nms(order, poses, score, 1.0, 2, 0.1)) == [0, 2]
    assert list(be.nms(order, poses, score, 1.0, 0, 0.1)) == [0]
    assert list(be.nms(order, poses, score, 1.0, 10, 0.75)) == [0]
    assert len(be.nms([], poses, score, 1.0, 10, 0.1)) == 0
    with pytest.raises(sherd.SherdError):
        be.nms([7], poses, score, 1.0, 10, 0.1)


# ---- on the device ---------------------------------------------------------------------------------


def _pair(sherd, gpu_ctx, oracle, slab):
    st = _stage1()
    fa, fb = (st.Frames(**_frames(slab, n)) for n in ("pieceA", "pieceB"))
    return st.PairStage1(gpu_ctx, fa, fb, sherd.Scales(*[float(x) for x in slab["scales"]]))


@pytest.mark.gpu
def test_device_hypotheses_and_scores_are_bit_identical(sherd, gpu_ctx, oracle, slab, hyp):
    pair = _pair(sherd, gpu_ctx, oracle, slab)
    h, cs = pair.hypotheses_coarse(slab["coarse_idx"])
    assert np.array_equal(h.pa, slab["hyp_pa"]) and np.array_equal(h.pb, slab["hyp_pb"])
    assert np.array_equal(h.poses, hyp[2])
    assert np.array_equal(cs, slab["coarse_cs"])


@pytest.mark.gpu
def test_device_chain_reproduces_the_fixture(sherd, gpu_ctx, oracle, slab):
    """With the fixture's walk orders (its Python pipeline's unstable sort): the same kept
    hypotheses, refined poses within the injected rows, the same second suppression and so the
    fixture's stage-2 starts."""
    pair = _pair(sherd, gpu_ctx, oracle, slab)
    t = float(slab["scales"][0])
    res = pair.run(seed=0, order1=slab["nms1_order"], order2=slab["nms2_order"])
    assert np.array_equal(res.kept, slab["nms1_kept"])
    for mine, theirs in zip(res.transforms, slab["s1_T"]):
        assert trace_deg(mine, theirs) <= ROT_DEG and origin_t(mine, theirs, t) <= TRANS_T
    assert np.abs(res.scores - slab["s1_score"]).max() <= SCORE
    assert np.array_equal(res.kept2, slab["nms2_kept"])
    for mine, theirs in zip(res.starts, slab["starts"]):
        assert trace_deg(mine, theirs) <= ROT_DEG and origin_t(mine, theirs, t) <= TRANS_T


@pytest.mark.gpu
def test_device_chain_on_its_own_orders(sherd, gpu_ctx, oracle, slab):
    """With its own stable orders: most of the fixture's kept hypotheses, and a start at the
    fixture's accepted pose among the ten."""
    pair = _pair(sherd, gpu_ctx, oracle, slab)
    t = float(slab["scales"][0])
    res = pair.run(seed=0)
    assert len(np.intersect1d(res.kept, slab["nms1_kept"])) >= 150
    accepted = slab["starts"][int(np.argmax(slab["s2_accepted"]))]
    assert min(trace_deg(s, accepted) + origin_t(s, accepted, t) for s in res.starts) < 0.05
    assert res.best == pytest.approx(float(slab["s1_score"].max()), abs=SCORE)


@pytest.mark.gpu
def test_device_hypotheses_edge_cases(sherd, gpu_ctx, slab):
    import ctypes as C
    A = importlib.import_module("sherd-refit_b200._abi")
    be = importlib.import_module("sherd-refit_b200.backend")
    st = _stage1()
    fa, fb = (st.Frames(**_frames(slab, n)) for n in ("pieceA", "pieceB"))
    target = gpu_ctx.cloud(fa.p, fa.ns)
    # Empty subsets: no hypothesis.
    pa, pb, poses, cs = gpu_ctx.hypotheses_coarse(fa, fb, [], fb.sub, 25.0, target,
                                                  fb.p[:3], fb.ns[:3], 1.0)
    assert len(pa) == 0 and poses.shape == (0, 4, 4)
    # A capacity below the count is refused, with the count reported.
    sa, sb = be._frames(fa), be._frames(fb)
    count = C.c_uint32(0)
    ia, ib = np.ascontiguousarray(fa.sub, np.uint32), np.ascontiguousarray(fb.sub, np.uint32)
    q, qn = np.ascontiguousarray(fb.p[:3]), np.ascontiguousarray(fb.ns[:3])
    out_pa, out_pb = np.empty(1, np.uint32), np.empty(1, np.uint32)
    out_poses, out_scores = np.empty(16), np.empty(1)
    rc = A.lib().sherd_hypotheses_coarse(
        gpu_ctx.h, C.byref(sa[0]), C.byref(sb[0]), ia, len(ia), ib, len(ib), 25.0, target.h,
        q, qn, 3, 1.0, 0.7, 1, out_pa.ctypes.data, out_pb.ctypes.data, out_poses.ctypes.data,
        out_scores.ctypes.data, C.byref(count))
    assert rc == A.E_INVALID and count.value == len(slab["hyp_pa"])
    # An index beyond the frames is refused.
    with pytest.raises(sherd.SherdError):
        gpu_ctx.hypotheses_coarse(fa, fb, [len(fa.p)], fb.sub, 25.0, target, fb.p[:3],
                                  fb.ns[:3], 1.0)
