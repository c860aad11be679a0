"""The oracle pinned against the reference's own golden vectors (the slab fixture).

Rows follow the reference's parity harness (crates/sherd-parity/src/stages/*.rs):
thickness bit-exact from injected hits, first hits and cone votes statistically against the
Embree answers the fixture carries, the stage-2 ladder within D 10.2's pose rows and the
verification within its score rows with identical verdicts.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from _slab import (CHAOTIC_SHARE, ROT_DEG, TRANS_T, VERIFY_TOL, origin_t, oracle_pair, piece,
                   reference_scores, score_dict, slab_params, trace_deg)


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_thickness_from_the_fixture_hits_is_bit_exact(slab, oracle, name):
    """thickness.rs:139-162 fed thick.idx/t_hit/prim reproduces thick.t and thick_mode."""
    p = piece(slab, name)
    normals, _, _ = oracle.face_geometry(p["V0"], p["F"])
    t, mode = oracle.thickness_from_hits(normals, p["thick_idx"], p["thick_t_hit"], p["thick_prim"])
    assert t == p["thick_t"] and mode == p["thick_mode"], (t, p["thick_t"], mode, p["thick_mode"])


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_face_geometry_matches_numpy_element_for_element(slab, oracle, name):
    p = piece(slab, name)
    normals, areas, cent = oracle.face_geometry(p["V"], p["F"])
    v = p["V"]
    f = p["F"].astype(np.int64)
    assert np.array_equal(cent, (v[f[:, 0]] + v[f[:, 1]] + v[f[:, 2]]) / 3.0)
    assert np.all(np.abs(np.linalg.norm(normals, axis=1) - 1.0) < 1e-12)
    assert np.isclose(areas[p["frac"].astype(bool)].sum(), p["frac_area"], rtol=1e-12)


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_first_hits_agree_with_the_fixture_rays(slab, oracle, name):
    """E4's measurement (spatial/bvh.rs:10-19): the same rays, the same answers up to grazing
    edges; and the thickness from our own hits lands in the reference's histogram bin."""
    p = piece(slab, name)
    normals, _, cent = oracle.face_geometry(p["V0"], p["F"])
    mesh = oracle.Mesh(p["V0"], p["F"])
    idx = oracle.face_indices(len(p["F"]))
    assert np.array_equal(idx, p["thick_idx"])
    t, prim = oracle.cast_inward_rays(mesh, cent, normals, idx)
    ref_t, ref_prim = p["thick_t_hit"], p["thick_prim"]
    hit, ref_hit = np.isfinite(t), np.isfinite(ref_t)
    assert np.mean(hit == ref_hit) > 0.999
    both = hit & ref_hit
    assert np.mean(prim[both] == ref_prim[both]) > 0.995
    same = both & (prim == ref_prim)
    assert np.max(np.abs(t[same] - ref_t[same])) < 1e-4 * float(p["thick_t"])
    mine = oracle.thickness_from_hits(normals, idx, t, prim)
    bin_width = float(p["thick_t"]) * 2.0 / 60.0
    assert abs(float(mine[0]) - float(p["thick_t"])) <= bin_width


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_cone_votes_agree_with_the_fixture(slab, oracle, name):
    """R 3.4.3 over the dump's own smoothed normals (segment.rs:318-376) against seg.good."""
    p = piece(slab, name)
    normals, _, cent = oracle.face_geometry(p["V"], p["F"])
    mesh = oracle.Mesh(p["V"], p["F"])
    good = oracle.cone_votes(mesh, cent, normals, p["seg_NS"], normals, float(p["thick_t"]))
    ref = p["seg_good"]
    assert np.mean(good == ref) > 0.998
    assert np.mean((good >= 5) == (ref >= 5)) > 0.999


def test_stage2_ladder_matches_the_reference(slab, oracle):
    """The four rungs from s1.T[nms2.kept] against s2.T_reg1..T_frac2 (stage2.rs:40-50): every
    rung within 0.05 deg / 0.01 t, except chaotic ladders the reference itself refused."""
    op = oracle_pair(oracle, slab)
    sc = op["scales"]
    t = sc.t
    poses = slab["starts"].reshape(-1, 16)
    rungs = [(op["b"]["arrays"]["reg_p"], op["reg_t"], 0.2), (op["b"]["arrays"]["reg_p"], op["reg_t"], 0.08),
             (op["b"]["arrays"]["frac_p"], op["frac_t"], 0.08), (op["b"]["arrays"]["frac_p"], op["frac_t"], 0.04)]
    names = ("s2_T_reg1", "s2_T_reg2", "s2_T_frac1", "s2_T_frac2")
    chaotic = set()
    for (src, tgt, k), name in zip(rungs, names):
        regs = oracle.icp_rung(src, tgt, poses, k * t * sc.icp, 30)
        poses = np.array([np.array(r.transform[:]) for r in regs])
        for c in range(len(poses)):
            mine = poses[c].reshape(4, 4)
            ref = slab[name][c]
            if trace_deg(mine, ref) > ROT_DEG or origin_t(mine, ref, t) > TRANS_T:
                chaotic.add(c)
    accepted = slab["s2_accepted"].astype(bool)
    assert len(chaotic) <= CHAOTIC_SHARE * len(accepted), chaotic
    assert not any(accepted[c] for c in chaotic), chaotic


def test_verify_matches_the_reference_scores(slab, oracle):
    """R 6 at s2.T_frac2 against s2.scores.json and s2.accepted (verify.rs:74-86)."""
    op = oracle_pair(oracle, slab)
    params = slab_params(oracle, slab)
    for k, pose in enumerate(slab["s2_T_frac2"]):
        s = oracle.verify(op["a"]["surf"], op["b"]["surf"], pose, op["scales"], True)
        mine, ref = score_dict(s), reference_scores(slab, k)
        for key, tol in VERIFY_TOL.items():
            assert abs(mine[key] - ref[key]) <= tol, (k, key, mine[key], ref[key])
        assert oracle.accept(s, params, op["scales"]) == bool(slab["s2_accepted"][k]), k


def test_the_batched_ladder_reproduces_the_reference_verdicts(slab, oracle):
    """The whole stage-2 work item (4 rungs + R 6 + R 6.5) on the oracle's thread pool."""
    op = oracle_pair(oracle, slab)
    params = slab_params(oracle, slab)
    items = [oracle.WorkItem(0, k, (C.c_double * 16)(*slab["starts"][k].reshape(16)))
             for k in range(len(slab["starts"]))]
    cands, used = oracle.ladder_verify_batch([op["pair"]], items, params)
    assert used >= 1
    got = np.array([c.accepted for c in cands], bool)
    assert np.array_equal(got, slab["s2_accepted"].astype(bool))
    for k, c in enumerate(cands):
        ref = slab["s2_T_frac2"][k]
        mine = np.array(c.rungs[3].transform[:]).reshape(4, 4)
        if slab["s2_accepted"][k]:
            assert trace_deg(mine, ref) <= ROT_DEG and origin_t(mine, ref, op["scales"].t) <= TRANS_T
            assert abs(c.scores.tight - reference_scores(slab, k)["tight"]) <= VERIFY_TOL["tight"]


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_segmentation_reproduces_every_stage_of_the_fixture(slab, oracle, name):
    """R 3.4 end to end (segment.rs:511-631) on the dump's working mesh, t and res, against
    every intermediate the fixture records. The reference's own gate (sherd-parity
    stages/segmentation.rs:48-63) is area agreement >= 0.995; the restatement, with its balls
    summed in ascending face order as PointTree::within returns them, meets it exactly."""
    p = piece(slab, name)
    mesh = oracle.Mesh(p["V"], p["F"])
    labels, info, tr = oracle.segment(mesh, p["V"], p["F"], float(p["thick_t"]), float(p["res"]))
    votes, radius, angle, _ = p["seg_info"]
    assert info.votes == votes and info.smooth_radius == radius and info.boundary_angle == angle
    assert info.n_rep == len(p["seg_rep"])
    assert np.array_equal(tr["rep"][tr["near"]], p["seg_rep"][p["seg_near"]])
    cos = np.clip(np.sum(tr["ns"] * p["seg_NS"], axis=1), -1.0, 1.0)
    assert np.degrees(np.arccos(cos)).max() < 1e-4
    assert np.array_equal(tr["good"], p["seg_good"])
    for k in ("frac_raw", "frac_majority", "frac_islands", "has_ref"):
        assert np.array_equal(tr[k], p["seg_" + k]), k
    assert np.array_equal(labels, p["frac"])


def test_early_rejection_keeps_the_partial_scores_and_skips_the_fine_rungs(slab, oracle):
    """R 5.6 (pair.rs:315-340): below early_reject_tight at the pc_reg pose an item keeps the
    fracture and seam scores there, is rejected and runs no pc_frac rung; the others are the
    same as without the rule."""
    op = oracle_pair(oracle, slab)
    params = slab_params(oracle, slab)
    items = [oracle.WorkItem(0, k, (C.c_double * 16)(*slab["starts"][k].reshape(16)))
             for k in range(len(slab["starts"]))]
    base, _ = oracle.ladder_verify_batch([op["pair"]], items, params)
    params.early_reject_tight = 0.3
    early, _ = oracle.ladder_verify_batch([op["pair"]], items, params)
    rejected = [c.scores.partial == 1 for c in early]
    assert 0 < sum(rejected) < len(items)
    for b, e, r in zip(base, early, rejected):
        assert bytes(e.rungs[0]) == bytes(b.rungs[0]) and bytes(e.rungs[1]) == bytes(b.rungs[1])
        if r:
            assert e.accepted == 0 and e.scores.tight < 0.3
            assert e.scores.cont == 1.0 and e.scores.cont_n == -1.0 and e.scores.pen == 0.0
            for q in (2, 3):
                assert e.rungs[q].transform[:] == b.rungs[1].transform[:]
                assert e.rungs[q].iterations == 0 and e.rungs[q].correspondences == 0
        else:
            assert bytes(e) == bytes(b)


def test_coarse_scores_reproduce_the_stage1_rescore(slab, oracle):
    """R 5.4's re-score (executor/cpu.rs:46-68,136-169): B's breakline subset against A's whole
    breakline at scales.stage1, at the fixture's refined poses s1.T, gives s1.score exactly."""
    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    target = oracle.Cloud(a["brk_P"], a["brk_ns"])
    sub = b["brk_sub"].astype(np.int64)
    got = oracle.coarse_scores(target, b["brk_P"][sub], b["brk_ns"][sub], slab["s1_T"],
                               float(slab["scales"][3]))
    assert np.array_equal(got, slab["s1_score"])


def test_svd_rotation_matches_lapack(oracle):
    """umeyama's rotation U diag(1, 1, det U det V) V^T (icp.rs:585-590) against numpy's SVD,
    on full-rank, rank-2 and ill-conditioned matrices over twelve decades of scale."""
    rng = np.random.default_rng(0)
    for k in range(600):
        m = rng.normal(size=(3, 3)) * 10 ** rng.uniform(-6, 6)
        if k % 3 == 1:
            m[:, 2] = m[:, 0] * 0.5 + m[:, 1]
        elif k % 3 == 2:
            m = m @ np.diag([1.0, 1e-9, 1.0])
        u, _, vt = np.linalg.svd(m)
        ref = u @ np.diag([1.0, 1.0, np.sign(np.linalg.det(u) * np.linalg.det(vt))]) @ vt
        assert np.abs(oracle.svd_rotation(m) - ref).max() < 1e-11, k


def test_the_stage1_rung_holds_the_fixture_poses(slab, oracle):
    """R 5.4's last point-to-point rung (ladder.rs:131-141: 0.08 t icp, 20 iterations) started at
    the reference's refined stage-1 poses s1.T leaves every one of them where it is."""
    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    t, icp = float(slab["scales"][0]), float(slab["scales"][11])
    sub = b["brk_sub"].astype(np.int64)
    regs = oracle.icp_rung(b["brk_P"][sub], oracle.Cloud(a["brk_P"]), slab["s1_T"],
                           0.08 * t * icp, 20, point_to_point=True)
    for r, pose in zip(regs, slab["s1_T"]):
        mine = np.array(r.transform[:]).reshape(4, 4)
        assert trace_deg(mine, pose) < 1e-3 and origin_t(mine, pose, t) < 1e-6


@pytest.mark.parametrize("point_to_point", [False, True])
def test_a_single_pose_rung_is_the_same_on_one_thread_and_on_eight(slab, oracle, point_to_point):
    """With one pose, the oracle splits each pass's correspondence searches over its threads and
    still sums in point order: the registration is the same bytes on one thread and on eight."""
    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    t, icp = float(slab["scales"][0]), float(slab["scales"][11])
    target = oracle.Cloud(a["reg_p"], a["reg_n"])
    src = b["reg_p"]
    assert len(src) >= 4096
    for k in (0, 1, 2):
        init = slab["starts"][k].reshape(1, 16)
        one = oracle.icp_rung(src, target, init, 0.2 * t * icp, 30, threads=1,
                              point_to_point=point_to_point)
        eight = oracle.icp_rung(src, target, init, 0.2 * t * icp, 30, threads=8,
                                point_to_point=point_to_point)
        assert bytes(one[0]) == bytes(eight[0]), k
