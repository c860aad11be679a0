"""Every fixture check can be made to fail (the reference's own rule for its parity harness,
sherd-parity/tests/stages_slab.rs:1-8: "a harness that cannot be made to fail is not evidence").

For each stage the oracle is pinned on, one mistake is planted in the oracle's input or in one
of its parameters, on the CPU, and the same comparison the pinning test makes is shown to
reject the result.
"""

from __future__ import annotations

import numpy as np
import pytest

from _slab import (ROT_DEG, TRANS_T, VERIFY_TOL, origin_t, oracle_pair, piece, reference_scores,
                   score_dict, trace_deg)


def test_thickness_rejects_shifted_hits(slab, oracle):
    p = piece(slab, "pieceA")
    normals, _, _ = oracle.face_geometry(p["V0"], p["F"])
    t, _ = oracle.thickness_from_hits(normals, p["thick_idx"], p["thick_t_hit"] * np.float32(1.01),
                                      p["thick_prim"])
    assert t != p["thick_t"]


def test_segmentation_rejects_a_wrong_thickness(slab, oracle):
    p = piece(slab, "pieceB")
    mesh = oracle.Mesh(p["V"], p["F"])
    labels, info, _ = oracle.segment(mesh, p["V"], p["F"], 1.2 * float(p["thick_t"]), float(p["res"]))
    assert info.n_rep != len(p["seg_rep"]) or not np.array_equal(labels, p["frac"])


def test_verification_rejects_a_displaced_pose(slab, oracle):
    op = oracle_pair(oracle, slab)
    k = int(np.argmax(slab["s2_accepted"]))
    pose = slab["s2_T_frac2"][k].copy()
    pose[:3, 3] += 0.03 * op["scales"].t * np.array([0.6, 0.0, 0.8])
    mine = score_dict(oracle.verify(op["a"]["surf"], op["b"]["surf"], pose, op["scales"], True))
    ref = reference_scores(slab, k)
    assert any(abs(mine[key] - ref[key]) > tol for key, tol in VERIFY_TOL.items())


def test_stage2_ladder_rejects_a_wrong_radius(slab, oracle):
    op = oracle_pair(oracle, slab)
    sc = op["scales"]
    k = int(np.argmax(slab["s2_accepted"]))
    start = slab["starts"][k]
    reg = oracle.icp_rung(op["b"]["arrays"]["reg_p"], op["reg_t"], start, 0.02 * sc.t * sc.icp, 30)
    mine = np.array(reg[0].transform[:]).reshape(4, 4)
    ref = slab["s2_T_reg1"][k]
    assert trace_deg(mine, ref) > ROT_DEG or origin_t(mine, ref, sc.t) > TRANS_T


def test_coarse_scores_reject_a_wrong_radius(slab, oracle):
    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    hyp = oracle.hypotheses({"p": a["brk_P"], "ns": a["brk_ns"], "f": a["brk_f"], "dih": a["brk_dih"]},
                            {"p": b["brk_P"], "ns": b["brk_ns"], "f": b["brk_f"], "dih": b["brk_dih"]},
                            a["brk_sub"], b["brk_sub"])
    idx = slab["coarse_idx"].astype(np.int64)
    sc = oracle.scales_from(slab["scales"])
    cs = oracle.coarse_scores(oracle.Cloud(a["brk_P"], a["brk_ns"]), b["brk_P"][idx], b["brk_ns"][idx],
                              hyp[2], 1.05 * sc.coarse)
    assert not np.array_equal(cs, slab["coarse_cs"])


def test_hypotheses_reject_a_wrong_dihedral_tolerance(slab, oracle):
    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    pa, _, _ = oracle.hypotheses({"p": a["brk_P"], "ns": a["brk_ns"], "f": a["brk_f"], "dih": a["brk_dih"]},
                                 {"p": b["brk_P"], "ns": b["brk_ns"], "f": b["brk_f"], "dih": b["brk_dih"]},
                                 a["brk_sub"], b["brk_sub"], 24.0)
    assert len(pa) != len(slab["hyp_pa"])


def test_suppression_rejects_a_wrong_translation_tolerance(slab, oracle):
    sc = oracle.scales_from(slab["scales"])
    kept2 = oracle.nms(slab["nms2_order"], slab["s1_T"], slab["s1_score"], 3.0 * sc.nms, 10,
                       oracle.STAGE1_FLOOR)
    assert not np.array_equal(kept2, slab["nms2_kept"])


def test_breaklines_reject_a_flipped_label(slab, oracle):
    p = piece(slab, "pieceB")
    frac = p["frac"].copy()
    edge = int(np.flatnonzero(frac)[0])
    frac[edge] = 0
    b = oracle.breaklines(p["V"], p["F"], frac, float(p["md_params"][0]))
    assert len(b["p"]) != len(p["brk_P"]) or not np.array_equal(b["p"], p["brk_P"])


def test_samples_reject_another_seed(slab, oracle):
    p = piece(slab, "pieceB")
    s = oracle.samples(p["V"], p["F"], p["frac"], p["brk_P"], float(p["md_params"][0]), seed=1)
    assert not np.array_equal(s["S"], p["S"])


def test_refinement_rejects_a_wrong_rung(slab, oracle, monkeypatch):
    monkeypatch.setattr(oracle, "REFINE_RUNGS", (0.04, 0.02))
    pieces = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        thick, res = (float(x) for x in p["stats_thick_res"])
        pieces.append(oracle.RefinePiece(thick, res, oracle.cloud_from_indices(
            p["V0"], oracle.vertex_normals(p["V0"], p["F"]), p["refine_idx"])))
    _, joins = oracle.refine_joins(pieces, list(slab["refine_before"]), [[0, 1]], [(0, 1)])
    assert joins[0].dist != list(slab["refine_join_dist"][0])


def test_refine_selection_rejects_a_wrong_radius(slab, oracle, monkeypatch):
    """A radius under the vertex spacing (0.01 t, 0.1 res instead of 0.15 t, 1.5 res) drops
    vertices the reference keeps."""
    monkeypatch.setattr(oracle, "REFINE_SELECT_T", 0.01)
    monkeypatch.setattr(oracle, "REFINE_SELECT_RES", 0.1)
    p = piece(slab, "pieceA")
    v, f = p["V"], p["F"].astype(np.int64)
    cent = (v[f[:, 0]] + v[f[:, 1]] + v[f[:, 2]]) / 3.0
    thick, res = (float(x) for x in p["stats_thick_res"])
    idx = oracle.select_candidates(p["V0"], cent, p["frac"], thick, res)
    assert not np.array_equal(idx, p["refine_idx"])


@pytest.mark.parametrize("name", ["pieceA"])
def test_vertex_normals_reject_unit_face_weights(slab, oracle, name):
    """Open3D's rule weights each face by twice its area; the mean of unit normals is another
    answer, and the comparison sees it."""
    p = piece(slab, name)
    v, f = p["V0"], p["F"].astype(np.int64)
    fn, _, _ = oracle.face_geometry(v, f)
    acc = np.zeros_like(v)
    np.add.at(acc, f.reshape(-1), np.repeat(fn, 3, axis=0))
    unit = acc / np.linalg.norm(acc, axis=1, keepdims=True)
    assert not np.array_equal(unit, oracle.vertex_normals(v, p["F"]))
