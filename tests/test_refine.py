"""R 9, full-resolution join refinement (refine.rs), on the oracle and on the device.

Pinned to the reference's slab fixture: each fragment's vertex selection (`refine/<name>.idx`),
the joins its walk took (`refine/joins.json`: ends, radii, both rung poses, fitness, rmse / t)
and the refined poses (`refine/poses_final.json`), at the `refine` row's own tolerances
(sherd-parity/src/stages/refine.rs:61-67: 0.2 deg and 0.02 t per pose, 1e-4 in fitness,
0.02 in rmse / t; the radii exact). The reference's own unit cases of refine.rs:389-525 are
restated here too: Open3D's area-weighted vertex normals, the selection predicate and its
radius floor, the walk's order, and a join without a cloud.

On the device: the vertex normals are bit-identical to the oracle's; the selection is the
fixture's; the wide rung (sherd_refine_join) matches the oracle's rungs at the row's tolerances
on the slab, on a perturbed slab that takes many iterations, and on a 60 000-point surface, and
is reproducible run to run.
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest

from _slab import origin_t, piece, trace_deg

ROT_DEG = 0.2        # sherd-parity/src/stages/refine.rs:62
TRANS_T = 0.02       # refine.rs:64 (parity)
FITNESS_TOL = 1e-4   # refine.rs:67 (parity)


def _refine_mod():
    return importlib.import_module("sherd-refit_b200.refine")


def _groups(slab):
    sizes = slab["refine_group_sizes"].astype(int)
    members = slab["refine_group_members"].astype(int)
    out, k = [], 0
    for s in sizes:
        out.append(list(members[k:k + s]))
        k += s
    return out


def _used(slab):
    return [tuple(int(x) for x in e) for e in slab["refine_used"]]


def _centroids(v, f):
    v = np.asarray(v, np.float64)
    f = np.asarray(f, np.int64)
    return (v[f[:, 0]] + v[f[:, 1]] + v[f[:, 2]]) / 3.0


def _oracle_pieces(oracle, slab, own_selection=False):
    pieces = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        thick, res = (float(x) for x in p["stats_thick_res"])
        if own_selection:
            idx = oracle.select_candidates(p["V0"], _centroids(p["V"], p["F"]), p["frac"], thick,
                                           res)
        else:
            idx = p["refine_idx"]
        normals = oracle.vertex_normals(p["V0"], p["F"])
        pieces.append(oracle.RefinePiece(thick, res, oracle.cloud_from_indices(p["V0"], normals,
                                                                               idx)))
    return pieces


def _assert_matches_fixture(slab, poses, joins, t_of, tight=False):
    """The parity rows of sherd-parity/src/stages/refine.rs:384-478 against the fixture."""
    ends = slab["refine_join_ends"].astype(int)
    assert [(j.fixed, j.moving) for j in joins] == [tuple(e) for e in ends]
    rot_tol, trans_tol = (1e-9, 1e-9) if tight else (ROT_DEG, TRANS_T)
    for k, j in enumerate(joins):
        assert j.dist == list(slab["refine_join_dist"][k])          # exact
        t = min(t_of[j.fixed], t_of[j.moving])
        for r in range(2):
            theirs = slab["refine_join_rungs"][k, r]
            assert trace_deg(j.rungs[r], theirs) <= rot_tol
            assert origin_t(j.rungs[r], theirs, t) <= trans_tol
        fit, rmse_t = slab["refine_join_fit_rmse"][k]
        assert abs(j.fitness - fit) <= (1e-12 if tight else FITNESS_TOL)
        assert abs(j.rmse_t - rmse_t) <= TRANS_T
    after = slab["refine_after"]
    for group in _groups(slab):
        if len(group) < 2:
            continue
        g0 = group[0]
        for n in group[1:]:
            mine = np.linalg.inv(poses[g0]) @ poses[n]
            theirs = np.linalg.inv(after[g0]) @ after[n]
            assert trace_deg(mine, theirs) <= rot_tol
            assert origin_t(mine, theirs, t_of[n]) <= trans_tol


def _saddle():
    """refine.rs:462-478's saddle patch: 20 x 20 points of z = 0.4x^2 - 0.25y^2 + 0.1xy with
    their unit normals."""
    pts, nrm = [], []
    for i in range(20):
        for j in range(20):
            x, y = i * 0.1, j * 0.1
            pts.append([x, y, 0.4 * x * x - 0.25 * y * y + 0.1 * x * y])
            g = np.array([-(0.8 * x + 0.1 * y), -(0.1 * x - 0.5 * y), 1.0])
            nrm.append(g / np.linalg.norm(g))
    return np.array(pts), np.array(nrm)


def _bumpy(n, seed):
    """Points and unit normals of the surface z = 3 sin(x/7) cos(y/9) + 0.002 x^2 over
    [-50, 50]^2, uniformly sampled."""
    rng = np.random.default_rng(seed)
    x, y = rng.uniform(-50.0, 50.0, size=(2, n))
    z = 3.0 * np.sin(x / 7.0) * np.cos(y / 9.0) + 0.002 * x * x
    gx = 3.0 / 7.0 * np.cos(x / 7.0) * np.cos(y / 9.0) + 0.004 * x
    gy = -3.0 / 9.0 * np.sin(x / 7.0) * np.sin(y / 9.0)
    nrm = np.stack([-gx, -gy, np.ones(n)], axis=1)
    return np.stack([x, y, z], axis=1), nrm / np.linalg.norm(nrm, axis=1, keepdims=True)


def _twist_pose(deg, axis, shift):
    axis = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    a = np.radians(deg)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    t = np.eye(4)
    t[:3, :3] = np.eye(3) + np.sin(a) * k + (1 - np.cos(a)) * (k @ k)
    t[:3, 3] = shift
    return t


def _oracle_join(oracle, src, tgt, tgt_n, pose_fixed, pose_moving, dist, iterations=40):
    """refine_one's two rungs on the oracle, for explicit clouds."""
    s = oracle.place_fused(src, pose_moving)
    cloud = oracle.Cloud(oracle.place_fused(tgt, pose_fixed),
                         oracle.place_fused(tgt_n, pose_fixed, rotate_only=True))
    pose, out = np.eye(4), []
    for d in dist:
        r = oracle.icp_rung(s, cloud, pose, d, iterations)[0]
        pose = np.array(r.transform[:]).reshape(4, 4)
        out.append(r)
    return out


# ---- the oracle, pinned ---------------------------------------------------------------------


def test_vertex_normals_are_open3ds_area_weighted_sum(oracle):
    """refine.rs:402-427: a small face with normal (0,0,1) and a 20 times larger one with normal
    (0,1,0) give (0,10,1)/sqrt(101); a vertex of one face keeps that face's normal; a vertex no
    face references gets (0,0,1)."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [10, 0, 0], [9, 9, 9]], float)
    f = np.array([[0, 1, 2], [0, 3, 4]], np.uint32)
    n = oracle.vertex_normals(v, f)
    assert np.all(np.abs(n[0] - np.array([0.0, 10.0, 1.0]) / np.sqrt(101.0)) < 1e-15)
    assert np.array_equal(n[1], [0.0, 0.0, 1.0])
    assert np.array_equal(n[5], [0.0, 0.0, 1.0])


def test_oracle_vertex_normals_are_the_face_order_sums(oracle, slab):
    """The C restatement against numpy's unbuffered np.add.at over the corners in face order
    (the reference's loop order), bit for bit, on both slab originals."""
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        v, f = p["V0"], p["F"].astype(np.int64)
        e1 = v[f[:, 1]] - v[f[:, 0]]
        e2 = v[f[:, 2]] - v[f[:, 0]]
        fn = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                       e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                       e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1)
        acc = np.zeros_like(v)
        np.add.at(acc, f.reshape(-1), np.repeat(fn, 3, axis=0))
        length = np.sqrt((acc[:, 0] * acc[:, 0] + acc[:, 1] * acc[:, 1]) + acc[:, 2] * acc[:, 2])
        want = np.where(length[:, None] > 0, acc / np.where(length > 0, length, 1.0)[:, None],
                        np.array([0.0, 0.0, 1.0]))
        assert np.array_equal(oracle.vertex_normals(v, p["F"]), want)


def test_selection_predicate_and_its_radius_floor(oracle):
    """refine.rs:434-453: a fracture centroid AND a distance strictly under
    max(0.15 t, 1.5 res); the cap keeps max_points of the candidates."""
    v = np.array([[0.0, 0, 0], [1.0, 0, 0], [10.0, 0, 0]])
    cent = np.array([[0.1, 0, 0], [1.2, 0, 0], [9.5, 0, 0]])
    frac = np.array([1, 0, 1], np.uint8)
    assert list(oracle.select_candidates(v, cent, frac, 2.0, 0.1)) == [0]
    assert list(oracle.select_candidates(v, cent, frac, 2.0, 1.0)) == [0, 2]
    capped = oracle.cap_selection(oracle.select_candidates(v, cent, frac, 2.0, 1.0), 1)
    assert len(capped) == 1 and capped[0] in (0, 2)


def test_oracle_selection_is_the_fixture_selection(oracle, slab):
    """The reference's refine/<name>.idx, entry for entry (both pieces are under the cap)."""
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        thick, res = (float(x) for x in p["stats_thick_res"])
        got = oracle.select_candidates(p["V0"], _centroids(p["V"], p["F"]), p["frac"], thick, res)
        assert len(p["refine_idx"]) < oracle.REFINE_MAX_POINTS
        assert np.array_equal(got, p["refine_idx"])


def test_oracle_refinement_reproduces_the_fixture(oracle, slab):
    """From the assembly's poses, groups and joins: the same walk, the same radii, the rung
    poses, fitness and refined poses at the row's tolerances; and here, on the slab, to within
    1e-9 (deg, t) and 1e-12 in fitness."""
    pieces = _oracle_pieces(oracle, slab)
    t_of = [pc.thick for pc in pieces]
    poses, joins = oracle.refine_joins(pieces, list(slab["refine_before"]), _groups(slab),
                                       _used(slab))
    _assert_matches_fixture(slab, poses, joins, t_of, tight=True)
    own, own_joins = oracle.refine_joins(_oracle_pieces(oracle, slab, own_selection=True),
                                         list(slab["refine_before"]), _groups(slab), _used(slab))
    _assert_matches_fixture(slab, own, own_joins, t_of, tight=True)


def test_the_walk_starts_at_the_groups_first_fragment(oracle):
    """refine.rs:456-500: used order (1,2),(0,1) inside group [0,1,2] walks (0,1) then (1,2);
    both displaced copies are pulled back onto fragment 0's saddle; the empty group adds
    nothing."""
    pts, nrm = _saddle()
    cloud = oracle.FractureCloud(np.arange(400), pts, nrm)
    pieces = [oracle.RefinePiece(1.0, 0.05, cloud) for _ in range(3)]
    poses = [np.eye(4) for _ in range(3)]
    poses[1][2, 3] = 0.004
    poses[2][2, 3] = 0.006
    out, joins = oracle.refine_joins(pieces, poses, [[0, 1, 2], []], [(1, 2), (0, 1)])
    assert [(j.fixed, j.moving) for j in joins] == [(0, 1), (1, 2)]
    for n in (1, 2):
        assert abs(out[n][2, 3]) < 1e-9, out[n]


def test_a_join_without_a_cloud_is_skipped(oracle):
    """refine.rs:503-524."""
    cloud = oracle.FractureCloud([0], [[0.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]])
    pieces = [oracle.RefinePiece(1.0, 0.1, cloud), oracle.RefinePiece(1.0, 0.1, None)]
    poses = [np.eye(4), np.eye(4)]
    out, joins = oracle.refine_joins(pieces, poses, [[0, 1]], [(0, 1)])
    assert joins == [] and all(np.array_equal(a, b) for a, b in zip(out, poses))


# ---- the package's host logic, on the CPU ---------------------------------------------------------


class _OracleDevice:
    """Answers the Context calls refine.py makes with the oracle, so that the walk, the
    selection mask and the radii of the package run here without a GPU."""

    def __init__(self, oracle):
        self.oracle = oracle

    def cloud(self, p, n=None):
        return self.oracle.Cloud(p, n)

    def vertex_normals(self, v, f):
        return self.oracle.vertex_normals(v, f)

    def fracture_cloud(self, v, f, centroids, fracture, radius):
        """sherd_fracture_cloud's contract on the oracle: the selected vertices (nearest
        centroid strictly within the radius is a fracture face), their points and normals."""
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
        j, _ = self.oracle.Cloud(np.ascontiguousarray(centroids, np.float64)).nearest_below(v, radius)
        keep = j != 0xFFFFFFFF
        keep[keep] = np.asarray(fracture).astype(bool).reshape(-1)[j[keep]]
        idx = np.flatnonzero(keep).astype(np.uint32)
        return idx, v[idx.astype(np.int64)], self.oracle.vertex_normals(v, f)[idx.astype(np.int64)]

    def refine_join(self, source, target, target_normals, pose_fixed, pose_moving, dist,
                    max_iteration=40):
        return _oracle_join(self.oracle, source, target, target_normals, pose_fixed,
                            pose_moving, dist, max_iteration)


def test_package_walk_and_selection_on_the_oracle(oracle, slab):
    """refine.py's fracture_cloud and refine_joins over an oracle-backed context give the fixture's
    selection and the oracle's own refinement, bit for bit."""
    rf = _refine_mod()
    dev = _OracleDevice(oracle)
    pieces = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        thick, res = (float(x) for x in p["stats_thick_res"])
        cloud = rf.fracture_cloud(dev, p["V0"], p["F"], _centroids(p["V"], p["F"]), p["frac"],
                                  thick, res)
        assert np.array_equal(cloud.idx, p["refine_idx"])
        pieces.append(rf.RefinePiece(thick, res, cloud))
    got = rf.refine_joins(dev, pieces, list(slab["refine_before"]), _groups(slab), _used(slab))
    want, want_joins = oracle.refine_joins(_oracle_pieces(oracle, slab),
                                           list(slab["refine_before"]), _groups(slab),
                                           _used(slab))
    assert [(j.fixed, j.moving, j.dist) for j in got.joins] == \
        [(j.fixed, j.moving, j.dist) for j in want_joins]
    for a, b in zip(got.poses, want):
        assert np.array_equal(a, b)
    _assert_matches_fixture(slab, got.poses, got.joins, [pc.thick for pc in pieces], tight=True)


def test_cap_selection_is_a_seeded_draw_without_replacement():
    rf = _refine_mod()
    idx = np.arange(0, 3 * 200_000, 3, dtype=np.uint32)
    assert np.array_equal(rf.cap_selection(idx[:1000]), idx[:1000])
    a = rf.cap_selection(idx)
    assert len(a) == rf.MAX_POINTS and len(np.unique(a)) == rf.MAX_POINTS
    assert np.all(np.isin(a, idx)) and not np.all(np.diff(a.astype(np.int64)) > 0)
    assert np.array_equal(a, rf.cap_selection(idx))


# ---- on the device ----------------------------------------------------------------------------


@pytest.mark.gpu
def test_device_vertex_normals_are_bit_identical(gpu_ctx, oracle, slab):
    synth = importlib.import_module("sherd-refit_b200.synth")
    cases = [(piece(slab, n)["V0"], piece(slab, n)["F"]) for n in ("pieceA", "pieceB")]
    fr = synth.make("pot", 0).fragments[0]
    cases.append((fr.v.astype(np.float64), fr.f))
    # A repeated corner, a collinear face and a vertex no face references.
    cases.append((np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 0, 0], [7, 7, 7]], float),
                  np.array([[0, 1, 2], [0, 0, 2], [0, 1, 3]], np.uint32)))
    for v, f in cases:
        assert np.array_equal(gpu_ctx.vertex_normals(v, f), oracle.vertex_normals(v, f))


@pytest.mark.gpu
def test_device_selection_is_the_fixture_selection(gpu_ctx, slab):
    rf = _refine_mod()
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        thick, res = (float(x) for x in p["stats_thick_res"])
        cloud = rf.fracture_cloud(gpu_ctx, p["V0"], p["F"], _centroids(p["V"], p["F"]),
                                  p["frac"], thick, res)
        assert np.array_equal(cloud.idx, p["refine_idx"])


@pytest.mark.gpu
def test_fused_fracture_cloud_equals_the_two_call_path(gpu_ctx, oracle, slab):
    """sherd_fracture_cloud (one upload, selection, normals and gathers on the device) gives the
    selection of sherd_nearest_below over the centroids and the sherd_vertex_normals values,
    bit for bit, on both slab pieces and on a pot fragment (with a cap that draws)."""
    rf = _refine_mod()
    synth = importlib.import_module("sherd-refit_b200.synth")
    cases = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        cases.append((p["V0"], p["F"], _centroids(p["V"], p["F"]), p["frac"],
                      *(float(x) for x in p["stats_thick_res"])))
    fr = synth.make("pot", 0).fragments[1]
    v = fr.v.astype(np.float64)
    cases.append((v, fr.f, _centroids(v, fr.f), fr.frac, float(fr.t), float(fr.res)))
    for v, f, cen, frac, thick, res in cases:
        idx = rf.select_candidates(gpu_ctx, v, cen, frac, thick, res)
        nrm = gpu_ctx.vertex_normals(v, f)
        radius = max(rf.SELECT_T * thick, rf.SELECT_RES * res)
        got_idx, got_p, got_n = gpu_ctx.fracture_cloud(v, f, cen, frac, radius)
        assert len(idx) > 0 and np.array_equal(got_idx, idx)
        assert np.array_equal(got_p, np.asarray(v, np.float64)[idx.astype(np.int64)])
        assert np.array_equal(got_n, nrm[idx.astype(np.int64)])
        assert np.array_equal(got_n, oracle.vertex_normals(v, f)[idx.astype(np.int64)])
        small = max(1, len(idx) // 3)   # the cap's draw among the fused path's vertices
        want = rf.cap_selection(idx, small, 0)
        got = rf.FractureCloud(got_idx, got_p, got_n)
        at = np.searchsorted(got.idx, want)
        assert np.array_equal(got.idx[at], want)
        assert np.array_equal(got.normals[at], nrm[want.astype(np.int64)])


@pytest.mark.gpu
def test_device_refinement_reproduces_the_fixture(gpu_ctx, slab):
    rf = _refine_mod()
    pieces = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        thick, res = (float(x) for x in p["stats_thick_res"])
        cloud = rf.fracture_cloud(gpu_ctx, p["V0"], p["F"], _centroids(p["V"], p["F"]),
                                  p["frac"], thick, res)
        pieces.append(rf.RefinePiece(thick, res, cloud))
    out = rf.refine_joins(gpu_ctx, pieces, list(slab["refine_before"]), _groups(slab),
                          _used(slab))
    _assert_matches_fixture(slab, out.poses, out.joins, [pc.thick for pc in pieces])


@pytest.mark.gpu
def test_device_rungs_match_the_oracle_on_a_perturbed_slab(gpu_ctx, oracle, slab):
    """B moved 0.6 deg and 0.08 t off its assembled pose, so that both rungs iterate: the wide
    rung against the oracle's at the row's tolerances."""
    pieces = _oracle_pieces(oracle, slab)
    before = [np.array(p) for p in slab["refine_before"]]
    t = min(pc.thick for pc in pieces)
    before[1] = _twist_pose(0.6, [0.3, -1.0, 0.4], [0.08 * t, -0.03 * t, 0.02 * t]) @ before[1]
    sc = oracle.scales_for(oracle.default_params(), t, max(pc.res for pc in pieces))
    dist = [k * sc.t * sc.icp for k in oracle.REFINE_RUNGS]
    a, b = pieces
    want = _oracle_join(oracle, b.cloud.points, a.cloud.points, a.cloud.normals, before[0],
                        before[1], dist)
    got = gpu_ctx.refine_join(b.cloud.points, a.cloud.points, a.cloud.normals, before[0],
                              before[1], dist, 40)
    assert want[0].iterations > 3
    for g, w in zip(got, want):
        gt, wt = np.array(g.transform[:]).reshape(4, 4), np.array(w.transform[:]).reshape(4, 4)
        assert trace_deg(gt, wt) <= ROT_DEG and origin_t(gt, wt, t) <= TRANS_T
        assert abs(g.fitness - w.fitness) <= FITNESS_TOL
        assert abs(g.inlier_rmse - w.inlier_rmse) / t <= TRANS_T


@pytest.mark.gpu
def test_device_wide_rung_on_a_large_surface(gpu_ctx, oracle):
    """60 000 source points against 80 000 target points of one bumpy surface, the source moved
    1.5 deg and 0.6 off: both rungs against the oracle's, and the same answer twice."""
    src, _ = _bumpy(60_000, 1)
    tgt, tgt_n = _bumpy(80_000, 2)
    moving = _twist_pose(1.5, [1.0, 0.5, -0.2], [0.6, -0.3, 0.2])
    dist = [3.0, 1.2]
    want = _oracle_join(oracle, src, tgt, tgt_n, np.eye(4), moving, dist)
    got = gpu_ctx.refine_join(src, tgt, tgt_n, np.eye(4), moving, dist, 40)
    again = gpu_ctx.refine_join(src, tgt, tgt_n, np.eye(4), moving, dist, 40)
    for g, w, h in zip(got, want, again):
        gt, wt = np.array(g.transform[:]).reshape(4, 4), np.array(w.transform[:]).reshape(4, 4)
        assert trace_deg(gt, wt) <= ROT_DEG and origin_t(gt, wt, 30.0) <= TRANS_T
        assert abs(g.fitness - w.fitness) <= FITNESS_TOL
        assert bytes(g) == bytes(h)
    # The correction undoes most of the displacement.
    final = np.array(got[1].transform[:]).reshape(4, 4) @ moving
    assert trace_deg(final, np.eye(4)) < 0.3 and np.linalg.norm(final[:3, 3]) < 0.2
    # Rungs cut short by the iteration cap (0: the first pass's numbers only).
    for cap in (0, 2):
        want = _oracle_join(oracle, src, tgt, tgt_n, np.eye(4), moving, dist, cap)
        got = gpu_ctx.refine_join(src, tgt, tgt_n, np.eye(4), moving, dist, cap)
        for g, w in zip(got, want):
            assert (g.iterations, g.converged) == (w.iterations, w.converged)
            assert abs(g.fitness - w.fitness) <= FITNESS_TOL
            assert abs(g.inlier_rmse - w.inlier_rmse) <= 1e-6 * max(w.inlier_rmse, 1.0)
            if cap == 0:   # both passes at the identity: the same points, the same matches
                assert g.correspondences == w.correspondences


@pytest.mark.gpu
def test_device_walk_saddle_and_edge_cases(sherd, gpu_ctx):
    rf = _refine_mod()
    pts, nrm = _saddle()
    cloud = rf.FractureCloud(np.arange(400, dtype=np.uint32), pts, nrm)
    pieces = [rf.RefinePiece(1.0, 0.05, cloud) for _ in range(3)]
    poses = [np.eye(4) for _ in range(3)]
    poses[1][2, 3] = 0.004
    poses[2][2, 3] = 0.006
    out = rf.refine_joins(gpu_ctx, pieces, poses, [[0, 1, 2], []], [(1, 2), (0, 1)])
    assert [(j.fixed, j.moving) for j in out.joins] == [(0, 1), (1, 2)]
    for n in (1, 2):
        assert abs(out.poses[n][2, 3]) < 1e-9
    # An empty side leaves both rungs at the identity; bad arguments are refused.
    regs = gpu_ctx.refine_join(np.zeros((0, 3)), pts, nrm, np.eye(4), np.eye(4), [0.1, 0.05])
    assert all(np.array_equal(np.array(r.transform[:]).reshape(4, 4), np.eye(4)) for r in regs)
    bad = np.eye(4)
    bad[0, 3] = np.nan
    with pytest.raises(sherd.SherdError):
        gpu_ctx.refine_join(pts, pts, nrm, bad, np.eye(4), [0.1, 0.05])
    with pytest.raises(sherd.SherdError):
        gpu_ctx.refine_join(pts, pts, nrm, np.eye(4), np.eye(4), [0.1, 0.05], -1)
    with pytest.raises(sherd.SherdError):
        gpu_ctx.vertex_normals(pts, np.array([[0, 1, 400]], np.uint32))


@pytest.mark.gpu
def test_fused_cloud_and_face_inputs_are_checked_on_the_device(sherd, gpu_ctx, slab):
    """The face indices, the vertices and the centroids are checked after their upload: an index
    at the vertex count, or one non-finite coordinate anywhere, is refused with E_INVALID and the
    context stays usable; with clean inputs the call then gives the same cloud as before."""
    _abi = importlib.import_module("sherd-refit_b200._abi")
    p = piece(slab, "pieceA")
    v = np.asarray(p["V0"], np.float64)
    f = np.asarray(p["F"], np.uint32)
    cen = _centroids(p["V"], p["F"])
    frac = p["frac"]
    thick, res = (float(x) for x in p["stats_thick_res"])
    radius = max(_refine_mod().SELECT_T * thick, _refine_mod().SELECT_RES * res)
    want = gpu_ctx.fracture_cloud(v, f, cen, frac, radius)
    bad_f = f.copy()
    bad_f[len(f) // 2, 1] = len(v)
    for call in (lambda: gpu_ctx.fracture_cloud(v, bad_f, cen, frac, radius),
                 lambda: gpu_ctx.vertex_normals(v, bad_f),
                 lambda: gpu_ctx.face_geometry(v, bad_f)):
        with pytest.raises(sherd.SherdError) as e:
            call()
        assert e.value.code == _abi.E_INVALID
    for which in ("v", "cen"):
        for x in (np.nan, np.inf):
            vv, cc = v.copy(), cen.copy()
            (vv if which == "v" else cc)[len(vv if which == "v" else cc) - 1, 2] = x
            with pytest.raises(sherd.SherdError) as e:
                gpu_ctx.fracture_cloud(vv, f, cc, frac, radius)
            assert e.value.code == _abi.E_INVALID
    # No vertices but faces: every index is out of range.
    with pytest.raises(sherd.SherdError):
        gpu_ctx.vertex_normals(np.zeros((0, 3)), f[:1])
    got = gpu_ctx.fracture_cloud(v, f, cen, frac, radius)
    assert all(np.array_equal(a, b) for a, b in zip(got, want))
