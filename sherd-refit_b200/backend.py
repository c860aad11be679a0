"""The CUDA backend as Python objects: a context, device meshes and clouds, and the calls of
include/sherd_cuda.h with numpy arrays in and out.

Names follow the reference: `Mesh` is its `RayScene` (spatial/bvh.rs:36-192), `Cloud` its
`PointTree` with optional normals (spatial/kdtree.rs:31-258; `IcpTarget`, matching/icp.rs:
205-302), `Surfaces` its R 6 view of a fragment (matching/verify.rs:223-299), `Pair` what
`Pair::stage2_batch` reads (matching/pair.rs:298-372, 592-630).
"""

from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass

import numpy as np

from . import _abi as A
from ._abi import check, ptr


def _f32(a, shape=(-1, 3)):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(shape)


def _f64(a, shape=(-1, 3)):
    return np.ascontiguousarray(a, dtype=np.float64).reshape(shape)


def _u32(a, shape=(-1,)):
    return np.ascontiguousarray(a, dtype=np.uint32).reshape(shape)


def _pose(t) -> np.ndarray:
    return _f64(t, (16,))


def _frames(fr):
    """A sherd_frames over contiguous f64 copies of fr.p, fr.ns, fr.f, fr.dih (kept alive in the
    returned tuple)."""
    p, ns, f = _f64(fr.p), _f64(fr.ns), _f64(fr.f)
    dih = _f64(fr.dih, (-1,))
    if not (len(p) == len(ns) == len(f) == len(dih)):
        raise A.SherdError(A.E_INVALID, "frame arrays differ in length")
    return A.Frames(ptr(p), ptr(ns), ptr(f), ptr(dih), len(p)), (p, ns, f, dih)


ALL = 0xFFFFFFFF


def order_by_score(score, limit: int = ALL) -> np.ndarray:
    """nms::order_by_score (nms.rs:46-59): descending (f64 total order), ties by ascending
    index, the first `limit`."""
    s = _f64(score, (-1,))
    m = min(len(s), int(limit))
    out = np.empty(m, np.uint32)
    n = C.c_uint32(0)
    if A.lib().sherd_order_by_score(s, len(s), int(min(limit, ALL)), ptr(out), C.byref(n)):
        raise A.SherdError(A.E_INVALID, "order_by_score")
    return out[:n.value]


def nms(order, poses, score, trans_tol: float, topk: int, floor: float) -> np.ndarray:
    """nms::nms (nms.rs:61-86) over row-major 4x4 poses: the kept indices, in keeping order."""
    order = _u32(order)
    poses = _f64(poses, (-1, 16))
    score = _f64(score, (-1,))
    if len(poses) != len(score):
        raise A.SherdError(A.E_INVALID, "one score per pose")
    kept = np.empty(max(min(len(order), max(int(topk), 1)), 1), np.uint32)
    n = C.c_uint32(0)
    if A.lib().sherd_nms(order, len(order), poses, score, len(poses), float(trans_tol), int(topk),
                         float(floor), ptr(kept), C.byref(n)):
        raise A.SherdError(A.E_INVALID, "nms: an order entry names no pose")
    return kept[:n.value].copy()


def read_mesh(path) -> tuple[np.ndarray, np.ndarray]:
    """io::load_mesh (io/mod.rs:114-137) for a PLY file: the cleaned (v f64 (nv, 3), f u32
    (nf, 3)). Raises SherdError on a malformed file or one with no triangle."""
    h, nv, nf = C.c_void_p(), C.c_uint32(0), C.c_uint32(0)
    rc = A.lib().sherd_mesh_read(str(path).encode(), C.byref(h), C.byref(nv), C.byref(nf))
    if rc:
        msg = A.lib().sherd_last_error(None)
        raise A.SherdError(rc, msg.decode() if msg else "sherd_mesh_read")
    try:
        v = np.empty((nv.value, 3))
        f = np.empty((nf.value, 3), np.uint32)
        A.lib().sherd_host_mesh_copy(h, v, f)
    finally:
        A.lib().sherd_host_mesh_free(h)
    return v, f


class _Handle:
    _free = ""

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                getattr(A.lib(), self._free)(h)
            except Exception:
                pass
            self.h = None


def default_params() -> A.Params:
    """Params::default (params.rs:141-190), the fields the C ABI reads."""
    p = A.Params()
    A.lib().sherd_params_default(C.byref(p))
    return p


def scales_for_pair(params: A.Params, t: float, res: float) -> A.Scales:
    """Scales::for_pair (matching/scales.rs:72-88)."""
    s = A.Scales()
    rc = A.lib().sherd_scales_for_pair(C.byref(params), float(t), float(res), C.byref(s))
    if rc:
        raise A.SherdError(rc, "scales_for_pair")
    return s


def accept(scores: A.Scores, params: A.Params, scales: A.Scales) -> bool:
    """verify::accept (matching/verify.rs:632-638)."""
    return bool(A.lib().sherd_accept(C.byref(scores), C.byref(params), C.byref(scales)))


class Context:
    """One device and its stream (sherd_open); every call of this backend goes through one."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        rc = A.lib().sherd_open(int(device), C.byref(self.h))
        if rc:
            msg = A.lib().sherd_last_error(None)
            raise A.SherdError(rc, msg.decode() if msg else "sherd_open failed")
        self.device = device

    def close(self):
        if self.h:
            A.lib().sherd_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- context ---------------------------------------------------------------------------
    @property
    def name(self) -> str:
        """Executor::name (executor/mod.rs:107)."""
        return A.lib().sherd_name().decode()

    def device_slack(self) -> int:
        """Executor::device_slack (executor/mod.rs:134-136)."""
        return int(A.lib().sherd_device_slack(self.h))

    def set_timeout_ms(self, ms: int) -> None:
        check(self.h, A.lib().sherd_set_timeout_ms(self.h, int(ms)))

    def abort(self) -> None:
        check(self.h, A.lib().sherd_abort(self.h))

    def stats(self) -> dict:
        buf = C.create_string_buffer(1 << 16)
        check(self.h, A.lib().sherd_stats_json(self.h, buf, len(buf)))
        return json.loads(buf.value.decode())

    # -- objects -------------------------------------------------------------------------------
    def mesh(self, v, f) -> "Mesh":
        return Mesh(self, v, f)

    def cloud(self, p, n=None) -> "Cloud":
        return Cloud(self, p, n)

    # -- Executor-shaped calls -------------------------------------------------------------------
    def first_hit(self, mesh: "Mesh", origins, dirs):
        """RayScene::first_hit for every ray: (t f32, prim u32), +inf / 0xFFFFFFFF on a miss."""
        o, d = _f32(origins), _f32(dirs)
        n = len(o)
        t = np.empty(n, np.float32)
        prim = np.empty(n, np.uint32)
        check(self.h, A.lib().sherd_first_hit(self.h, mesh.h, o, d, n, t, prim))
        return t, prim

    def bounded_distance(self, mesh: "Mesh", points, pose, max_dist, reduce=A.REDUCE_ALL):
        """Executor::bounded_distance (executor/cpu.rs:84-113)."""
        p = _f64(points)
        out = np.empty(1 if reduce == A.REDUCE_MIN else len(p), np.float64)
        check(self.h, A.lib().sherd_bounded_distance(self.h, mesh.h, p, len(p), _pose(pose),
                                                    float(max_dist), int(reduce), out))
        return out

    def inside(self, mesh: "Mesh", points, pose):
        """Executor::inside (executor/cpu.rs:115-128): (depth f32, inside u32) per point."""
        p = _f64(points)
        out = (A.InsideOutcome * max(len(p), 1))()
        check(self.h, A.lib().sherd_inside(self.h, mesh.h, p, len(p), _pose(pose),
                                          C.cast(out, C.c_void_p)))
        arr = np.frombuffer(out, dtype=np.dtype([("depth", np.float32), ("inside", np.uint32)]),
                            count=len(p))
        return arr["depth"].copy(), arr["inside"].copy()

    def icp_rung(self, source, target: "Cloud", inits, distance, max_iteration=30,
                 estimation=A.POINT_TO_PLANE):
        """Executor::icp_rung (executor/cpu.rs:70-82): point-to-plane, or the stage-1
        point-to-point rung (estimation=POINT_TO_POINT)."""
        s = _f64(source)
        inits = _f64(inits, (-1, 16))
        out = (A.Registration * max(len(inits), 1))()
        opt = A.IcpOptions(int(estimation), int(max_iteration), float(distance))
        check(self.h, A.lib().sherd_icp_rung(self.h, ptr(s), len(s), target.h, inits, len(inits),
                                            opt, C.cast(out, C.c_void_p)))
        return list(out)[:len(inits)]

    def icp_rung_array(self, source, target: "Cloud", inits, distance, max_iteration=30,
                       estimation=A.POINT_TO_PLANE) -> np.ndarray:
        """icp_rung with its registrations as one REGISTRATION record array (no per-start
        Python objects): rec["transform"] is the (n, 16) row-major poses."""
        s = _f64(source)
        inits = _f64(inits, (-1, 16))
        out = np.zeros(max(len(inits), 1), REGISTRATION)
        opt = A.IcpOptions(int(estimation), int(max_iteration), float(distance))
        check(self.h, A.lib().sherd_icp_rung(self.h, ptr(s), len(s), target.h, inits, len(inits),
                                            opt, out.ctypes.data_as(C.c_void_p)))
        return out[:len(inits)]

    # -- preprocessing rays ---------------------------------------------------------------------
    def face_geometry(self, v, f):
        """mesh::geometry::face_geometry (mesh/geometry.rs:70-96): normals, areas, centroids."""
        v, f = _f64(v), _u32(f, (-1, 3))
        nf = len(f)
        n = np.empty((nf, 3))
        a = np.empty(nf)
        c = np.empty((nf, 3))
        check(self.h, A.lib().sherd_face_geometry(self.h, v, len(v), f, nf, ptr(n), ptr(a), ptr(c)))
        return n, a, c

    def thickness(self, mesh: "Mesh", centroids, normals, max_rays=300_000, return_hits=False):
        """R 3.2 (fragment/thickness.rs:99-162): (t, thick_mode) or None when < 100 rays hit."""
        cen, nrm = _f64(centroids), _f64(normals)
        nf = len(nrm)
        stride = max(1, -(-nf // max(max_rays, 1)))
        n = -(-nf // stride)
        t, m, found = C.c_float(), C.c_float(), C.c_uint32()
        th = np.empty(n, np.float32) if return_hits else None
        pr = np.empty(n, np.uint32) if return_hits else None
        check(self.h, A.lib().sherd_thickness(self.h, mesh.h, cen, nrm, nf, int(max_rays),
                                             C.byref(t), C.byref(m), C.byref(found), ptr(th),
                                             ptr(pr)))
        res = (np.float32(t.value), np.float32(m.value)) if found.value else None
        return (res, th, pr) if return_hits else res

    def thickness_from_hits(self, normals, idx, t_hit, prim):
        """thickness_from_hits (fragment/thickness.rs:139-162) on the device."""
        nrm = _f64(normals)
        t, m, found = C.c_float(), C.c_float(), C.c_uint32()
        idx, th, pr = _u32(idx), _f32(t_hit, (-1,)), _u32(prim)
        check(self.h, A.lib().sherd_thickness_from_hits(self.h, nrm, len(nrm), idx, th, pr,
                                                       len(idx), C.byref(t), C.byref(m),
                                                       C.byref(found)))
        return (np.float32(t.value), np.float32(m.value)) if found.value else None

    def cone_votes(self, mesh: "Mesh", centroids, normals, ns, hit_normals, thick):
        """R 3.4.3's seven-ray cone vote per face (fragment/segment.rs:318-376)."""
        nf = len(normals)
        good = np.empty(nf, np.uint8)
        check(self.h, A.lib().sherd_cone_votes(self.h, mesh.h, _f64(centroids), _f64(normals),
                                              _f64(ns), _f64(hit_normals), nf, float(thick), good))
        return good

    # -- verification and the batched stage-2 path ---------------------------------------------
    def surfaces(self, fracture: "Mesh", mesh: "Mesh | None", watertight, frac_area, pf, s,
                 brk_p, brk_ns, margin_p, margin_n) -> "Surfaces":
        return Surfaces(self, fracture, mesh, watertight, frac_area, pf, s, brk_p, brk_ns,
                        margin_p, margin_n)

    def verify(self, a: "Surfaces", b: "Surfaces", pose, scales: A.Scales, full=True) -> A.Scores:
        """verify::verify (matching/verify.rs:590-626) on the device."""
        out = A.Scores()
        check(self.h, A.lib().sherd_verify(self.h, a.h, b.h, _pose(pose), C.byref(scales),
                                          int(full), C.byref(out)))
        return out

    def pair(self, a: "Surfaces", b: "Surfaces", reg_target: "Cloud", frac_target: "Cloud",
             reg_source, frac_source, scales: A.Scales) -> "Pair":
        return Pair(self, a, b, reg_target, frac_target, reg_source, frac_source, scales)

    def batch(self, pairs, items, params: A.Params, sched=A.SCHED_BATCHED) -> "Batch":
        return Batch(self, pairs, items, params, sched)

    def ladder_verify_batch(self, pairs, items, params: A.Params, sched=A.SCHED_BATCHED,
                            out=None):
        """R 5.6 + R 6 + R 6.5 for every (pair, start); `items` is a ctypes WorkItem array, a
        WORK_ITEM numpy array, or a list of (pair, start, init 4x4) tuples. The candidates go
        into `out` when given (a CANDIDATE numpy array or ctypes Candidate array with room for
        every item, e.g. in pinned memory reused from call to call), else into a new ctypes
        Candidate array; either is returned."""
        if isinstance(items, np.ndarray):
            if items.dtype != WORK_ITEM or not items.flags.c_contiguous:
                raise A.SherdError(A.E_INVALID, "items must be a contiguous WORK_ITEM array")
            n_items, items_ptr = len(items), items.ctypes.data_as(C.c_void_p)
        else:
            if not isinstance(items, C.Array):
                items = work_items(items)
            n_items, items_ptr = len(items), C.cast(items, C.c_void_p)
        if out is None:
            out = (A.Candidate * max(n_items, 1))()
            out_ptr = C.cast(out, C.c_void_p)
        elif isinstance(out, np.ndarray):
            if out.dtype != CANDIDATE or not out.flags.c_contiguous or not out.flags.writeable \
                    or len(out) < n_items:
                raise A.SherdError(A.E_INVALID, "out must be a writable contiguous CANDIDATE "
                                                "array with room for every item")
            out_ptr = out.ctypes.data_as(C.c_void_p)
        else:
            if len(out) < n_items:
                raise A.SherdError(A.E_INVALID, "out has no room for every item")
            out_ptr = C.cast(out, C.c_void_p)
        arr = (C.c_void_p * max(len(pairs), 1))(*[p.h for p in pairs])
        check(self.h, A.lib().sherd_ladder_verify_batch(self.h, arr, len(pairs), items_ptr,
                                                       n_items, C.byref(params), int(sched),
                                                       out_ptr))
        return out

    def penetration_share(self, mesh: "Mesh", points, pose, pen) -> float:
        """verify::penetration_share (verify.rs:509-527), R 8's assembly question: the share
        of `points` moved by `pose` inside `mesh` deeper than `pen`."""
        p = _f64(points)
        out = C.c_double(0.0)
        check(self.h, A.lib().sherd_penetration_share(self.h, mesh.h, p, len(p), _pose(pose),
                                                      float(pen), C.byref(out)))
        return out.value

    # -- the coarse breakline score -----------------------------------------------------------
    def coarse_scores(self, target: "Cloud", points, normals, poses, radius, normal_agree=0.7):
        """Executor::coarse_scores (executor/cpu.rs:46-68, 136-169): per 4x4 pose the fraction
        of `points` whose nearest `target` point (A's breakline, with normals) is strictly
        within `radius` and whose turned normal agrees with it (dot > normal_agree)."""
        p, n = _f64(points), _f64(normals)
        t = _f64(poses, (-1, 16))
        out = np.empty(len(t))
        check(self.h, A.lib().sherd_coarse_scores(self.h, target.h, p, n, len(p), t, len(t),
                                                  float(radius), float(normal_agree), out))
        return out

    # -- segmentation ---------------------------------------------------------------------------
    def segment(self, mesh: "Mesh", v, f, thick, res, params: A.SegParams | None = None,
                trace=False):
        """segment::segment_faces (fragment/segment.rs:476-631): shell (0) / fracture (1)
        labels of the working mesh (v f64, f) whose ray scene is `mesh`, with R 3.2's wall
        `thick` and the median edge `res`. Returns (labels, SegInfo) or, with trace=True,
        (labels, SegInfo, dict of every intermediate array)."""
        v = _f64(v)
        f = _u32(f, (-1, 3))
        nf = len(f)
        labels = np.zeros(nf, np.uint8)
        info = A.SegInfo()
        tr = None
        if trace:
            tr = {"rep": np.zeros(nf, np.uint32), "near": np.zeros(nf, np.uint32),
                  "ns": np.zeros((nf, 3)), "good": np.zeros(nf, np.uint8),
                  "frac_raw": np.zeros(nf, np.uint8), "frac_majority": np.zeros(nf, np.uint8),
                  "frac_islands": np.zeros(nf, np.uint8), "has_ref": np.zeros(nf, np.uint8)}
            ct = A.SegTrace(*[a.ctypes.data for a in tr.values()])
        check(self.h, A.lib().sherd_segment(self.h, mesh.h, v, len(v), f, nf, float(thick),
                                            float(res), C.byref(params) if params else None,
                                            labels, C.byref(info),
                                            C.byref(ct) if trace else None))
        if not trace:
            return labels, info
        tr["rep"] = tr["rep"][:info.n_rep]
        return labels, info, tr

    # -- differentiation ------------------------------------------------------------------------
    def adjoint(self, edges, poses, inverses, opts: A.AdjointOptions):
        """The group-alignment objectives of every (pose, edge): `poses` and `inverses` are
        (P, E, 4, 4) arrays of T (B's frame into A's) and T^-1 for the E pairs in `edges`.
        Returns values (P, E, 5) = E, T_B, F_B, T_A, F_A and their twist gradients (P, E, 5, 6):
        the first three in A's frame (T -> exp(xi^) T), the last two in B's (T^-1 ->
        exp(xi^) T^-1)."""
        n_e = len(edges)
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, n_e, 16)
        inverses = np.ascontiguousarray(inverses, np.float64).reshape(-1, n_e, 16)
        if poses.shape != inverses.shape:
            raise A.SherdError(A.E_INVALID, "poses and inverses differ in shape")
        n_p = poses.shape[0]
        values = np.empty((n_p, n_e, A.ADJOINT_VALUES))
        grads = np.empty((n_p, n_e, A.ADJOINT_VALUES, 6))
        arr = (C.c_void_p * max(n_e, 1))(*[e.h for e in edges])
        check(self.h, A.lib().sherd_adjoint(self.h, arr, n_e, poses, inverses, n_p, C.byref(opts),
                                            values, grads))
        return values, grads

    # -- R 3.5 -----------------------------------------------------------------------------------
    def breaklines(self, v, f, frac, t, macro_inner=0.15, macro_outer=0.60, brk_voxel=0.5):
        """breakline::build (breakline.rs:207-300) on the device: a dict of p, ns, nf, f (n, 3),
        dih (n,), valid (n,) bool and sub (ascending)."""
        v, f = _f64(v), _u32(f, (-1, 3))
        frac = np.ascontiguousarray(np.asarray(frac).astype(bool), np.uint8).reshape(-1)
        if len(frac) != len(f):
            raise A.SherdError(A.E_INVALID, "one label per face")
        args = (self.h, v, len(v), f, len(f), frac, float(t), float(macro_inner),
                float(macro_outer), float(brk_voxel))
        count, n_sub = C.c_uint32(0), C.c_uint32(0)
        check(self.h, A.lib().sherd_breaklines(*args, 0, None, None, None, None, None, None,
                                               None, C.byref(n_sub), C.byref(count)))
        n = count.value
        out = {"p": np.zeros((n, 3)), "ns": np.zeros((n, 3)), "nf": np.zeros((n, 3)),
               "f": np.zeros((n, 3)), "dih": np.zeros(n), "valid": np.zeros(n, np.uint8),
               "sub": np.zeros(max(n, 1), np.uint32)}
        if n:
            check(self.h, A.lib().sherd_breaklines(
                *args, n, ptr(out["p"]), ptr(out["ns"]), ptr(out["nf"]), ptr(out["f"]),
                ptr(out["dih"]), ptr(out["valid"]), ptr(out["sub"]), C.byref(n_sub),
                C.byref(count)))
        out["sub"] = out["sub"][:n_sub.value].copy()
        out["valid"] = out["valid"].astype(bool)
        return out

    # -- stage 1 ---------------------------------------------------------------------------------
    def hypotheses_coarse(self, frames_a, frames_b, ia, ib, dihedral_tol, target: "Cloud", q, qn,
                          delta, normal_agree=0.7):
        """R 5.1 + R 5.2 (hypotheses.rs:149-211, coarse.rs:113-133) on the device:
        (pa, pb, poses (n, 4, 4), scores) of every complementary (ia[i], ib[j]) frame pair, in
        row-major (i, j) order. `frames_*` have p, ns, f (n, 3) and dih (n,) as f64 arrays."""
        ia, ib = _u32(ia), _u32(ib)
        q, qn = _f64(q), _f64(qn)
        fa, fb = _frames(frames_a), _frames(frames_b)
        count = C.c_uint32(0)
        grid = len(ia) * len(ib)
        if grid <= HYP_ONE_CALL:
            # Room for every (i, j): one call, the outputs cut to the count.
            pa, pb = np.empty(grid, np.uint32), np.empty(grid, np.uint32)
            poses, scores = np.empty((grid, 4, 4)), np.empty(grid)
            if grid:
                check(self.h, A.lib().sherd_hypotheses_coarse(
                    self.h, C.byref(fa[0]), C.byref(fb[0]), ia, len(ia), ib, len(ib),
                    float(dihedral_tol), target.h, q, qn, len(q), float(delta),
                    float(normal_agree), grid, ptr(pa), ptr(pb), ptr(poses), ptr(scores),
                    C.byref(count)))
            n = count.value
            return pa[:n].copy(), pb[:n].copy(), poses[:n].copy(), scores[:n].copy()
        check(self.h, A.lib().sherd_hypotheses_coarse(
            self.h, C.byref(fa[0]), C.byref(fb[0]), ia, len(ia), ib, len(ib), float(dihedral_tol),
            target.h, q, qn, len(q), float(delta), float(normal_agree), 0, None, None, None, None,
            C.byref(count)))
        n = count.value
        pa, pb = np.empty(n, np.uint32), np.empty(n, np.uint32)
        poses, scores = np.empty((n, 4, 4)), np.empty(n)
        if n:
            check(self.h, A.lib().sherd_hypotheses_coarse(
                self.h, C.byref(fa[0]), C.byref(fb[0]), ia, len(ia), ib, len(ib),
                float(dihedral_tol), target.h, q, qn, len(q), float(delta), float(normal_agree),
                n, ptr(pa), ptr(pb), ptr(poses), ptr(scores), C.byref(count)))
        return pa, pb, poses, scores

    # -- R 9 join refinement ----------------------------------------------------------------------
    def vertex_normals(self, v, f):
        """refine::vertex_normals (refine.rs:121-151), bit-identical: (nv, 3) f64."""
        v, f = _f64(v), _u32(f, (-1, 3))
        out = np.empty((len(v), 3))
        check(self.h, A.lib().sherd_vertex_normals(self.h, v, len(v), f, len(f), out))
        return out

    def fracture_cloud(self, v, f, centroids, fracture, radius):
        """refine::fracture_cloud (refine.rs:217-227) before the cap, in one device call: the
        selected vertex indices (ascending), their points and their vertex normals."""
        v, f = _f64(v), _u32(f, (-1, 3))
        cen = _f64(centroids)
        frac = np.ascontiguousarray(np.asarray(fracture).astype(bool).reshape(-1), np.uint8)
        if len(cen) != len(frac):
            raise A.SherdError(A.E_INVALID, "one fracture label per centroid")
        nv = len(v)
        idx = np.empty(max(nv, 1), np.uint32)
        pts = np.empty((max(nv, 1), 3))
        nrm = np.empty((max(nv, 1), 3))
        n = C.c_uint32(0)
        check(self.h, A.lib().sherd_fracture_cloud(self.h, v, nv, f, len(f), cen, frac, len(cen),
                                                   float(radius), nv, idx, pts, nrm,
                                                   C.byref(n)))
        m = int(n.value)
        return idx[:m].copy(), pts[:m].copy(), nrm[:m].copy()

    def refine_join(self, source, target, target_normals, pose_fixed, pose_moving, dist,
                    max_iteration=40):
        """refine_one's two point-to-plane rungs (refine.rs:334-386) for one join, the clouds
        placed by their fragments' poses on the device: [rung 1, rung 2] Registrations."""
        s = _f64(source)
        t, n = _f64(target), _f64(target_normals)
        if t.shape != n.shape:
            raise A.SherdError(A.E_INVALID, "target points and normals differ in shape")
        d = np.ascontiguousarray(dist, np.float64).reshape(2)
        out = (A.Registration * 2)()
        check(self.h, A.lib().sherd_refine_join(self.h, s, len(s), t, n, len(t), _pose(pose_fixed),
                                                _pose(pose_moving), d, int(max_iteration),
                                                C.cast(out, C.c_void_p)))
        return list(out)


# Up to this many (i, j) frame pairs, hypotheses_coarse makes one call with room for all of
# them (128 B of poses each); above it, a counting call first.
HYP_ONE_CALL = 1 << 20

WORK_ITEM = np.dtype(A.WorkItem)
CANDIDATE = np.dtype(A.Candidate)
REGISTRATION = np.dtype(A.Registration)


def work_items(items) -> C.Array:
    """(pair index, start id, 4x4 init) tuples as the C ABI's work-item array."""
    pair = np.array([int(p) for p, _, _ in items], np.uint32)
    start = np.array([int(s) for _, s, _ in items], np.uint32)
    inits = np.array([_pose(t) for _, _, t in items], np.float64).reshape(-1, 16)
    return work_item_array(pair, start, inits)


def work_item_array(pair, start, inits) -> C.Array:
    """The work-item array from three aligned numpy arrays (vectorised)."""
    n = len(pair)
    arr = (A.WorkItem * max(n, 1))()
    view = np.ctypeslib.as_array(arr)[:n]
    view["pair"] = pair
    view["start"] = start
    view["init"] = np.asarray(inits, np.float64).reshape(n, 16)
    return arr


def candidates(arr) -> np.ndarray:
    """A structured numpy view of a Candidate array (fields as in sherd_candidate)."""
    return np.ctypeslib.as_array(arr)


class Batch(_Handle):
    """A device-resident stage-2 batch (sherd_batch_*): upload once, run many times."""
    _free = "sherd_batch_free"

    def __init__(self, ctx: Context, pairs, items, params: A.Params, sched=A.SCHED_BATCHED):
        self.ctx = ctx
        self.keep = list(pairs)
        if not isinstance(items, C.Array):
            items = work_items(items)
        self.n = len(items)
        arr = (C.c_void_p * max(len(pairs), 1))(*[p.h for p in pairs])
        h = C.c_void_p()
        check(ctx.h, A.lib().sherd_batch_create(ctx.h, arr, len(pairs), C.cast(items, C.c_void_p),
                                               self.n, C.byref(params), int(sched), C.byref(h)))
        self.h = h

    STAGES = ("ladder", "verify", "pen_inside", "pen_min", "finalize", "total")

    def run(self) -> dict:
        """Runs the batch; returns the device milliseconds of each stage and of the run."""
        ms = np.zeros(len(self.STAGES), np.float32)
        check(self.ctx.h, A.lib().sherd_batch_run(self.h, ms))
        return {k: float(x) for k, x in zip(self.STAGES, ms)}

    def results(self):
        out = (A.Candidate * self.n)()
        check(self.ctx.h, A.lib().sherd_batch_results(self.h, C.cast(out, C.c_void_p)))
        return out


class Mesh(_Handle):
    """A device triangle LBVH (RayScene::of_mesh, spatial/bvh.rs:56-62)."""
    _free = "sherd_mesh_free"

    def __init__(self, ctx: Context, v, f, _handle=None):
        self.ctx = ctx
        if _handle is not None:
            self.h = _handle
            return
        v, f = _f32(v), _u32(f, (-1, 3))
        h = C.c_void_p()
        check(ctx.h, A.lib().sherd_mesh_upload(ctx.h, v, len(v), f, len(f), C.byref(h)))
        self.h = h

    def subset(self, keep) -> "Mesh":
        """RayScene::of_subset (spatial/bvh.rs:71-78)."""
        keep = np.ascontiguousarray(keep, dtype=np.uint8)
        h = C.c_void_p()
        check(self.ctx.h, A.lib().sherd_mesh_subset(self.ctx.h, self.h, keep, C.byref(h)))
        return Mesh(self.ctx, None, None, _handle=h)

    @property
    def n_faces(self) -> int:
        return int(A.lib().sherd_mesh_faces(self.h))

    def aabb(self):
        lo, hi = np.empty(3, np.float32), np.empty(3, np.float32)
        A.lib().sherd_mesh_aabb(self.h, lo, hi)
        return lo, hi


class Cloud(_Handle):
    """A device point LBVH with optional normals (PointTree / IcpTarget)."""
    _free = "sherd_cloud_free"

    def __init__(self, ctx: Context, p, n=None):
        self.ctx = ctx
        p = _f64(p)
        nn = None if n is None else _f64(n)
        h = C.c_void_p()
        check(ctx.h, A.lib().sherd_cloud_upload(ctx.h, p, ptr(nn), len(p), C.byref(h)))
        self.h = h
        self.n = len(p)

    def nearest_within_sq(self, queries, r2):
        """PointTree::nearest_within_squared (spatial/kdtree.rs:202-217)."""
        q = _f64(queries)
        idx = np.empty(len(q), np.uint32)
        d2 = np.empty(len(q), np.float64)
        check(self.ctx.h, A.lib().sherd_nearest_within_sq(self.ctx.h, self.h, q, len(q),
                                                         float(r2), idx, d2))
        return idx, d2

    def nearest_below(self, queries, bound):
        """PointTree::nearest_below (spatial/kdtree.rs:182-190)."""
        q = _f64(queries)
        idx = np.empty(len(q), np.uint32)
        d = np.empty(len(q), np.float64)
        check(self.ctx.h, A.lib().sherd_nearest_below(self.ctx.h, self.h, q, len(q), float(bound),
                                                     idx, d))
        return idx, d


class Surfaces(_Handle):
    """verify::Surfaces (matching/verify.rs:223-299) on the device."""
    _free = "sherd_surfaces_free"

    def __init__(self, ctx, fracture, mesh, watertight, frac_area, pf, s, brk_p, brk_ns, margin_p,
                 margin_n):
        self.ctx = ctx
        self.keep = (fracture, mesh)
        arrs = [_f64(x) for x in (pf, s, brk_p, brk_ns, margin_p, margin_n)]
        pf, s, bp, bn, mp, mn = arrs
        h = C.c_void_p()
        check(ctx.h, A.lib().sherd_surfaces_create(
            ctx.h, fracture.h, mesh.h if mesh is not None else None, int(bool(watertight)),
            float(frac_area), ptr(pf), len(pf), ptr(s), len(s), ptr(bp), ptr(bn), len(bp),
            ptr(mp), ptr(mn), len(mp), C.byref(h)))
        self.h = h


class Pair(_Handle):
    """One pair of the batched stage-2 path (matching/pair.rs:298-372, 592-630)."""
    _free = "sherd_pair_free"

    def __init__(self, ctx, a, b, reg_target, frac_target, reg_source, frac_source, scales):
        self.ctx = ctx
        self.keep = (a, b, reg_target, frac_target)
        rs, fs = _f64(reg_source), _f64(frac_source)
        self.scales = scales
        self.n_reg, self.n_frac = len(rs), len(fs)
        h = C.c_void_p()
        check(ctx.h, A.lib().sherd_pair_create(ctx.h, a.h, b.h, reg_target.h, frac_target.h,
                                              ptr(rs), len(rs), ptr(fs), len(fs),
                                              C.byref(scales), C.byref(h)))
        self.h = h


# ---------------------------------------------------------------------------------------------
# The reference's Executor trait (executor/mod.rs:105-137), over this backend
# ---------------------------------------------------------------------------------------------

@dataclass
class IcpBatch:
    """IcpBatch (executor/batch.rs:218-228)."""
    source: np.ndarray
    target: Cloud
    inits: np.ndarray
    max_correspondence_distance: float
    max_iteration: int = 30
    estimation: int = A.POINT_TO_PLANE


@dataclass
class CoarseBatch:
    """CoarseBatch (executor/batch.rs:152-177), with Poses::Homogeneous 4x4 poses (a Split batch
    stacks its rotations and translations into 4x4s). `target` is a Cloud over A's breakline
    with its shell normals; the reference's NearMask moves no score and is not carried."""
    target: Cloud
    points: np.ndarray
    normals: np.ndarray
    poses: np.ndarray
    radius: float
    normal_agree: float = 0.7


@dataclass
class DistBatch:
    """DistBatch (executor/batch.rs:283-296)."""
    points: np.ndarray
    transform: np.ndarray
    scene: Mesh
    max_dist: float
    reduce: int = A.REDUCE_ALL


@dataclass
class InsideBatch:
    """InsideBatch (executor/batch.rs:314-323)."""
    points: np.ndarray
    transform: np.ndarray
    scene: Mesh


class CudaExecutor:
    """`impl Executor for CudaExecutor`: every method of the trait, answered on the device
    only. Errors raise `SherdError`: there is no silent CPU fallback.
    """

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def name(self) -> str:
        return self.ctx.name

    def coarse_scores(self, batch: CoarseBatch) -> np.ndarray:
        return self.ctx.coarse_scores(batch.target, batch.points, batch.normals, batch.poses,
                                      batch.radius, batch.normal_agree)

    def icp_rung(self, batch: IcpBatch):
        return self.ctx.icp_rung(batch.source, batch.target, batch.inits,
                                 batch.max_correspondence_distance, batch.max_iteration,
                                 batch.estimation)

    def bounded_distance(self, batch: DistBatch) -> np.ndarray:
        return self.ctx.bounded_distance(batch.scene, batch.points, batch.transform,
                                         batch.max_dist, batch.reduce)

    def inside(self, batch: InsideBatch):
        return self.ctx.inside(batch.scene, batch.points, batch.transform)

    def device_slack(self) -> int:
        return self.ctx.device_slack()
