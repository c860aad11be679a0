"""ctypes view of the oracle (oracle.cpp), the CPU restatement of the reference's hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by bench.py's
CPU-baseline leg. The product package never imports it.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

_HERE = Path(__file__).resolve().parent
_lib = None

F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class IcpOptions(C.Structure):
    _fields_ = [("estimation", C.c_int32), ("max_iteration", C.c_int32),
                ("max_correspondence_distance", C.c_double)]


class Registration(C.Structure):
    _fields_ = [("transform", C.c_double * 16), ("fitness", C.c_double),
                ("inlier_rmse", C.c_double), ("correspondences", C.c_uint64),
                ("iterations", C.c_uint32), ("converged", C.c_uint32)]


class Scales(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "t", "res", "coarse", "stage1", "tight", "facing", "gap", "seam", "near", "pen", "nms",
        "icp")]


class Params(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n",
        "coarse_delta", "stage1_delta", "tight_delta", "facing_delta", "seam_delta",
        "near_delta", "pen_delta", "nms_delta", "icp_delta",
        "coarse_res", "stage1_res", "tight_res", "facing_res", "gap_res", "seam_res",
        "near_res", "pen_res", "icp_res", "early_reject_tight")]


SCORE_FIELDS = ("tight_a", "tight_b", "tight", "gap_a", "gap_b", "gap", "contact_a",
                "contact_b", "contact", "seam", "gap_limit", "tight_delta", "cont", "cont_n",
                "pen", "pen_depth")


class Scores(C.Structure):
    _fields_ = [(k, C.c_double) for k in SCORE_FIELDS] + [
        ("pen_unavailable", C.c_uint32), ("partial", C.c_uint32),
        ("brk", C.c_double), ("brk_best", C.c_double)]


class WorkItem(C.Structure):
    _fields_ = [("pair", C.c_uint32), ("start", C.c_uint32), ("init", C.c_double * 16)]


class Candidate(C.Structure):
    _fields_ = [("pair", C.c_uint32), ("start", C.c_uint32), ("accepted", C.c_uint32),
                ("status", C.c_uint32), ("rungs", Registration * 4), ("scores", Scores)]


class AdjointOptions(C.Structure):
    _fields_ = [("radius_k", C.c_double), ("width_k", C.c_double), ("window_k", C.c_double)]


class SegParams(C.Structure):
    _fields_ = [("smooth_res", C.c_double), ("coarse_at", C.c_double),
                ("boundary_angle", C.c_double), ("votes", C.c_uint32),
                ("votes_coarse", C.c_uint32), ("smoothed_hit_normal", C.c_uint32),
                ("boundary_angle_auto", C.c_uint32)]


class SegInfo(C.Structure):
    _fields_ = [("votes", C.c_uint32), ("n_rep", C.c_uint32), ("smooth_radius", C.c_double),
                ("boundary_angle", C.c_double)]


class SegTrace(C.Structure):
    _fields_ = [("rep", C.c_void_p), ("near", C.c_void_p), ("ns", C.c_void_p),
                ("good", C.c_void_p), ("frac_raw", C.c_void_p), ("frac_majority", C.c_void_p),
                ("frac_islands", C.c_void_p), ("has_ref", C.c_void_p)]


class InsideOutcome(C.Structure):
    _fields_ = [("depth", C.c_float), ("inside", C.c_uint32)]


def lib() -> C.CDLL:
    """The loaded oracle, built first when its sources are newer than the library."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.OUT
    if (_HERE / "oracle.cpp").exists():
        path = _build.build()
    L = C.CDLL(str(path))
    vp = C.c_void_p
    sig = {
        "or_mesh_new": (vp, [F32P, C.c_uint32, U32P, C.c_uint32]),
        "or_mesh_subset": (vp, [vp, U8P]),
        "or_mesh_free": (None, [vp]),
        "or_mesh_aabb": (None, [vp, F32P, F32P]),
        "or_first_hit": (None, [vp, F32P, F32P, C.c_uint32, F32P, U32P, C.c_int]),
        "or_bounded_distance": (None, [vp, F64P, C.c_uint32, F64P, C.c_double, C.c_int, F64P]),
        "or_inside": (None, [vp, F64P, C.c_uint32, F64P, vp, C.c_int]),
        "or_crossings": (C.c_uint32, [vp, F32P, F32P]),
        "or_cloud_new": (vp, [F64P, vp, C.c_uint32]),
        "or_cloud_free": (None, [vp]),
        "or_nearest_within_sq": (None, [vp, F64P, C.c_uint32, C.c_double, U32P, F64P, C.c_int]),
        "or_nearest_below": (None, [vp, F64P, C.c_uint32, C.c_double, U32P, F64P, C.c_int]),
        "or_icp_rung": (None, [F64P, C.c_uint32, vp, F64P, C.c_uint32, IcpOptions, vp, C.c_int]),
        "or_surfaces_new": (vp, [vp, vp, C.c_uint32, C.c_double, F64P, C.c_uint32, F64P,
                                 C.c_uint32, F64P, F64P, C.c_uint32, F64P, F64P, C.c_uint32]),
        "or_surfaces_free": (None, [vp]),
        "or_verify": (None, [vp, vp, F64P, C.POINTER(Scales), C.c_int, C.POINTER(Scores)]),
        "or_accept": (C.c_uint32, [C.POINTER(Scores), C.POINTER(Params), C.POINTER(Scales)]),
        "or_pair_new": (vp, [vp, vp, vp, vp, F64P, C.c_uint32, F64P, C.c_uint32,
                             C.POINTER(Scales)]),
        "or_pair_free": (None, [vp]),
        "or_ladder_verify_batch": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32, C.POINTER(Params),
                                             C.c_int, vp]),
        "or_face_geometry": (None, [F64P, U32P, C.c_uint32, vp, vp, vp]),
        "or_face_indices": (C.c_uint32, [C.c_uint32, C.c_uint32, vp]),
        "or_cast_inward_rays": (None, [vp, F64P, F64P, U32P, C.c_uint32, F32P, U32P, C.c_int]),
        "or_thickness_from_hits": (C.c_int, [F64P, C.c_uint32, U32P, F32P, U32P, C.c_uint32,
                                             C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "or_percentile90": (C.c_float, [F32P, C.c_uint32]),
        "or_hist_mode": (C.c_float, [F32P, C.c_uint32]),
        "or_cone_votes": (None, [vp, F64P, F64P, F64P, F64P, C.c_uint32, C.c_double, U8P,
                                 C.c_int]),
        "or_eigen_pivots": (None, [F64P, I32P]),
        "or_solve_ldlt": (C.c_int, [F64P, F64P, F64P]),
        "or_pose_inverse": (None, [F64P, F64P]),
        "or_euler_zyx": (None, [C.c_double, C.c_double, C.c_double, F64P]),
        "or_tri_distance": (C.c_float, [F32P, F32P, F32P, F32P]),
        "or_moller_trumbore": (C.c_float, [F32P, F32P, F32P, F32P, F32P]),
        "or_default_threads": (C.c_int, []),
        "or_adjoint": (None, [vp, F64P, F64P, C.POINTER(AdjointOptions), C.c_int, I32P, F64P,
                              F64P]),
        "or_normal_equations": (None, [F64P, C.c_uint32, vp, F64P, C.c_double, F64P, F64P]),
        "or_coarse_scores": (None, [vp, F64P, F64P, C.c_uint32, F64P, C.c_uint32, C.c_double,
                                    C.c_double, F64P]),
        "or_svd_rotation": (None, [F64P, F64P]),
        "or_penetration_share": (C.c_double, [vp, F64P, C.c_uint32, F64P, C.c_double]),
        "or_segment": (None, [vp, F64P, U32P, C.c_uint32, C.c_double, C.c_double,
                              C.POINTER(SegParams), vp, U8P, C.POINTER(SegInfo),
                              C.POINTER(SegTrace)]),
        "or_vertex_normals": (None, [F64P, C.c_uint32, U32P, C.c_uint32, F64P]),
        "or_ball_normals": (None, [F64P, C.c_uint32, F64P, F64P, F64P, C.c_uint32, C.c_double,
                                   F64P, U8P]),
        "or_voxel_representatives": (C.c_uint32, [F64P, C.c_uint32, C.c_double, U32P]),
        "or_nms": (C.c_uint32, [U32P, C.c_uint32, F64P, F64P, C.c_double, C.c_uint32, C.c_double,
                                U32P]),
        "or_place_fused": (None, [F64P, C.c_uint32, F64P, C.c_int, F64P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


class Mesh:
    """RayScene over f32 vertices (spatial/bvh.rs:36-192)."""

    def __init__(self, v, f, _handle=None):
        self.v = f32(v).reshape(-1, 3)
        self.f = u32(f).reshape(-1, 3)
        self.h = _handle or lib().or_mesh_new(self.v, len(self.v), self.f, len(self.f))
        if not self.h:
            raise ValueError("a mesh needs at least one face")

    def subset(self, keep) -> "Mesh":
        keep = np.ascontiguousarray(keep, dtype=np.uint8)
        h = lib().or_mesh_subset(self.h, keep)
        m = Mesh.__new__(Mesh)
        m.v, m.f, m.h = self.v, self.f[keep.astype(bool)] if keep.any() else self.f[:1], h
        return m

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mesh_free(self.h)
            self.h = None

    def aabb(self):
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        lib().or_mesh_aabb(self.h, lo, hi)
        return lo, hi

    def first_hit(self, org, dirs, threads=0):
        org, dirs = f32(org).reshape(-1, 3), f32(dirs).reshape(-1, 3)
        n = len(org)
        t = np.empty(n, np.float32)
        prim = np.empty(n, np.uint32)
        lib().or_first_hit(self.h, org, dirs, n, t, prim, threads or lib().or_default_threads())
        return t, prim

    def bounded_distance(self, pts, pose, max_dist, reduce=0):
        pts = f64(pts).reshape(-1, 3)
        out = np.empty(1 if reduce else len(pts), np.float64)
        lib().or_bounded_distance(self.h, pts, len(pts), f64(pose).reshape(16), max_dist,
                                  reduce, out)
        return out

    def inside(self, pts, pose, threads=0):
        pts = f64(pts).reshape(-1, 3)
        out = (InsideOutcome * max(len(pts), 1))()
        lib().or_inside(self.h, pts, len(pts), f64(pose).reshape(16), C.cast(out, C.c_void_p),
                        threads or lib().or_default_threads())
        depth = np.array([o.depth for o in out[:len(pts)]], np.float32)
        inside = np.array([o.inside for o in out[:len(pts)]], np.uint32)
        return depth, inside


class Cloud:
    """PointTree over f64 points (spatial/kdtree.rs:31-258), with optional normals."""

    def __init__(self, p, n=None):
        self.p = f64(p).reshape(-1, 3)
        self.n = None if n is None else f64(n).reshape(-1, 3)
        nptr = None if self.n is None else self.n.ctypes.data_as(C.c_void_p)
        self.h = lib().or_cloud_new(self.p, nptr, len(self.p))
        if not self.h:
            raise ValueError("a cloud needs at least one point")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_cloud_free(self.h)
            self.h = None

    def nearest_within_sq(self, q, r2, threads=0):
        q = f64(q).reshape(-1, 3)
        idx = np.empty(len(q), np.uint32)
        d2 = np.empty(len(q), np.float64)
        lib().or_nearest_within_sq(self.h, q, len(q), r2, idx, d2,
                                   threads or lib().or_default_threads())
        return idx, d2

    def nearest_below(self, q, bound, threads=0):
        q = f64(q).reshape(-1, 3)
        idx = np.empty(len(q), np.uint32)
        d = np.empty(len(q), np.float64)
        lib().or_nearest_below(self.h, q, len(q), bound, idx, d,
                               threads or lib().or_default_threads())
        return idx, d


def icp_rung(source, target: Cloud, inits, distance, max_iteration=30, threads=0,
             point_to_point=False):
    """icp::register for every init (icp.rs:308-356): point-to-plane, or the stage-1
    point-to-point rung (umeyama, icp.rs:527-592) with point_to_point."""
    source = f64(source).reshape(-1, 3)
    inits = f64(inits).reshape(-1, 16)
    out = (Registration * len(inits))()
    opt = IcpOptions(0 if point_to_point else 1, max_iteration, distance)
    lib().or_icp_rung(source, len(source), target.h, inits, len(inits), opt,
                      C.cast(out, C.c_void_p), threads or lib().or_default_threads())
    return list(out)


class Surfaces:
    """verify::Surfaces (verify.rs:223-299)."""

    def __init__(self, fracture: Mesh, mesh: Mesh | None, watertight, frac_area, pf, s, brk_p,
                 brk_ns, margin_p, margin_n):
        self.keep = (fracture, mesh)
        self.arrays = [f64(x).reshape(-1, 3) for x in (pf, s, brk_p, brk_ns, margin_p, margin_n)]
        pf, s, bp, bn, mp, mn = self.arrays
        self.h = lib().or_surfaces_new(fracture.h, mesh.h if mesh else None, int(watertight),
                                       float(frac_area), pf, len(pf), s, len(s), bp, bn, len(bp),
                                       mp, mn, len(mp))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_surfaces_free(self.h)
            self.h = None


def verify(a: Surfaces, b: Surfaces, pose, scales: Scales, full=True) -> Scores:
    out = Scores()
    lib().or_verify(a.h, b.h, f64(pose).reshape(16), C.byref(scales), int(full), C.byref(out))
    return out


def accept(scores: Scores, params: Params, scales: Scales) -> bool:
    return bool(lib().or_accept(C.byref(scores), C.byref(params), C.byref(scales)))


class Pair:
    def __init__(self, a: Surfaces, b: Surfaces, reg_target: Cloud, frac_target: Cloud,
                 reg_source, frac_source, scales: Scales):
        self.keep = (a, b, reg_target, frac_target)
        self.rs = f64(reg_source).reshape(-1, 3)
        self.fs = f64(frac_source).reshape(-1, 3)
        self.scales = scales
        self.h = lib().or_pair_new(a.h, b.h, reg_target.h, frac_target.h, self.rs, len(self.rs),
                                   self.fs, len(self.fs), C.byref(scales))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_pair_free(self.h)
            self.h = None


def adjoint(pair: Pair, t, t_inv, opts: AdjointOptions, assign=None):
    """The group-alignment objectives of one pair at pose t (B into A) and t_inv: values (5,)
    = E, T_B, F_B, T_A, F_A and their twist gradients (5, 6). Returns (values, grads, assign);
    passing `assign` back holds the matches and faces fixed (for finite differences)."""
    a_pf = pair.keep[0].arrays[0]
    b_pf = pair.keep[1].arrays[0]
    n = len(pair.fs) + len(b_pf) + len(a_pf)
    frozen = assign is not None
    assign = np.ascontiguousarray(assign, np.int32) if frozen else np.empty(n, np.int32)
    assert len(assign) == n
    values = np.empty(5)
    grads = np.empty((5, 6))
    lib().or_adjoint(pair.h, f64(t).reshape(16), f64(t_inv).reshape(16), C.byref(opts),
                     int(frozen), assign, values, grads)
    return values, grads, assign


def coarse_scores(target: Cloud, points, normals, poses, radius, normal_agree=0.7):
    """CpuExecutor::coarse_scores (executor/cpu.rs:46-68,136-169) for 4x4 poses."""
    p, n = f64(points).reshape(-1, 3), f64(normals).reshape(-1, 3)
    t = f64(poses).reshape(-1, 16)
    out = np.empty(len(t))
    lib().or_coarse_scores(target.h, p, n, len(p), t, len(t), float(radius), float(normal_agree),
                           out)
    return out


def penetration_share(mesh: Mesh, points, pose, pen):
    """verify::penetration_share (verify.rs:509-527)."""
    p = f64(points).reshape(-1, 3)
    return lib().or_penetration_share(mesh.h, p, len(p), f64(pose).reshape(16), float(pen))


def svd_rotation(m):
    """The rotation U diag(1, 1, det U det V) V^T of a 3x3's SVD (umeyama's, icp.rs:585-590)."""
    r = np.empty(9)
    lib().or_svd_rotation(f64(m).reshape(9), r)
    return r.reshape(3, 3)


def seg_params(**kw) -> SegParams:
    """SegParams::default (segment.rs:107-118), with keyword overrides."""
    p = SegParams(smooth_res=0.0, coarse_at=0.1, boundary_angle=25.0, votes=5, votes_coarse=4,
                  smoothed_hit_normal=0, boundary_angle_auto=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def segment(mesh: Mesh, v, f, thick, res, params: SegParams | None = None, good=None):
    """segment::segment_faces (segment.rs:476-631) on the working mesh (v f64, f) whose ray
    scene is `mesh`. `good` (optional votes per face) replaces the cone vote. Returns
    (labels (nf,) u8, SegInfo, trace dict of every intermediate array)."""
    v = f64(v).reshape(-1, 3)
    f = u32(f).reshape(-1, 3)
    nf = len(f)
    params = params or seg_params()
    tr = {"rep": np.zeros(nf, np.uint32), "near": np.zeros(nf, np.uint32),
          "ns": np.zeros((nf, 3)), "good": np.zeros(nf, np.uint8),
          "frac_raw": np.zeros(nf, np.uint8), "frac_majority": np.zeros(nf, np.uint8),
          "frac_islands": np.zeros(nf, np.uint8), "has_ref": np.zeros(nf, np.uint8)}
    trace = SegTrace(*[a.ctypes.data for a in tr.values()])
    labels = np.zeros(nf, np.uint8)
    info = SegInfo()
    g = None if good is None else np.ascontiguousarray(good, np.uint8)
    lib().or_segment(mesh.h, v, f, nf, float(thick), float(res), C.byref(params),
                     None if g is None else g.ctypes.data, labels, C.byref(info),
                     C.byref(trace))
    tr["rep"] = tr["rep"][:info.n_rep]
    return labels, info, tr


def normal_equations(source, target: Cloud, pose, distance):
    """icp::correspondences + normal_equations at `pose`: (J^T J (6, 6), J^T r (6,))."""
    src = f64(source).reshape(-1, 3)
    jtj = np.empty((6, 6))
    jtr = np.empty(6)
    lib().or_normal_equations(src, len(src), target.h, f64(pose).reshape(16), float(distance),
                              jtj, jtr)
    return jtj, jtr


def ladder_verify_batch(pairs, items, params: Params, threads=0):
    """The CPU baseline of the batched stage-2 path: returns (candidates, threads used)."""
    arr = (C.c_void_p * len(pairs))(*[p.h for p in pairs])
    it = (WorkItem * len(items))(*items)
    out = (Candidate * len(items))()
    used = lib().or_ladder_verify_batch(arr, len(pairs), C.cast(it, C.c_void_p), len(items),
                                        C.byref(params), threads, C.cast(out, C.c_void_p))
    return list(out), used


def face_geometry(v, f):
    v = f64(v).reshape(-1, 3)
    f = u32(f).reshape(-1, 3)
    n = np.empty((len(f), 3))
    a = np.empty(len(f))
    c = np.empty((len(f), 3))
    lib().or_face_geometry(v, f, len(f), n.ctypes.data_as(C.c_void_p),
                           a.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p))
    return n, a, c


def face_indices(n_faces, n=300_000):
    k = lib().or_face_indices(n_faces, n, None)
    out = np.empty(k, np.uint32)
    lib().or_face_indices(n_faces, n, out.ctypes.data_as(C.c_void_p))
    return out


def cast_inward_rays(mesh: Mesh, centroids, normals, idx, threads=0):
    idx = u32(idx)
    t = np.empty(len(idx), np.float32)
    prim = np.empty(len(idx), np.uint32)
    lib().or_cast_inward_rays(mesh.h, f64(centroids), f64(normals), idx, len(idx), t, prim,
                              threads or lib().or_default_threads())
    return t, prim


def thickness_from_hits(normals, idx, t_hit, prim):
    normals = f64(normals).reshape(-1, 3)
    t = C.c_float()
    m = C.c_float()
    ok = lib().or_thickness_from_hits(normals, len(normals), u32(idx), f32(t_hit), u32(prim),
                                      len(idx), C.byref(t), C.byref(m))
    return (np.float32(t.value), np.float32(m.value)) if ok else None


def cone_votes(mesh: Mesh, centroids, normals, ns, hit_normals, thick, threads=0):
    nf = len(normals)
    good = np.empty(nf, np.uint8)
    lib().or_cone_votes(mesh.h, f64(centroids), f64(normals), f64(ns), f64(hit_normals), nf,
                        float(thick), good, threads or lib().or_default_threads())
    return good


def scales_array(s: Scales) -> np.ndarray:
    return np.array([getattr(s, k) for k, _ in Scales._fields_])


def scales_from(arr) -> Scales:
    return Scales(*[float(x) for x in arr])


def default_params() -> Params:
    """Params::default (params.rs:141-190), the fields this ABI reads."""
    return Params(min_tight=0.25, max_gap=0.03, max_pen=0.005, min_seam=3.0, min_cont_n=0.8,
                  coarse_delta=0.15, stage1_delta=0.06, tight_delta=0.01, facing_delta=0.3,
                  seam_delta=0.12, near_delta=0.5, pen_delta=0.06, nms_delta=0.5,
                  icp_delta=0.04, coarse_res=2.3, stage1_res=0.9, tight_res=0.15,
                  facing_res=1.0, gap_res=0.45, seam_res=1.8, near_res=4.0, pen_res=0.9,
                  icp_res=0.6, early_reject_tight=0.0)


def collection(wl, params=None):
    """The oracle's objects for a synthetic collection (the package's synth.Workload), built the
    way the CUDA backend's workload.to_device builds its own: returns (pairs, keepalive)."""
    params = params or default_params()
    keep = []
    surfaces, reg_t, frac_t = [], [], []
    for fr in wl.fragments:
        m = Mesh(fr.v, fr.f)
        fm = m.subset(fr.frac)
        s = Surfaces(fm, m, True, fr.frac_area, fr.pf, fr.s, fr.brk_p, fr.brk_ns, fr.margin_p,
                     fr.margin_n)
        keep += [m, fm]
        surfaces.append(s)
        reg_t.append(Cloud(fr.reg_p, fr.reg_n))
        frac_t.append(Cloud(fr.pf, fr.pf_n))
    pairs = []
    for p in wl.pairs:
        a, b = wl.fragments[p.a], wl.fragments[p.b]
        sc = scales_for(params, min(a.t, b.t), max(a.res, b.res))
        pairs.append(Pair(surfaces[p.a], surfaces[p.b], reg_t[p.a], frac_t[p.a], b.reg_p, b.pf, sc))
    return pairs, (keep, surfaces, reg_t, frac_t)


def scales_for(params: Params, t: float, res: float) -> Scales:
    """Scales::for_pair (matching/scales.rs:72-88)."""
    def f(k, m):
        return max(k * t, m * res)
    return Scales(t=t, res=res, coarse=f(params.coarse_delta, params.coarse_res),
                  stage1=f(params.stage1_delta, params.stage1_res),
                  tight=f(params.tight_delta, params.tight_res),
                  facing=f(params.facing_delta, params.facing_res),
                  gap=f(params.max_gap, params.gap_res), seam=f(params.seam_delta, params.seam_res),
                  near=f(params.near_delta, params.near_res), pen=f(params.pen_delta, params.pen_res),
                  nms=params.nms_delta * t,
                  icp=f(params.icp_delta, params.icp_res) / (params.icp_delta * t))


def work_items_from(pair, start, inits):
    """A WorkItem array from aligned numpy arrays."""
    n = len(pair)
    arr = (WorkItem * max(n, 1))()
    view = np.ctypeslib.as_array(arr)[:n]
    view["pair"] = pair
    view["start"] = start
    view["init"] = np.asarray(inits, np.float64).reshape(n, 16)
    return arr


def ladder_verify_items(pairs, items, params: Params, threads=0):
    """or_ladder_verify_batch over a prepared WorkItem array: (Candidate array, threads used)."""
    arr = (C.c_void_p * len(pairs))(*[p.h for p in pairs])
    out = (Candidate * len(items))()
    used = lib().or_ladder_verify_batch(arr, len(pairs), C.cast(items, C.c_void_p), len(items),
                                        C.byref(params), threads, C.cast(out, C.c_void_p))
    return out, used


# ---- R 9: full-resolution join refinement (refine.rs) ------------------------------------------

REFINE_MAX_POINTS = 150_000   # refine.rs:56
REFINE_CAP_SEED = 0           # refine.rs:64
REFINE_SELECT_T = 0.15        # refine.rs:66
REFINE_SELECT_RES = 1.5       # refine.rs:68
REFINE_RUNGS = (0.05, 0.02)   # refine.rs:70
REFINE_ITERATIONS = 40        # refine.rs:72
MISS = 0xFFFFFFFF


def vertex_normals(v, f):
    """refine::vertex_normals (refine.rs:121-151): face-order sums of the unnormalised face
    normals, normalised once, (0, 0, 1) where the sum is zero."""
    v = f64(v).reshape(-1, 3)
    f = u32(f).reshape(-1, 3)
    out = np.empty_like(v)
    lib().or_vertex_normals(v, len(v), f, len(f), out)
    return out


def place_fused(points, pose, rotate_only=False):
    """types::apply_transform_fused / rotate_fused (types.rs:202-214), row-major pose."""
    p = f64(points).reshape(-1, 3)
    out = np.empty_like(p)
    lib().or_place_fused(p, len(p), f64(pose).reshape(16), int(bool(rotate_only)), out)
    return out


def refine_radius(thick, res):
    """The acceptance radius of select_candidates (refine.rs:168)."""
    return max(REFINE_SELECT_T * float(thick), REFINE_SELECT_RES * float(res))


def select_candidates(v, centroids, fracture, thick, res):
    """refine::select_candidates (refine.rs:161-178): every vertex whose nearest working-mesh
    centroid is a fracture face at a distance below max(0.15 t, 1.5 res), ascending. The bounded
    search (kdtree.rs:182-190) finds the unbounded nearest whenever it passes that test."""
    v = f64(v).reshape(-1, 3)
    centroids = f64(centroids).reshape(-1, 3)
    if len(centroids) == 0 or len(v) == 0:
        return np.zeros(0, np.uint32)
    j, _ = Cloud(centroids).nearest_below(v, refine_radius(thick, res))
    frac = np.asarray(fracture).astype(bool)
    keep = j != MISS
    keep[keep] = frac[j[keep]]
    return np.nonzero(keep)[0].astype(np.uint32)


def cap_selection(idx, max_points=REFINE_MAX_POINTS, seed=REFINE_CAP_SEED):
    """refine::cap_selection (refine.rs:186-193). Above the cap this draws numpy's
    default_rng(seed).choice(idx, max_points, replace=False), the draw refine.rs:30-37 names;
    under it the selection comes back untouched."""
    idx = np.asarray(idx, np.uint32)
    if len(idx) > max_points:
        idx = np.random.default_rng(seed).choice(idx, max_points, replace=False).astype(np.uint32)
    return idx


class FractureCloud:
    """refine::FractureCloud (refine.rs:78-113): indices, points and normals in ICP order."""

    def __init__(self, idx, points, normals):
        self.idx = np.asarray(idx, np.uint32)
        self.points = f64(points).reshape(-1, 3)
        self.normals = f64(normals).reshape(-1, 3)


def cloud_from_indices(v, normals, idx):
    """refine::cloud_from_indices (refine.rs:208-214)."""
    idx = np.asarray(idx, np.int64)
    return FractureCloud(idx, f64(v).reshape(-1, 3)[idx], f64(normals).reshape(-1, 3)[idx])


class RefinePiece:
    """refine::RefinePiece (refine.rs:236-244): the fragment's thickness and res, and its cloud
    (None when it has none)."""

    def __init__(self, thick, res, cloud):
        self.thick, self.res, self.cloud = float(thick), float(res), cloud


class RefinedJoin:
    """refine::RefinedJoin (refine.rs:247-262)."""

    def __init__(self, fixed, moving, dist, rungs, fitness, rmse_t):
        self.fixed, self.moving = int(fixed), int(moving)
        self.dist, self.rungs = list(dist), [np.asarray(r, np.float64) for r in rungs]
        self.fitness, self.rmse_t = float(fitness), float(rmse_t)


def matmul4(a, b):
    """A 4x4 product summed k = 0..3 left to right, without fused multiply-adds."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return ((a[:, 0:1] * b[0] + a[:, 1:2] * b[1]) + a[:, 2:3] * b[2]) + a[:, 3:4] * b[3]


def refine_one(pieces, poses, fixed, moving, params: Params):
    """refine::refine_one (refine.rs:334-386): the moving cloud placed by its pose against the
    fixed one placed by its own (normals rotated), two point-to-plane rungs from the identity."""
    tp, sp = pieces[fixed], pieces[moving]
    if tp.cloud is None or sp.cloud is None:
        return None
    sc = scales_for(params, min(tp.thick, sp.thick), max(tp.res, sp.res))
    source = place_fused(sp.cloud.points, poses[moving])
    tpts = place_fused(tp.cloud.points, poses[fixed])
    tnrm = place_fused(tp.cloud.normals, poses[fixed], rotate_only=True)
    target = Cloud(tpts, tnrm) if len(tpts) and len(source) else None
    pose = np.eye(4)
    rungs, dist, last = [], [], None
    for k in REFINE_RUNGS:
        d = k * sc.t * sc.icp
        if target is None:   # an empty side: the rung keeps its start, with no correspondence
            last = Registration(transform=(C.c_double * 16)(*pose.reshape(16)))
        else:
            last = icp_rung(source, target, pose, d, REFINE_ITERATIONS)[0]
        pose = np.array(last.transform[:]).reshape(4, 4)
        rungs.append(pose)
        dist.append(d)
    return RefinedJoin(fixed, moving, dist, rungs, last.fitness, last.inlier_rmse / sc.t)


def refine_joins(pieces, poses, groups, used, params: Params | None = None, one=None):
    """refine::refine_joins (refine.rs:282-318): per group of two or more, starting from its first
    fragment, repeatedly the first join of `used` (in `used` order) with exactly one endpoint
    placed; the placed end is fixed and poses[moving] <- rung2 . poses[moving]. Returns
    (poses, joins). `one` replaces refine_one (same signature)."""
    params = params or default_params()
    one = one or refine_one
    out = [np.asarray(p, np.float64).reshape(4, 4).copy() for p in poses]
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
            join = one(pieces, out, fixed, moving, params)
            if join is not None:
                out[moving] = matmul4(join.rungs[1], out[moving])
                joins.append(join)
            done.append(moving)
    return out, joins


# ---- stage 1: R 5.1-5.5 (hypotheses.rs, coarse.rs, nms.rs, ladder.rs, pair.rs:150-238) ----------

STAGE1_RUNGS = (0.2, 0.08)   # ladder.rs:51
STAGE1_ITERATIONS = 20       # ladder.rs:53
STAGE1_FLOOR = 0.05          # ladder.rs:61
COARSE_ORDER_LIMIT = 5000    # pair.rs:50
COARSE_FLOOR = 0.1           # pair.rs:52
NMS_ROT_TOL = 2.9            # nms.rs:40


def tangents(ns, f):
    """Breaklines::tangents_f64 (breakline.rs:180-182, 361-363): ns x f in f64."""
    ns, f = f64(ns).reshape(-1, 3), f64(f).reshape(-1, 3)
    return np.stack([ns[:, 1] * f[:, 2] - ns[:, 2] * f[:, 1], ns[:, 2] * f[:, 0] - ns[:, 0] * f[:, 2],
                     ns[:, 0] * f[:, 1] - ns[:, 1] * f[:, 0]], axis=1)


def hypotheses(a, b, ia, ib, dihedral_tol=25.0):
    """hypotheses::build_with + poses (hypotheses.rs:149-211). `a`, `b` are dicts of f64 arrays
    p, ns, f, dih. Returns (pa, pb, poses (n, 4, 4)) in row-major (i, j) order."""
    ia, ib = np.asarray(ia, np.int64), np.asarray(ib, np.int64)
    ok = np.abs(a["dih"][ia][:, None] + b["dih"][ib][None, :] - 180.0) < dihedral_tol
    pa, pb = np.nonzero(ok)
    ka, kb = ia[pa], ib[pb]
    ta, tb = tangents(a["ns"], a["f"])[ka], tangents(b["ns"], b["f"])[kb]
    axa = (ta, a["ns"][ka], a["f"][ka])
    axb = (tb, b["ns"][kb], b["f"][kb])
    n = len(pa)
    poses = np.zeros((n, 4, 4))
    poses[:, 3, 3] = 1.0
    for i in range(3):
        for k in range(3):
            poses[:, i, k] = ((axa[0][:, i] * -axb[0][:, k] + axa[1][:, i] * axb[1][:, k])
                              + axa[2][:, i] * -axb[2][:, k])
    pA, pB = a["p"][ka], b["p"][kb]
    for i in range(3):
        poses[:, i, 3] = pA[:, i] - ((poses[:, i, 0] * pB[:, 0] + poses[:, i, 1] * pB[:, 1])
                                     + poses[:, i, 2] * pB[:, 2])
    return pa.astype(np.uint32), pb.astype(np.uint32), poses


def order_by_score(score, limit=None):
    """nms::order_by_score (nms.rs:46-59): descending, ties by ascending index."""
    score = np.asarray(score, np.float64)
    order = np.lexsort((np.arange(len(score)), -score))
    return order[:limit] if limit is not None else order


def nms(order, poses, score, trans_tol, topk, floor):
    """nms::nms (nms.rs:61-86) with trace(A^T B) summed as nms.rs:93-99 sums it (or_nms)."""
    order = u32(order)
    poses = f64(poses).reshape(-1, 16)
    score = f64(score).reshape(-1)
    kept = np.empty(max(len(order), 1), np.uint32)
    m = lib().or_nms(order, len(order), poses, score, float(trans_tol), int(topk), float(floor),
                     kept) if len(order) else 0
    return kept[:m].copy()


def stage1_ladder(source, target: Cloud, inits, scales: Scales):
    """ladder::climb_all over stage1_rungs (ladder.rs:105-140): two point-to-point rungs."""
    poses = np.asarray(inits, np.float64).reshape(-1, 4, 4)
    for k in STAGE1_RUNGS:
        regs = icp_rung(source, target, poses, k * scales.t * scales.icp, STAGE1_ITERATIONS,
                        point_to_point=True)
        poses = np.stack([np.array(r.transform[:]).reshape(4, 4) for r in regs])
    return poses


# ---- R 3.5: breaklines, frames and samples (breakline.rs, samples.rs) --------------------------

MACRO_INNER, MACRO_OUTER, BRK_VOXEL = 0.15, 0.60, 0.5   # breakline.rs:72-76
FRAME_FLOOR, VALID_MIN = 1e-9, 0.5                      # breakline.rs:78-80
MARGIN_INNER, MARGIN_OUTER = 0.12, 1.5                  # samples.rs:82-84


def _dot3(a, b):
    return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]


def _norm3(a):
    return np.sqrt(_dot3(a, a))


def face_adjacency_edges(f):
    """face_adjacency (adjacency.rs:43-51, 138-160): the face pairs (fa, fb) sharing an edge and
    the edge's two vertices (lo, hi), in ascending edge-key order (slot-major, stable)."""
    f = np.asarray(f, np.int64).reshape(-1, 3)
    nf = len(f)
    keys, ends = [], []
    for x, y in ((0, 1), (1, 2), (2, 0)):
        lo, hi = np.minimum(f[:, x], f[:, y]), np.maximum(f[:, x], f[:, y])
        keys.append(lo * (1 << 32) + hi)
        ends.append(np.stack([lo, hi], axis=1))
    keys, ends = np.concatenate(keys), np.concatenate(ends)
    order = np.argsort(keys, kind="stable")
    k = keys[order]
    w = np.flatnonzero(k[:-1] == k[1:])
    return order[w] % nf, order[w + 1] % nf, ends[order[w], 0], ends[order[w], 1]


def ball_normals(points, normals, areas, queries, radius):
    """ball_normals (segment.rs:267-296) of `queries` over `points`: (unit normals, non-empty)."""
    p, q = f64(points).reshape(-1, 3), f64(queries).reshape(-1, 3)
    out = np.zeros((len(q), 3))
    has = np.zeros(len(q), np.uint8)
    if len(p) and len(q):
        lib().or_ball_normals(p, len(p), f64(normals).reshape(-1, 3), f64(areas).reshape(-1), q,
                              len(q), float(radius), out, has)
    return out, has


def voxel_representatives(points, spacing):
    """voxel_representatives (segment.rs:217-259): the lowest index per voxel, ascending."""
    p = f64(points).reshape(-1, 3)
    out = np.empty(max(len(p), 1), np.uint32)
    k = lib().or_voxel_representatives(p, len(p), float(spacing), out) if len(p) else 0
    return out[:k].copy()


def breaklines(v, f, frac, t, macro_inner=MACRO_INNER, macro_outer=MACRO_OUTER,
               brk_voxel=BRK_VOXEL):
    """breakline::build (breakline.rs:207-300) in f64: the midpoints of the edges whose two faces
    differ in label, in adjacency order; the shell and fracture macro normals over the faces
    between macro_inner t and macro_outer t of each point (the whole macro_outer ball where the
    annulus is empty); f = nf - (nf.ns) ns normalised; the validity mask; the hypothesis subset
    (voxel representatives at brk_voxel t that are valid); and the dihedral in degrees
    (breakline.rs:189-195). Returns a dict of arrays."""
    v = f64(v).reshape(-1, 3)
    f = np.asarray(f, np.int64).reshape(-1, 3)
    frac = np.asarray(frac).astype(bool)
    normals, areas, cent = face_geometry(v, f)
    fa, fb, lo, hi = face_adjacency_edges(f)
    change = frac[fa] != frac[fb]
    a, b = v[lo[change]], v[hi[change]]
    p = 0.5 * (a + b)
    n = len(p)
    empty = {"p": p, "ns": np.zeros((n, 3)), "nf": np.zeros((n, 3)), "f": np.zeros((n, 3)),
             "valid": np.zeros(n, bool), "sub": np.zeros(0, np.uint32), "dih": np.zeros(n)}
    if n == 0:
        return empty
    inner, outer = macro_inner * t, macro_outer * t
    _, dist = Cloud(p).nearest_below(cent, inner)

    def macro(fracture):
        every = np.flatnonzero(frac == fracture)
        out = np.zeros((n, 3))
        if len(every) == 0:
            return out
        far = every[dist[every] >= inner]
        if len(far):
            out, _ = ball_normals(cent[far], normals[far], areas[far], p, outer)
        bad = np.flatnonzero(_norm3(out) < VALID_MIN)
        if len(bad):
            out[bad], _ = ball_normals(cent[every], normals[every], areas[every], p[bad], outer)
        return out

    ns, nf = macro(False), macro(True)
    d = _dot3(nf, ns)
    fr = nf - d[:, None] * ns
    fr = fr / np.maximum(_norm3(fr), FRAME_FLOOR)[:, None]
    t_ = np.stack([ns[:, 1] * fr[:, 2] - ns[:, 2] * fr[:, 1], ns[:, 2] * fr[:, 0] - ns[:, 0] * fr[:, 2],
                   ns[:, 0] * fr[:, 1] - ns[:, 1] * fr[:, 0]], axis=1)
    valid = (_norm3(ns) > VALID_MIN) & (_norm3(nf) > VALID_MIN) & (_norm3(t_) > VALID_MIN)
    rep = voxel_representatives(p, brk_voxel * t)
    sub = rep[valid[rep]]
    dih = np.degrees(np.arccos(np.clip(_dot3(ns, nf), -1.0, 1.0)))
    return {"p": p, "ns": ns, "nf": nf, "f": fr, "valid": valid, "sub": sub.astype(np.uint32),
            "dih": dih}


def sample_on_faces(rng, v, f, areas, faces, n):
    """samples::sample_on_faces (samples.rs:281-305) with numpy's generator: the face picks
    (searchsorted of the normalised cumulative areas, side right, n uniforms), then n uniforms
    for u and n for v, folded where u + v > 1. Returns (points, picks, u, v) (u, v unfolded)."""
    faces = np.asarray(faces, np.int64)
    if len(faces) == 0 or n == 0:
        return np.zeros((0, 3)), np.zeros(0, np.int64), np.zeros(0), np.zeros(0)
    w = areas[faces] / areas[faces].sum()
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    picks = faces[np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), len(faces) - 1)]
    u, vv = rng.random(n), rng.random(n)
    fold = u + vv > 1.0
    al, be = np.where(fold, 1.0 - u, u), np.where(fold, 1.0 - vv, vv)
    o, pu, pv = v[f[picks, 0]], v[f[picks, 1]], v[f[picks, 2]]
    pts = (o + al[:, None] * (pu - o)) + be[:, None] * (pv - o)
    return pts, picks, u, vv


def samples(v, f, frac, brk_points, t, seed=0, surface_points=20000, frac_per_t2=150.0,
            min_frac=5000, max_frac=12000, margin_points=6000):
    """samples::build (samples.rs:201-248) with the reference's one numpy stream per fragment
    (samples.rs:33-42): the surface samples, the fracture samples
    clip(150 A_frac / t^2, 5000, 12000), and the shell margin 0.12 t < d_brk < 1.5 t thinned to
    margin_points by choice(..., replace=False), sorted."""
    v = f64(v).reshape(-1, 3)
    f = np.asarray(f, np.int64).reshape(-1, 3)
    frac = np.asarray(frac).astype(bool)
    _, areas, _ = face_geometry(v, f)
    rng = np.random.default_rng(seed)
    s, sp, su, sv = sample_on_faces(rng, v, f, areas, np.arange(len(f)), surface_points)
    fr = np.flatnonzero(frac)
    raw = frac_per_t2 * areas[fr].sum() / (t * t)
    n_frac = min_frac if np.isnan(raw) else int(np.clip(raw, min_frac, max_frac))
    pf, fp, fu, fv = sample_on_faces(rng, v, f, areas, fr, n_frac)
    bp = f64(brk_points).reshape(-1, 3)
    if len(bp):
        _, d_brk = Cloud(bp).nearest_below(s, MARGIN_OUTER * t)
    else:
        d_brk = np.full(len(s), np.inf)
    margin = np.flatnonzero(~frac[sp] & (d_brk > MARGIN_INNER * t) & (d_brk < MARGIN_OUTER * t))
    if margin_points and len(margin) > margin_points:
        margin = np.sort(rng.choice(margin, margin_points, replace=False))
    return {"S": s, "sp": sp, "S_u": su, "S_v": sv, "Pf": pf, "fp": fp, "Pf_u": fu, "Pf_v": fv,
            "margin_idx": margin}
