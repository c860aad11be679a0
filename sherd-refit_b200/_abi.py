"""ctypes declarations of include/sherd_cuda.h, and the loader of the built library.

The library is `_lib/libsherd_cuda.so`, built in-tree by `build.py`. There is no fallback: if
the library is missing or cannot be loaded, importing the backend raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_lib" / "libsherd_cuda.so"

OK, E_INVALID, E_OOM, E_TIMEOUT, E_ABORTED, E_DEVICE, E_EMPTY = 0, -1, -2, -3, -4, -5, -6
REDUCE_ALL, REDUCE_MIN = 0, 1
POINT_TO_POINT, POINT_TO_PLANE = 0, 1
SCHED_BATCHED, SCHED_PLAIN = 0, 1
NOALLOC_CAPACITY = 1 << 20

F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
VP = C.c_void_p


class InsideOutcome(C.Structure):
    """InsideOutcome (executor/batch.rs:339-368), 8 bytes."""
    _fields_ = [("depth", C.c_float), ("inside", C.c_uint32)]


class IcpOptions(C.Structure):
    """Options (matching/icp.rs:139-152)."""
    _fields_ = [("estimation", C.c_int32), ("max_iteration", C.c_int32),
                ("max_correspondence_distance", C.c_double)]


class Registration(C.Structure):
    """Registration (matching/icp.rs:181-195); transform row-major."""
    _fields_ = [("transform", C.c_double * 16), ("fitness", C.c_double),
                ("inlier_rmse", C.c_double), ("correspondences", C.c_uint64),
                ("iterations", C.c_uint32), ("converged", C.c_uint32)]

    def pose(self) -> np.ndarray:
        return np.array(self.transform[:], dtype=np.float64).reshape(4, 4)


SCALE_FIELDS = ("t", "res", "coarse", "stage1", "tight", "facing", "gap", "seam", "near", "pen",
                "nms", "icp")


class Scales(C.Structure):
    """Scales (matching/scales.rs:28-56)."""
    _fields_ = [(k, C.c_double) for k in SCALE_FIELDS]


PARAM_FIELDS = ("min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n",
                "coarse_delta", "stage1_delta", "tight_delta", "facing_delta", "seam_delta",
                "near_delta", "pen_delta", "nms_delta", "icp_delta",
                "coarse_res", "stage1_res", "tight_res", "facing_res", "gap_res", "seam_res",
                "near_res", "pen_res", "icp_res", "early_reject_tight")


class Params(C.Structure):
    """The Params fields (params.rs:141-190) that R 1.2 and R 6.5 read."""
    _fields_ = [(k, C.c_double) for k in PARAM_FIELDS]


SCORE_FIELDS = ("tight_a", "tight_b", "tight", "gap_a", "gap_b", "gap", "contact_a", "contact_b",
                "contact", "seam", "gap_limit", "tight_delta", "cont", "cont_n", "pen",
                "pen_depth")


class Scores(C.Structure):
    """Scores (matching/verify.rs:72-135)."""
    _fields_ = [(k, C.c_double) for k in SCORE_FIELDS] + [
        ("pen_unavailable", C.c_uint32), ("partial", C.c_uint32),
        ("brk", C.c_double), ("brk_best", C.c_double)]

    def as_dict(self) -> dict:
        d = {k: float(getattr(self, k)) for k in SCORE_FIELDS + ("brk", "brk_best")}
        d["pen_unavailable"] = bool(self.pen_unavailable)
        d["partial"] = bool(self.partial)
        return d


class WorkItem(C.Structure):
    _fields_ = [("pair", C.c_uint32), ("start", C.c_uint32), ("init", C.c_double * 16)]


class Candidate(C.Structure):
    _fields_ = [("pair", C.c_uint32), ("start", C.c_uint32), ("accepted", C.c_uint32),
                ("status", C.c_uint32), ("rungs", Registration * 4), ("scores", Scores)]


class AdjointOptions(C.Structure):
    _fields_ = [("radius_k", C.c_double), ("width_k", C.c_double), ("window_k", C.c_double)]


ADJOINT_VALUES = 5


class SegParams(C.Structure):
    _fields_ = [("smooth_res", C.c_double), ("coarse_at", C.c_double),
                ("boundary_angle", C.c_double), ("votes", C.c_uint32),
                ("votes_coarse", C.c_uint32), ("smoothed_hit_normal", C.c_uint32),
                ("boundary_angle_auto", C.c_uint32)]


class SegInfo(C.Structure):
    _fields_ = [("votes", C.c_uint32), ("n_rep", C.c_uint32), ("smooth_radius", C.c_double),
                ("boundary_angle", C.c_double)]


class Frames(C.Structure):
    """sherd_frames: one fragment's breakline (p, ns, f: xyz f64; dih: degrees)."""
    _fields_ = [("p", C.c_void_p), ("ns", C.c_void_p), ("f", C.c_void_p), ("dih", C.c_void_p),
                ("n", C.c_uint32)]


class SegTrace(C.Structure):
    _fields_ = [("rep", C.c_void_p), ("near", C.c_void_p), ("ns", C.c_void_p),
                ("good", C.c_void_p), ("frac_raw", C.c_void_p), ("frac_majority", C.c_void_p),
                ("frac_islands", C.c_void_p), ("has_ref", C.c_void_p)]

_lib = None

_SIGNATURES = {
    "sherd_name": (C.c_char_p, []),
    "sherd_open": (C.c_int, [C.c_int, C.POINTER(VP)]),
    "sherd_close": (C.c_int, [VP]),
    "sherd_last_error": (C.c_char_p, [VP]),
    "sherd_set_timeout_ms": (C.c_int, [VP, C.c_uint32]),
    "sherd_abort": (C.c_int, [VP]),
    "sherd_stats_json": (C.c_int, [VP, C.c_char_p, C.c_size_t]),
    "sherd_device_slack": (C.c_uint32, [VP]),
    "sherd_mesh_upload": (C.c_int, [VP, F32P, C.c_uint32, U32P, C.c_uint32, C.POINTER(VP)]),
    "sherd_mesh_subset": (C.c_int, [VP, VP, U8P, C.POINTER(VP)]),
    "sherd_mesh_free": (C.c_int, [VP]),
    "sherd_mesh_aabb": (C.c_int, [VP, F32P, F32P]),
    "sherd_mesh_faces": (C.c_uint32, [VP]),
    "sherd_first_hit": (C.c_int, [VP, VP, F32P, F32P, C.c_uint32, F32P, U32P]),
    "sherd_bounded_distance": (C.c_int, [VP, VP, F64P, C.c_uint32, F64P, C.c_double, C.c_int,
                                         F64P]),
    "sherd_inside": (C.c_int, [VP, VP, F64P, C.c_uint32, F64P, VP]),
    "sherd_face_geometry": (C.c_int, [VP, F64P, C.c_uint32, U32P, C.c_uint32, VP, VP, VP]),
    "sherd_thickness": (C.c_int, [VP, VP, F64P, F64P, C.c_uint32, C.c_uint32,
                                  C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_uint32), VP, VP]),
    "sherd_thickness_from_hits": (C.c_int, [VP, F64P, C.c_uint32, U32P, F32P, U32P, C.c_uint32,
                                            C.POINTER(C.c_float), C.POINTER(C.c_float),
                                            C.POINTER(C.c_uint32)]),
    "sherd_cone_votes": (C.c_int, [VP, VP, F64P, F64P, F64P, F64P, C.c_uint32, C.c_double, U8P]),
    "sherd_cloud_upload": (C.c_int, [VP, F64P, VP, C.c_uint32, C.POINTER(VP)]),
    "sherd_cloud_free": (C.c_int, [VP]),
    "sherd_cloud_points": (C.c_uint32, [VP]),
    "sherd_nearest_within_sq": (C.c_int, [VP, VP, F64P, C.c_uint32, C.c_double, U32P, F64P]),
    "sherd_nearest_below": (C.c_int, [VP, VP, F64P, C.c_uint32, C.c_double, U32P, F64P]),
    "sherd_icp_rung": (C.c_int, [VP, VP, C.c_uint32, VP, F64P, C.c_uint32, IcpOptions, VP]),
    "sherd_icp_rung_noalloc": (C.c_int, [VP, VP, C.c_uint32, VP, VP, C.c_uint32, IcpOptions, VP]),
    "sherd_surfaces_create": (C.c_int, [VP, VP, VP, C.c_uint32, C.c_double, VP, C.c_uint32, VP,
                                        C.c_uint32, VP, VP, C.c_uint32, VP, VP, C.c_uint32,
                                        C.POINTER(VP)]),
    "sherd_surfaces_free": (C.c_int, [VP]),
    "sherd_verify": (C.c_int, [VP, VP, VP, F64P, C.POINTER(Scales), C.c_int, C.POINTER(Scores)]),
    "sherd_scales_for_pair": (C.c_int, [C.POINTER(Params), C.c_double, C.c_double,
                                        C.POINTER(Scales)]),
    "sherd_params_default": (None, [C.POINTER(Params)]),
    "sherd_accept": (C.c_uint32, [C.POINTER(Scores), C.POINTER(Params), C.POINTER(Scales)]),
    "sherd_pair_create": (C.c_int, [VP, VP, VP, VP, VP, VP, C.c_uint32, VP, C.c_uint32,
                                    C.POINTER(Scales), C.POINTER(VP)]),
    "sherd_pair_free": (C.c_int, [VP]),
    "sherd_ladder_verify_batch": (C.c_int, [VP, VP, C.c_uint32, VP, C.c_uint32,
                                            C.POINTER(Params), C.c_int, VP]),
    "sherd_batch_create": (C.c_int, [VP, VP, C.c_uint32, VP, C.c_uint32, C.POINTER(Params),
                                     C.c_int, C.POINTER(VP)]),
    "sherd_batch_run": (C.c_int, [VP, np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")]),
    "sherd_batch_results": (C.c_int, [VP, VP]),
    "sherd_batch_free": (C.c_int, [VP]),
    "sherd_adjoint": (C.c_int, [VP, VP, C.c_uint32, F64P, F64P, C.c_uint32,
                                C.POINTER(AdjointOptions), F64P, F64P]),
    "sherd_penetration_share": (C.c_int, [VP, VP, F64P, C.c_uint32, F64P, C.c_double,
                                          C.POINTER(C.c_double)]),
    "sherd_coarse_scores": (C.c_int, [VP, VP, F64P, F64P, C.c_uint32, F64P, C.c_uint32,
                                      C.c_double, C.c_double, F64P]),
    "sherd_seg_params_default": (None, [C.POINTER(SegParams)]),
    "sherd_segment": (C.c_int, [VP, VP, F64P, C.c_uint32, U32P, C.c_uint32, C.c_double,
                                C.c_double, C.POINTER(SegParams), U8P, C.POINTER(SegInfo),
                                C.POINTER(SegTrace)]),
    "sherd_hypotheses_coarse": (C.c_int, [VP, C.POINTER(Frames), C.POINTER(Frames), U32P,
                                          C.c_uint32, U32P, C.c_uint32, C.c_double, VP, F64P,
                                          F64P, C.c_uint32, C.c_double, C.c_double, C.c_uint32,
                                          VP, VP, VP, VP, C.POINTER(C.c_uint32)]),
    "sherd_mesh_read": (C.c_int, [C.c_char_p, C.POINTER(VP), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32)]),
    "sherd_host_mesh_copy": (C.c_int, [VP, F64P, U32P]),
    "sherd_host_mesh_free": (C.c_int, [VP]),
    "sherd_breaklines": (C.c_int, [VP, F64P, C.c_uint32, U32P, C.c_uint32, U8P, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_uint32, VP, VP, VP, VP,
                                   VP, VP, VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "sherd_order_by_score": (C.c_int, [F64P, C.c_uint32, C.c_uint32, VP, C.POINTER(C.c_uint32)]),
    "sherd_nms": (C.c_int, [U32P, C.c_uint32, F64P, F64P, C.c_uint32, C.c_double, C.c_uint32,
                            C.c_double, VP, C.POINTER(C.c_uint32)]),
    "sherd_vertex_normals": (C.c_int, [VP, F64P, C.c_uint32, U32P, C.c_uint32, F64P]),
    "sherd_fracture_cloud": (C.c_int, [VP, F64P, C.c_uint32, U32P, C.c_uint32, F64P, U8P,
                                       C.c_uint32, C.c_double, C.c_uint32, U32P, F64P, F64P,
                                       C.POINTER(C.c_uint32)]),
    "sherd_refine_join": (C.c_int, [VP, F64P, C.c_uint32, F64P, F64P, C.c_uint32, F64P, F64P,
                                    F64P, C.c_int32, VP]),
}


def exported_symbols() -> tuple[str, ...]:
    """Every symbol include/sherd_cuda.h declares."""
    return tuple(_SIGNATURES)


def lib() -> C.CDLL:
    """The loaded backend library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        raise RuntimeError(
            f"the CUDA backend is not built ({LIBRARY} is missing); run "
            "`python -c 'import __graft_entry__; __graft_entry__.build()'`")
    L = C.CDLL(str(LIBRARY))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class SherdError(RuntimeError):
    """A non-zero status of the C ABI, with the library's message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def check(ctx_handle, code: int) -> None:
    if code != OK:
        msg = lib().sherd_last_error(ctx_handle)
        raise SherdError(code, msg.decode() if msg else "")


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(VP)
