"""Builders that turn the golden slab arrays into oracle or CUDA-backend objects.

The pair is the reference's `pieceA__pieceB`: A is fixed, B moves (R 0's convention), the
stage-2 clouds are A's `pc_reg`/`pc_frac` as ICP targets and B's as sources, exactly as
`sherd-parity/src/stages/pairs.rs:253-304` assembles them from the dump.
"""

from __future__ import annotations

import numpy as np

# D 10.2's stage-2 pose rows (sherd-parity/src/stages/stage2.rs:40-50).
ROT_DEG = 0.05
TRANS_T = 0.01
CHAOTIC_SHARE = 0.4
# D 10.2's verification rows (sherd-parity/src/stages/verify.rs:74-86).
VERIFY_TOL = {"tight": 0.01, "gap": 0.002, "seam": 0.34, "cont": 0.005, "cont_n": 0.01,
              "pen": 0.0005}
SCORE_KEYS = ("tight_a", "tight_b", "tight", "gap_a", "gap_b", "gap", "contact_a", "contact_b",
              "contact", "seam", "gap_limit", "tight_delta", "cont", "cont_n", "pen",
              "pen_depth", "brk")


def piece(slab, name):
    return {k.split(".", 1)[1]: v for k, v in slab.items() if k.startswith(name + ".")}


def trace_deg(a, b):
    """pose_gap::trace_deg (matching/icp.rs:820-829)."""
    tr = float(np.sum(a[:3, :3] * b[:3, :3]))
    return float(np.degrees(np.arccos(np.clip((tr - 1.0) / 2.0, -1.0, 1.0))))


def origin_t(a, b, t):
    """pose_gap::origin_t (matching/icp.rs:851-857)."""
    return float(np.linalg.norm(a[:3, 3] - b[:3, 3]) / t)


def oracle_pair(oracle, slab):
    """Oracle surfaces, targets and pair for the slab's one pair."""
    out = {}
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        mesh = oracle.Mesh(p["V"], p["F"])
        frac = mesh.subset(p["frac"])
        surf = oracle.Surfaces(frac, mesh, int(p["watertight"]), float(p["frac_area"]), p["Pf"],
                               p["S"], p["brk_P"], p["brk_ns"], p["margin_p"], p["margin_n"])
        out[name] = dict(mesh=mesh, frac=frac, surf=surf, arrays=p)
    a, b = out["pieceA"], out["pieceB"]
    reg_t = oracle.Cloud(a["arrays"]["reg_p"], a["arrays"]["reg_n"])
    frac_t = oracle.Cloud(a["arrays"]["frac_p"], a["arrays"]["frac_n"])
    scales = oracle.scales_from(slab["scales"])
    pair = oracle.Pair(a["surf"], b["surf"], reg_t, frac_t, b["arrays"]["reg_p"],
                       b["arrays"]["frac_p"], scales)
    return dict(a=a, b=b, reg_t=reg_t, frac_t=frac_t, scales=scales, pair=pair)


def slab_params(oracle, slab):
    p = oracle.default_params()
    for k, v in zip(("min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n"), slab["params"]):
        setattr(p, k, float(v))
    return p


def score_dict(scores):
    return {k: float(getattr(scores, k)) for k in SCORE_KEYS if hasattr(scores, k)}


def reference_scores(slab, k):
    return dict(zip(SCORE_KEYS, (float(x) for x in slab["s2_scores"][k])))
