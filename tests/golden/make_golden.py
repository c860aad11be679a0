"""Extract the golden vectors of the reference's slab fixture into tests/golden/slab.npz.

The reference commits one full stage dump of its pipeline over a two-piece synthetic slab
(`fixtures/slab/dump`, written by its Python original with Open3D/Embree; see
`fixtures/slab/README.md`). This script copies the arrays the geometry hot path reads and the
answers the reference produced from them, so the tests can pin the oracle and the CUDA backend
without the reference tree present:

* thickness (`fragment/thickness.rs:139-162`): the original component `load.V0`/`F0`, the
  face ids of the rays `thick.idx`, the Embree hits `thick.t_hit`/`thick.prim`, and the two
  answers `thick.t` / `thick.thick_mode` (bit-exact targets);
* segmentation (`fragment/segment.rs:189-631`): the working mesh `mesh.V`/`mesh.F` and its
  `mesh.res`, the voxel representatives `seg.rep` and each face's `seg.near`, the smoothed
  normals `seg.NS`, the cone votes `seg.good`, every intermediate mask (`seg.frac_raw`,
  `seg.frac_majority`, `seg.frac_islands`), `seg.has_ref`, the final mask `seg.frac_final` and
  `seg.info` (votes, smoothing radius, growth angle, raw fraction);
* stage 2 and verification (`sherd-parity/src/stages/{stage2,verify}.rs`): the sample arrays
  at the pair's own `t` (`md.Pf`, `md.fp`, `md.S`, `md.sp`, `md.margin_idx`, `md.brk_P`,
  `md.brk_ns`), the pair's `scales.json`, the starts `s1.T[nms2.kept]`, the four rung poses
  `s2.T_reg1..s2.T_frac2`, the scores `s2.scores.json` and the verdicts `s2.accepted`;
* R 3.5 at the pair's t (`fragment/breakline.rs`, `fragment/samples.rs`): the breakline's
  fracture macro normals `md.brk_nf` and validity `md.valid`, the sample faces `md.sp`, `md.fp`,
  the uniforms `md.S_u/S_v`, `md.Pf_u/Pf_v`, the margin `md.margin_idx` and `md.params.json`;
* stage 1 (R 5.1-5.5, `hypotheses.rs`, `coarse.rs`, `nms.rs`, `ladder.rs`): the breakline
  frames' in-plane axes `md.brk_f` and dihedrals `md.brk_dih`, the subsets and kept pairs
  `hyp.ia/ib/pa/pb`, the probe `coarse.idx` and every hypothesis's score `coarse.cs`, both
  suppressions' walk orders and kept lists `nms1.*`, `nms2.*`, and R 5.7's ranked result
  `result.candidates.json` (pose, verdict, brk, brk_best, seam, tight of each of the 5 kept);
* the coarse breakline score (`executor/cpu.rs:46-68,136-169`) through R 5.4's re-score:
  B's breakline subset `md.brk_sub`, the refined stage-1 poses `s1.T` and their scores
  `s1.score` against A's whole breakline at `scales.stage1`;
* R 9's join refinement (`refine.rs:282-386`, `sherd-parity/src/stages/refine.rs`): each
  fragment's vertex selection `refine/<name>.idx` and its `mesh.stats` (thick, res), the
  assembly's poses, groups and joins in `used` order (`assembly/*.json`), the joins the
  refinement walked (`refine/joins.json`: ends, radii, both rung poses, fitness, rmse / t) and
  the refined poses `refine/poses_final.json`.

Derived arrays are computed here with numpy exactly as the reference's harness computes them:
the f64 face normals and areas of `mesh::geometry::face_geometry` (`mesh/geometry.rs:70-96`,
element-wise IEEE operations in the same order), `fracture_area` as numpy's pairwise
`A[frac].sum()` (the reference's own `masked_area`), and the registration cloud split of
`samples::registration_split` (`fragment/samples.rs:601-615`).

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

PIECES = ("pieceA", "pieceB")
MD_PARAMS = ("t", "seed", "surface_points", "frac_per_t2", "min_frac_points", "max_frac_points",
             "margin_points", "macro_inner", "macro_outer", "brk_voxel")
PAIR = "pieceA__pieceB"
SCORE_KEYS = (
    "tightA", "tightB", "tight", "gapA", "gapB", "gap", "contactA", "contactB", "contact",
    "seam", "gap_limit", "tight_delta", "cont", "cont_n", "pen", "pen_depth", "brk",
)


def face_geometry(v: np.ndarray, f: np.ndarray):
    """mesh/geometry.rs:70-96, element for element (normal floor 1e-12)."""
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    e1 = b - a
    e2 = c - a
    n = np.stack([
        e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
        e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
        e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0],
    ], axis=1)
    length = np.sqrt((n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2])
    den = np.maximum(length, 1e-12)
    normals = n / den[:, None]
    areas = 0.5 * length
    centroids = (a + b + c) / 3.0
    return normals, areas, centroids


def registration_split(n_frac: int, n_margin: int, reg_points: int):
    """fragment/samples.rs:601-615 (numpy's round-half-even)."""
    if reg_points == 0 or n_frac + n_margin <= reg_points:
        return n_frac, n_margin
    share = float(n_frac) * float(reg_points) / float(n_frac + n_margin)
    take_f = min(max(int(np.round(share)), 1), n_frac)
    return take_f, min(max(reg_points - take_f, 0), n_margin)


def arrays_at(frag_dir: Path, t: float, surface_points: int) -> Path:
    """sherd-parity/src/stages/pairs.rs:480-502: the md directory whose t matches bit for bit."""
    candidates = [frag_dir] + sorted(p for p in (frag_dir / "md_t").glob("*") if p.is_dir())
    for d in candidates:
        params = d / "md.params.json"
        if not params.is_file():
            continue
        value = json.loads(params.read_text())
        if float(value["t"]) == t and int(value["surface_points"]) == surface_points:
            return d
    raise SystemExit(f"no md arrays at t={t!r} under {frag_dir}")


def refine_arrays(dump: Path, out: dict) -> None:
    """R 9's inputs and answers, fragments numbered in PIECES order."""
    names = list(PIECES)

    def poses(path: Path) -> np.ndarray:
        value = json.loads(path.read_text())
        return np.stack([np.array(value[n], dtype=np.float64) for n in names])

    out["refine_before"] = poses(dump / "assembly" / "poses.json")
    out["refine_after"] = poses(dump / "refine" / "poses_final.json")
    used = json.loads((dump / "assembly" / "used.json").read_text())
    out["refine_used"] = np.array([[names.index(u["a"]), names.index(u["b"])] for u in used],
                                  dtype=np.uint32).reshape(-1, 2)
    groups = json.loads((dump / "assembly" / "groups.json").read_text())
    out["refine_group_sizes"] = np.array([len(g) for g in groups], dtype=np.uint32)
    out["refine_group_members"] = np.array([names.index(n) for g in groups for n in g],
                                           dtype=np.uint32)
    joins = json.loads((dump / "refine" / "joins.json").read_text())
    out["refine_join_ends"] = np.array([[names.index(j["fixed"]), names.index(j["moving"])]
                                        for j in joins], dtype=np.uint32).reshape(-1, 2)
    out["refine_join_dist"] = np.array([j["dist"] for j in joins]).reshape(-1, 2)
    out["refine_join_rungs"] = np.array([j["T_rung"] for j in joins]).reshape(-1, 2, 4, 4)
    out["refine_join_fit_rmse"] = np.array([[j["fitness"], j["rmse_t"]] for j in joins]).reshape(-1, 2)


def main(reference: Path) -> None:
    dump = reference / "fixtures" / "slab" / "dump"
    pair_dir = dump / "pairs" / PAIR
    used = json.loads((pair_dir / "md_used.json").read_text())
    manifest = json.loads((dump / "manifest.json").read_text())
    params = manifest["collection"]["params"]
    t_pair = float(used["t"])
    out: dict[str, np.ndarray] = {}
    for name in PIECES:
        fd = dump / "fragments" / name
        p = name + "."
        v0 = np.load(fd / "load.V0.npy")
        f = np.load(fd / "load.F0.npy").astype(np.uint32)
        v = np.load(fd / "mesh.V.npy")
        fw = np.load(fd / "mesh.F.npy").astype(np.uint32)
        out[p + "V0"] = v0
        out[p + "F"] = fw
        assert np.array_equal(f, fw)
        out[p + "V"] = v
        out[p + "thick_idx"] = np.load(fd / "thick.idx.npy").astype(np.uint32)
        out[p + "thick_t_hit"] = np.load(fd / "thick.t_hit.npy").astype(np.float32)
        out[p + "thick_prim"] = np.load(fd / "thick.prim.npy").astype(np.uint32)
        out[p + "thick_t"] = np.float32(json.loads((fd / "thick.t.json").read_text()))
        out[p + "thick_mode"] = np.float32(json.loads((fd / "thick.thick_mode.json").read_text()))
        out[p + "seg_NS"] = np.load(fd / "seg.NS.npy")
        out[p + "seg_good"] = np.load(fd / "seg.good.npy").astype(np.uint8)
        frac = np.load(fd / "seg.frac_final.npy").astype(bool)
        out[p + "frac"] = frac.astype(np.uint8)
        for k in ("frac_raw", "frac_majority", "frac_islands", "has_ref"):
            out[p + "seg_" + k] = np.load(fd / f"seg.{k}.npy").astype(np.uint8)
        out[p + "seg_rep"] = np.load(fd / "seg.rep.npy").astype(np.uint32)
        out[p + "seg_near"] = np.load(fd / "seg.near.npy").astype(np.uint32)
        info = json.loads((fd / "seg.info.json").read_text())
        out[p + "seg_info"] = np.array([info["votes"], info["smooth_radius"],
                                        info["boundary_angle"], info["raw_fraction"]])
        out[p + "res"] = np.float64(json.loads((fd / "mesh.res.json").read_text()))
        wt = json.loads((fd / "mesh.watertight.json").read_text())
        out[p + "watertight"] = np.uint32(bool(wt["watertight"]))
        out[p + "n_boundary"] = np.uint32(wt["n_boundary"])
        fn, areas, _ = face_geometry(v, fw.astype(np.int64))
        out[p + "frac_area"] = np.float64(areas[frac].sum())
        md = arrays_at(fd, t_pair, int(used["surface_points"]))
        pf = np.load(md / "md.Pf.npy")
        fp = np.load(md / "md.fp.npy").astype(np.int64)
        s = np.load(md / "md.S.npy")
        sp = np.load(md / "md.sp.npy").astype(np.int64)
        margin_idx = np.load(md / "md.margin_idx.npy").astype(np.int64)
        out[p + "Pf"] = pf
        out[p + "S"] = s
        out[p + "brk_P"] = np.load(md / "md.brk_P.npy")
        out[p + "brk_ns"] = np.load(md / "md.brk_ns.npy")
        out[p + "brk_sub"] = np.load(md / "md.brk_sub.npy").astype(np.uint32)
        out[p + "brk_f"] = np.load(md / "md.brk_f.npy")
        out[p + "brk_dih"] = np.load(md / "md.brk_dih.npy")
        out[p + "brk_nf"] = np.load(md / "md.brk_nf.npy")
        out[p + "brk_valid"] = np.load(md / "md.valid.npy").astype(np.uint8)
        out[p + "sp"] = np.load(md / "md.sp.npy").astype(np.uint32)
        out[p + "fp"] = np.load(md / "md.fp.npy").astype(np.uint32)
        out[p + "S_uv"] = np.stack([np.load(md / "md.S_u.npy"), np.load(md / "md.S_v.npy")])
        out[p + "Pf_uv"] = np.stack([np.load(md / "md.Pf_u.npy"), np.load(md / "md.Pf_v.npy")])
        out[p + "margin_idx"] = np.load(md / "md.margin_idx.npy").astype(np.uint32)
        mdp = json.loads((md / "md.params.json").read_text())
        out[p + "md_params"] = np.array([mdp[k] for k in MD_PARAMS], dtype=np.float64)
        nf_ = fn[fp]
        pm = s[margin_idx]
        nm = fn[sp[margin_idx]]
        out[p + "margin_p"] = pm
        out[p + "margin_n"] = nm
        take_f, take_m = registration_split(len(pf), len(pm), int(params["reg_points"]))
        out[p + "reg_p"] = np.concatenate([pf[:take_f], pm[:take_m]])
        out[p + "reg_n"] = np.concatenate([nf_[:take_f], nm[:take_m]])
        out[p + "frac_p"] = pf
        out[p + "frac_n"] = nf_
        out[p + "refine_idx"] = np.load(dump / "refine" / f"{name}.idx.npy").astype(np.uint32)
        stats = json.loads((fd / "mesh.stats.json").read_text())
        out[p + "stats_thick_res"] = np.array([float(stats["thick"]), float(stats["res"])])
    scales = json.loads((pair_dir / "scales.json").read_text())
    out["scales"] = np.array([scales[k] for k in (
        "t", "res", "coarse", "stage1", "tight", "facing", "gap", "seam", "near", "pen", "nms",
        "icp")], dtype=np.float64)
    for k in ("hyp.ia", "hyp.ib", "hyp.pa", "hyp.pb", "coarse.idx", "nms1.order", "nms1.kept",
              "nms2.order", "nms2.kept"):
        out[k.replace(".", "_")] = np.load(pair_dir / f"{k}.npy").astype(np.uint32)
    out["coarse_cs"] = np.load(pair_dir / "coarse.cs.npy")
    result = json.loads((pair_dir / "result.candidates.json").read_text())
    out["result_T"] = np.array([c["T"] for c in result], dtype=np.float64).reshape(-1, 4, 4)
    out["result_accepted"] = np.array([bool(c["accepted"]) for c in result], dtype=np.uint8)
    out["result_brk"] = np.array([[c["brk"], c["brk_best"]] for c in result]).reshape(-1, 2)
    out["result_seam_tight"] = np.array([[c["seam"], c["tight"]] for c in result]).reshape(-1, 2)
    out["s1_T"] = np.load(pair_dir / "s1.T.npy")
    out["s1_score"] = np.load(pair_dir / "s1.score.npy")
    kept = np.load(pair_dir / "nms2.kept.npy").astype(np.int64)
    s1 = np.load(pair_dir / "s1.T.npy")
    out["starts"] = s1[kept]
    for rung in ("T_reg1", "T_reg2", "T_frac1", "T_frac2"):
        out["s2_" + rung] = np.load(pair_dir / f"s2.{rung}.npy")
    scores = json.loads((pair_dir / "s2.scores.json").read_text())
    out["s2_scores"] = np.array([[float(s.get(k, 0.0)) for k in SCORE_KEYS] for s in scores])
    out["s2_pen_unavailable"] = np.array([float(s.get("pen_unavailable", 0.0)) for s in scores])
    out["s2_accepted"] = np.load(pair_dir / "s2.accepted.npy").astype(np.uint8)
    out["params"] = np.array([params[k] for k in (
        "min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n")], dtype=np.float64)
    refine_arrays(dump, out)
    target = Path(__file__).resolve().parent / "slab.npz"
    np.savez_compressed(target, **out)
    print(f"wrote {target} ({target.stat().st_size / 1e6:.2f} MB, {len(out)} arrays)")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(Path(sys.argv[1]))
