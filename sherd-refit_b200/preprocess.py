"""R 3.5 on the device: a labelled working mesh to the arrays pair matching reads
(fragment/breakline.rs, fragment/samples.rs, the MatchData of samples.rs:470-560).

* `breaklines`: sherd_breaklines, the breakline points, macro normals, frames, validity,
  dihedrals and hypothesis subset, all on the device.
* `samples`: the three area-weighted samples (surface, fracture, shell margin). The random draws
  are the reference's own: one numpy `default_rng(seed)` per fragment, consumed in the order
  samples.rs:33-42 gives (surface picks, u, v; fracture picks, u, v; the margin's
  `choice(..., replace=False)`), so the samples are the reference pipeline's bit for bit. The
  face areas come from the device (sherd_face_geometry, bit-identical), the picks are
  `searchsorted` on the host's sequential cumulative sum, and each sample's distance to the
  breakline is the device's bounded nearest-neighbour search (sherd_nearest_below).
* `match_data`: both, plus R 3.6's derived clouds (`pc_frac`, `pc_reg` by
  samples.rs:586-618's split) and the stage-1 `Frames`.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .backend import Context
from .stage1 import Frames

MACRO_INNER, MACRO_OUTER, BRK_VOXEL = 0.15, 0.60, 0.5   # breakline.rs:72-76
SURFACE_POINTS = 20_000      # samples.rs:70
FRAC_PER_T2 = 150.0          # samples.rs:72
MIN_FRAC_POINTS = 5_000      # samples.rs:74
MAX_FRAC_POINTS = 12_000     # samples.rs:76
MARGIN_POINTS = 6_000        # samples.rs:78
REG_POINTS = 6_000           # samples.rs:80
MARGIN_INNER, MARGIN_OUTER = 0.12, 1.5   # samples.rs:82-84


@dataclass
class Breaklines:
    """breakline::Breaklines (breakline.rs:85-130), in f64."""
    p: np.ndarray
    ns: np.ndarray
    nf: np.ndarray
    f: np.ndarray
    dih: np.ndarray
    valid: np.ndarray
    sub: np.ndarray

    def __len__(self) -> int:
        return len(self.p)

    def frames(self) -> Frames:
        """hypotheses::Frames::of (hypotheses.rs:70-82)."""
        return Frames(p=self.p, ns=self.ns, f=self.f, dih=self.dih, sub=self.sub)


@dataclass
class Samples:
    """samples::Samples (samples.rs:135-158), with the draws that made them."""
    s: np.ndarray
    sp: np.ndarray
    pf: np.ndarray
    fp: np.ndarray
    margin_idx: np.ndarray
    s_uv: np.ndarray
    pf_uv: np.ndarray


def breaklines(ctx: Context, v, f, frac, t: float, macro_inner=MACRO_INNER,
               macro_outer=MACRO_OUTER, brk_voxel=BRK_VOXEL) -> Breaklines:
    """breakline::build (breakline.rs:207-300) of a labelled working mesh at wall thickness t."""
    d = ctx.breaklines(v, f, frac, t, macro_inner, macro_outer, brk_voxel)
    return Breaklines(d["p"], d["ns"], d["nf"], d["f"], d["dih"], d["valid"], d["sub"])


def fracture_count(fracture_area: float, t: float, frac_per_t2=FRAC_PER_T2,
                   lo=MIN_FRAC_POINTS, hi=MAX_FRAC_POINTS) -> int:
    """samples::fracture_count (samples.rs:250-268): int(clip(150 A / t^2, 5000, 12000))."""
    raw = frac_per_t2 * fracture_area / (t * t)
    if np.isnan(raw):
        return int(lo)
    return int(np.clip(raw, lo, hi))


def _sample_on_faces(rng, v, f, areas, faces, n):
    """sample_on_faces (samples.rs:281-305) with numpy's stream: n uniforms pick the faces by
    searchsorted(cdf, u, 'right') over the normalised sequential cumulative area, then n for u
    and n for v, folded where u + v > 1 (points_from_uniforms, samples.rs:325-355)."""
    if len(faces) == 0 or n == 0:
        return np.zeros((0, 3)), np.zeros(0, np.int64), np.zeros((2, 0))
    w = areas[faces] / areas[faces].sum()
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    picks = faces[np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), len(faces) - 1)]
    u, vv = rng.random(n), rng.random(n)
    fold = u + vv > 1.0
    al, be = np.where(fold, 1.0 - u, u), np.where(fold, 1.0 - vv, vv)
    o, pu, pv = v[f[picks, 0]], v[f[picks, 1]], v[f[picks, 2]]
    return (o + al[:, None] * (pu - o)) + be[:, None] * (pv - o), picks, np.stack([u, vv])


def samples(ctx: Context, v, f, frac, brk_points, t: float, seed: int = 0,
            surface_points=SURFACE_POINTS, frac_per_t2=FRAC_PER_T2, min_frac=MIN_FRAC_POINTS,
            max_frac=MAX_FRAC_POINTS, margin_points=MARGIN_POINTS, areas=None) -> Samples:
    """samples::build (samples.rs:201-248) with the reference's numpy stream."""
    v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
    f = np.asarray(f, np.int64).reshape(-1, 3)
    frac = np.asarray(frac).astype(bool)
    if areas is None:
        _, areas, _ = ctx.face_geometry(v, f)
    rng = np.random.default_rng(seed)
    s, sp, s_uv = _sample_on_faces(rng, v, f, areas, np.arange(len(f)), surface_points)
    fr = np.flatnonzero(frac)
    n_frac = fracture_count(float(areas[fr].sum()), t, frac_per_t2, min_frac, max_frac)
    pf, fp, pf_uv = _sample_on_faces(rng, v, f, areas, fr, n_frac)
    bp = np.ascontiguousarray(brk_points, np.float64).reshape(-1, 3)
    if len(bp) and len(s):
        _, d_brk = ctx.cloud(bp).nearest_below(s, MARGIN_OUTER * t)
    else:
        d_brk = np.full(len(s), np.inf)
    margin = np.flatnonzero(~frac[sp] & (d_brk > MARGIN_INNER * t) & (d_brk < MARGIN_OUTER * t))
    if margin_points and len(margin) > margin_points:
        margin = np.sort(rng.choice(margin, margin_points, replace=False))
    return Samples(s, sp, pf, fp, margin, s_uv, pf_uv)


def registration_split(n_frac: int, n_margin: int, reg_points: int):
    """samples::registration_split (samples.rs:601-618): how many fracture and margin points the
    registration cloud takes (numpy's round-half-even)."""
    if reg_points == 0 or n_frac + n_margin <= reg_points:
        return n_frac, n_margin
    share = float(n_frac) * float(reg_points) / float(n_frac + n_margin)
    take_f = min(max(int(np.round(share)), 1), n_frac)
    return take_f, min(max(reg_points - take_f, 0), n_margin)


@dataclass
class MatchData:
    """One fragment's arrays at one t, as pair matching reads them (samples.rs:470-560)."""
    t: float
    brk: Breaklines
    samples: Samples
    frac_area: float
    pf_n: np.ndarray       # the fracture samples' face normals (pc_frac's normals)
    margin_p: np.ndarray
    margin_n: np.ndarray
    reg_p: np.ndarray      # pc_reg
    reg_n: np.ndarray

    @property
    def frames(self) -> Frames:
        return self.brk.frames()


def match_data(ctx: Context, v, f, frac, t: float, seed: int = 0,
               reg_points: int = REG_POINTS) -> MatchData:
    """R 3.5 and R 3.6 of one labelled working mesh at wall thickness t."""
    v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
    f = np.asarray(f, np.int64).reshape(-1, 3)
    frac = np.asarray(frac).astype(bool)
    normals, areas, _ = ctx.face_geometry(v, f)
    brk = breaklines(ctx, v, f, frac, t)
    smp = samples(ctx, v, f, frac, brk.p, t, seed, areas=areas)
    frac_area = float(areas[frac].sum())
    pf_n = normals[smp.fp]
    margin_p = smp.s[smp.margin_idx]
    margin_n = normals[smp.sp[smp.margin_idx]]
    take_f, take_m = registration_split(len(smp.pf), len(margin_p), reg_points)
    reg_p = np.concatenate([smp.pf[:take_f], margin_p[:take_m]])
    reg_n = np.concatenate([pf_n[:take_f], margin_n[:take_m]])
    return MatchData(t, brk, smp, frac_area, pf_n, margin_p, margin_n, reg_p, reg_n)
