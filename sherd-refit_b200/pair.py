"""R 5's whole pair chain on the device: matching/pair.rs:375-440 (`match_pair`).

Stage 1 (`stage1.PairStage1.run`: hypotheses, coarse score, suppression, the breakline ladder
and its re-score, the second suppression) gives at most `stage2` starts; each start goes through
the batched stage-2 path (sherd_ladder_verify_batch: the four point-to-plane rungs, R 6's scores
and R 6.5's verdict, one work item per start); R 5.7 then ranks the candidates by seam * tight,
descending and stable (ties keep the second suppression's order), writes the pair's best stage-1
score on every one and keeps the first `keep`. A pair whose best stage-1 score is under a
non-zero `stage1_floor` returns its best stage-1 pose alone, marked partial and refused
(pair.rs:413-432).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .backend import Context
from .stage1 import PairStage1, Stage1Result

KEEP_PER_PAIR = 5  # pipeline.rs:173


@dataclass
class PairResult:
    """match_pair's candidates (sherd_candidate records, R 5.7's order, at most `keep`) and the
    stage-1 result they came from. `starts[i]` is the start candidate i was refined from."""
    candidates: list
    stage1: Stage1Result
    starts: list = field(default_factory=list)

    @property
    def transforms(self) -> list:
        """Each candidate's pose: the last rung's (the R 5.6 ladder's result)."""
        return [np.array(c.rungs[3].transform[:]).reshape(4, 4) for c in self.candidates]


def _partial(scales: A.Scales, transform, brk: float) -> A.Candidate:
    """Scores::partial (verify.rs:183-195): nothing computed, the two limits filled in, `brk`
    and `brk_best` set, partial and refused."""
    c = A.Candidate()
    c.scores.gap_limit = scales.gap / scales.t
    c.scores.tight_delta = scales.tight / scales.t
    c.scores.partial = 1
    c.scores.brk = brk
    c.scores.brk_best = brk
    c.accepted = 0
    t = np.ascontiguousarray(transform, np.float64).reshape(16)
    for r in range(4):
        c.rungs[r].transform[:] = t.tolist()
    return c


def match_pair(ctx: Context, pair, stage1: PairStage1, params: A.Params,
               keep: int = KEEP_PER_PAIR, seed: int = 0, stage1_floor: float = 0.0,
               order1=None, order2=None) -> PairResult:
    """Pair::match_pair (pair.rs:375-440) for one device pair (`pair`, a backend.Pair over the
    same two fragments as `stage1`). `order1` / `order2` replace the two suppressions' walk
    orders (the reference's Python pipeline's unstable ones, for parity runs)."""
    s1 = stage1.run(seed=seed, order1=order1, order2=order2)
    if not len(s1.scores):
        return PairResult([], s1)
    best1 = s1.best
    if stage1_floor > 0.0 and best1 < stage1_floor:
        k = int(np.flatnonzero(s1.scores == best1)[0])   # pair.rs:793-796, the first maximum
        return PairResult([_partial(stage1.scales, s1.transforms[k], best1)], s1, [k])
    starts = s1.starts
    brk = s1.scores[s1.kept2.astype(np.int64)]
    out = ctx.ladder_verify_batch([pair], [(0, k, starts[k]) for k in range(len(starts))], params)
    cands = [A.Candidate.from_buffer_copy(out[k]) for k in range(len(starts))]
    for c, b in zip(cands, brk):
        c.scores.brk = float(b)
    order = sorted(range(len(cands)), key=lambda k: -(cands[k].scores.seam * cands[k].scores.tight))
    cands = [cands[k] for k in order]
    for c in cands:
        c.scores.brk_best = best1
    return PairResult(cands[:keep], s1, order[:keep])


@dataclass
class FragmentInput:
    """One labelled working mesh as the matching stage reads it: f64 vertices, faces, the
    fracture label per face, R 3.2's thickness, R 3.3's res and its watertightness."""
    v: np.ndarray
    f: np.ndarray
    frac: np.ndarray
    t: float
    res: float
    watertight: bool = True


def match_collection(ctx: Context, fragments, pairs, params: A.Params,
                     keep: int = KEEP_PER_PAIR, seed: int = 0, stage1_floor: float = 0.0,
                     timings: dict | None = None) -> list:
    """R 5 over a list of pairs (a, b) of `fragments` (FragmentInput), the collection form of
    match_pair: each fragment's R 3.5 arrays at each t a pair asks for (t_pair = min(t_a, t_b),
    R 4.2), stage 1 per pair, ONE batched stage-2 call over every pair's starts (the items are
    independent, batch.rs:417-423), then R 5.7 per pair. Returns one PairResult per pair, in
    order. `timings`, when given, receives the host seconds of each phase."""
    import time

    from . import preprocess
    from .backend import scales_for_pair
    clock = time.perf_counter
    t0 = clock()
    scales = [scales_for_pair(params, min(fragments[a].t, fragments[b].t),
                              max(fragments[a].res, fragments[b].res)) for a, b in pairs]
    data, dev = {}, {}
    meshes = {}
    for (a, b), sc in zip(pairs, scales):
        for k in (a, b):
            key = (k, sc.t)
            if key in data:
                continue
            fr = fragments[k]
            md = preprocess.match_data(ctx, fr.v, fr.f, fr.frac, sc.t, seed)
            if k not in meshes:
                mesh = ctx.mesh(fr.v, fr.f)
                meshes[k] = (mesh, mesh.subset(fr.frac))
            mesh, fm = meshes[k]
            surf = ctx.surfaces(fm, mesh, int(bool(fr.watertight)), md.frac_area, md.samples.pf,
                                md.samples.s, md.brk.p, md.brk.ns, md.margin_p, md.margin_n)
            data[key] = md
            dev[key] = (surf, ctx.cloud(md.reg_p, md.reg_n), ctx.cloud(md.samples.pf, md.pf_n))
    t1 = clock()
    results, items, handles, owner = [], [], [], []
    for k, ((a, b), sc) in enumerate(zip(pairs, scales)):
        ma, mb = data[(a, sc.t)], data[(b, sc.t)]
        if not all(len(m.samples.pf) and len(m.brk) for m in (ma, mb)):
            results.append(None)   # not matchable (pair.rs:161-165): no candidate
            continue
        s1 = PairStage1(ctx, ma.frames, mb.frames, sc).run(seed=seed)
        results.append(PairResult([], s1))
        if not len(s1.scores) or (stage1_floor > 0.0 and s1.best < stage1_floor):
            continue
        sa, reg_t, frac_t = dev[(a, sc.t)]
        sb = dev[(b, sc.t)][0]
        handles.append(ctx.pair(sa, sb, reg_t, frac_t, mb.reg_p, mb.samples.pf, sc))
        owner.append(k)
        items += [(len(handles) - 1, j, start) for j, start in enumerate(s1.starts)]
    t2 = clock()
    out = ctx.ladder_verify_batch(handles, items, params) if items else []
    t3 = clock()
    per = [[] for _ in pairs]
    for i in range(len(items)):
        c = A.Candidate.from_buffer_copy(out[i])
        per[owner[c.pair]].append(c)
    for k, (res, sc) in enumerate(zip(results, scales)):
        if res is None:
            results[k] = PairResult([], None)
            continue
        s1 = res.stage1
        if not len(s1.scores):
            continue
        if stage1_floor > 0.0 and s1.best < stage1_floor:
            j = int(np.flatnonzero(s1.scores == s1.best)[0])
            res.candidates, res.starts = [_partial(sc, s1.transforms[j], s1.best)], [j]
            continue
        cands = sorted(per[k], key=lambda c: c.start)
        brk = s1.scores[s1.kept2.astype(np.int64)]
        for c in cands:
            c.scores.brk = float(brk[c.start])
        order = sorted(range(len(cands)),
                       key=lambda i: -(cands[i].scores.seam * cands[i].scores.tight))
        ranked = [cands[i] for i in order]
        for c in ranked:
            c.scores.brk_best = s1.best
        res.candidates, res.starts = ranked[:keep], [cands[i].start for i in order[:keep]]
    if timings is not None:
        timings.update(preprocess=t1 - t0, stage1=t2 - t1, stage2=t3 - t2, rank=clock() - t3)
    return results
