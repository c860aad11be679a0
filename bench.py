"""Pair-pose verifications/s of the batched stage-2 path (4-rung point-to-plane ICP ladder +
R 6 verification + R 6.5 verdict per (pair, start)) on a B200.

Workload (default): the 40-fragment collection of three synthetic pots (t = 5, 8, 12), all
780 pairs x 128 ladder starts = 99 840 verifications per step, generated seeded (synth.py).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config collection] [--impl cuda]

Printed by rank 0: one JSON line with `value` (device throughput with every input resident in
HBM, CUDA events around the batch's graph on the library's stream, max over ranks), `e2e`
(the same metric through the host-buffer C-ABI call sherd_ladder_verify_batch, the work items
copied in and the candidates copied out every step), the roofline of the dominant kernel,
the clocks seen during the timed region and the oracle's CPU baseline on a bounded sample.
`--impl reference` times the reference algorithm's CPU restatement (the oracle; the Rust
reference cannot be built here) on all host cores instead. `--config group` measures the
differentiation workload instead (sherd_adjoint over 4096 perturbed poses of an assembled
8-fragment pot, and a 50-evaluation joint refinement). `--config refine` measures R 9, the
full-resolution join refinement of one assembled pot (fracture clouds and the spanning walk of
two-rung ICP joins). `--config stage1` measures R 5.1-5.5 on the reference's slab pair, and `--config chain` the
whole matching stage from labelled meshes (R 3.5 and R 5) on a synthetic workload.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "pair-pose verifications/s"
UNIT = "verifications/s"
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) of one launch of a stage's dominant kernel, per (workload, seed,
# kernel, ranks), from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of
# `python bench.py --steps 1 --warmup 3 --no-cpu --no-plain`, with the digest of the CUDA sources
# it was taken on: a capture of other sources is not reported.
TRAFFIC = {
    # the ladder stage's bucket launches together (> 16384 and > 4096 moving points; ncu runs
    # them one after the other): 104.48 + 147.47 GB read, 26.85 + 123.78 GB written
    ("collection", 0, "k_ladder", 1): (402.58e9, "bbb2f9119671"),
}


def _pkg(name=""):
    return importlib.import_module("sherd-refit_b200" + (("." + name) if name else ""))


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(world, x):
    return x if world == 1 else _pkg("shard").max_over_ranks(x, device="cuda")


def nn_query_rates(sbytes: dict, stage_ms: dict, step_ms: float, total_q: float) -> dict:
    """NN queries/s of the batched path: every ICP point-iteration of k_ladder is one bounded
    nearest-neighbour query (48 algorithmic bytes each), so the ladder stage's queries are its
    bytes / 48; the rate over this rank's ladder stage device time, and over the whole step
    (all ranks' queries, `total_q`, over the slowest rank's step)."""
    q = sbytes["ladder"] / 48.0
    ms = stage_ms.get("ladder", 0.0)
    return {"ladder_queries_per_step": total_q,
            "nn_queries_per_s": q / (ms / 1000.0) if ms > 0 else None,
            "nn_queries_per_s_whole_step": total_q / (step_ms / 1000.0) if step_ms > 0 else None,
            "unit": "queries/s",
            "what": "one bounded nearest-neighbour query per ICP point-iteration (k_ladder)"}


CPU_ITEMS = 512


def oracle_sample(wl, k: int) -> np.ndarray:
    """The CPU legs' sample: k items evenly spaced over the pair-major item list (ascending item
    indices). The same sample serves the CUDA arm's cpu_baseline and parity legs and every step
    of the reference arm, so the two CPU figures are of one workload."""
    n = wl.n_items
    return np.unique(np.linspace(0, n - 1, min(int(k), n)).round().astype(np.int64))


def oracle_run(oracle, wl, pairs, idx, params):
    """The oracle over the items idx on all host threads: (candidates in idx order, seconds).
    The items are handed over most expensive first (the threads take them in list order), the
    order the device queue takes them in, so the last thread to finish is not left holding the
    largest item."""
    workload = _pkg("workload")
    shard = _pkg("shard")
    pair, start, inits = workload.item_arrays(wl)
    cost = shard.pair_costs(wl)[pair[idx].astype(np.int64)]
    order = np.argsort(-cost, kind="stable")
    sel = idx[order]
    items = oracle.work_items_from(pair[sel], start[sel], inits[sel])
    t0 = time.perf_counter()
    out, _ = oracle.ladder_verify_items(pairs, items, params, 0)
    dt = time.perf_counter() - t0
    got = np.ctypeslib.as_array(out)[: len(idx)].copy()
    cands = np.empty_like(got)
    cands[order] = got
    return cands, dt


def cpu_baseline_and_parity(wl, k, gpu_cands):
    """The oracle (reference algorithm, f64, all host threads) on the deterministic sample:
    its rate as cpu_baseline, and its candidates compared with the CUDA path's at the same
    items (oracle.parity: verdicts, status and the final pose against the f64 answer, with the
    reference's one-ULP chaos probe for any item outside the bound)."""
    oracle = importlib.import_module("oracle")
    parity = importlib.import_module("oracle.parity")
    workload = _pkg("workload")
    pairs, keep = oracle.collection(wl)
    params = oracle.default_params()
    threads = oracle.lib().or_default_threads()
    idx = oracle_sample(wl, k)
    ref, dt = oracle_run(oracle, wl, pairs, idx, params)
    sample = (f"{len(idx)} of the {wl.n_items} (pair, start) items, evenly spaced over the "
              f"pair-major item list, on {threads} threads, {dt:.1f} s")
    cpu = {"value": len(idx) / dt, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": sample}
    par = None
    if gpu_cands is not None:
        arrays = workload.item_arrays(wl)
        t, c = parity.item_scale(wl, arrays[0][idx])
        probe = parity.collection_probe(oracle, pairs, params, arrays, idx, ref, t, c)
        t0 = time.perf_counter()
        par = parity.compare(gpu_cands[idx], ref, t, c, pair_ids=arrays[0][idx], probe=probe)
        par["probe_s"] = round(time.perf_counter() - t0, 1)
        par["sample"] = "the cpu_baseline sample: " + sample
        par["oracle"] = "oracle/oracle.cpp, the reference algorithm in f64 (source-order sums)"
    del keep
    return cpu, par


def run_reference(args):
    """The reference arm: the reference algorithm's CPU restatement (the oracle; the Rust
    reference cannot be built here) on all host cores, each timed step the whole deterministic
    sample (oracle_sample) of the same workload, most expensive item first. The warm-up steps
    run one item per thread of the same sample, untimed."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    synth = _pkg("synth")
    wl = synth.make(args.config, args.seed)
    oracle = importlib.import_module("oracle")
    pairs, keep = oracle.collection(wl)
    params = oracle.default_params()
    threads = oracle.lib().or_default_threads()
    idx = oracle_sample(wl, args.cpu_items)
    for _ in range(args.warmup):
        oracle_run(oracle, wl, pairs, idx[:: max(1, len(idx) // threads)], params)
    times = []
    for _ in range(args.steps):
        _, dt = oracle_run(oracle, wl, pairs, idx, params)
        times.append(dt)
    value = len(idx) * len(times) / sum(times)
    sample = (f"{len(idx)} of the {wl.n_items} (pair, start) items per step, evenly spaced over "
              f"the pair-major item list (the CUDA arm's cpu_baseline sample), {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, sherd-refit_b200/synth.py)",
        "config": _config_dict(wl, args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference's Rust CPU backend cannot be built in this image (no cargo); "
                 "this is its C++ restatement (oracle/oracle.cpp), pinned to the reference's "
                 "fixture, f64 point loops as the reference's Numerics::REFERENCE"),
    }
    print(json.dumps(line), flush=True)
    del keep


def run_group(args):
    """The differentiation workload: the 8-fragment pot assembled (its 18 adjacent pairs as
    edges), every fragment pose perturbed by 0.5 deg and 0.2 t, 4096 group poses. One step is
    one sherd_adjoint evaluation of all of them (values and twist gradients of every edge);
    the line also reports a 50-evaluation joint refinement of the same 4096 poses."""
    world, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    sherd = _pkg()
    synth = _pkg("synth")
    workload = _pkg("workload")
    adj = _pkg("adjoint")
    wl = synth.make("pot", args.seed)
    ctx = sherd.Context(local)
    dev = workload.to_device(ctx, wl)
    group = workload.assembled_group(dev, wl)
    truth, w0 = workload.perturbed_group_poses(wl, args.group_poses, seed=args.seed + 1)
    for _ in range(args.warmup):
        group.evaluate(w0)
    sampler = ClockSampler(local)
    sampler.start()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        values, _ = group.evaluate(w0)
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    step = float(np.mean(times))
    queries = args.group_poses * int(sum(
        len(wl.fragments[b].pf) * 2 + len(wl.fragments[a].pf) for a, b in zip(group.a, group.b)))
    t0 = time.perf_counter()
    w, history = adj.refine(group, w0, steps=50)
    t_refine = time.perf_counter() - t0
    rot0, disp0 = adj.edge_errors(w0, group, truth)
    rot1, disp1 = adj.edge_errors(w, group, truth)
    v1, _ = group.evaluate(w)
    t = float(np.min(group.t))
    line = {
        "metric": "group-pose adjoint evaluations/s", "value": args.group_poses / step,
        "unit": "group poses/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": f"pot group: {len(wl.fragments)} fragments, {len(group.a)} "
                               f"edges, {args.group_poses} perturbed group poses "
                               "(0.5 deg, 0.2 t per fragment)",
                   "queries_per_step": queries,
                   "timer": "host wall clock around the synchronous C-ABI call (poses in, "
                            "values and gradients out)"},
        "queries_per_s": queries / step,
        "refinement": {"evaluations": len(history), "seconds": t_refine,
                       "edge_rot_deg": [float(rot0.mean()), float(rot1.mean())],
                       "edge_disp_t": [float(disp0.mean()) / t, float(disp1.mean()) / t],
                       "tight": [float((values[..., 1] / values[..., 2]).mean()),
                                 float((v1[..., 1] / v1[..., 2]).mean())]},
        "gpu_launches": args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def _edge_errors(poses, truth, edges, t):
    """Mean rotation (deg) and translation (in t) of the relative poses over the joins."""
    rot, disp = [], []
    for a, b in edges:
        mine = np.linalg.inv(poses[a]) @ poses[b]
        want = np.linalg.inv(truth[a]) @ truth[b]
        r = mine[:3, :3].T @ want[:3, :3]
        rot.append(np.degrees(np.arccos(np.clip((np.trace(r) - 1.0) / 2.0, -1.0, 1.0))))
        disp.append(np.linalg.norm(mine[:3, 3] - want[:3, 3]) / t[b])
    return float(np.mean(rot)), float(np.mean(disp))


def run_refine(args):
    """R 9 on one assembled pot: every adjacent pair a join (in pair order), every fragment pose
    perturbed by 0.1 deg about its fracture centroid and 0.02 t (the assembly's poses are right
    to a fraction of the first rung's 0.05 t radius; larger errors are outside what R 9 can
    capture). One step is the whole stage: each fragment's fracture cloud (vertex normals and
    the vertex selection on the device, from the original mesh) and the spanning walk of
    sherd_refine_join calls (two 40-iteration rungs per join)."""
    world, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    sherd = _pkg()
    synth = _pkg("synth")
    workload = _pkg("workload")
    refine = _pkg("refine")
    t_gen = time.perf_counter()
    wl = synth.make(args.refine_workload, args.seed)
    t_gen = time.perf_counter() - t_gen
    ctx = sherd.Context(local)
    frags = wl.fragments
    meshes = [(fr.v.astype(np.float64), fr.f) for fr in frags]
    cents = [ctx.face_geometry(v, f)[2] for v, f in meshes]
    used = [(p.a, p.b) for p in wl.pairs if p.adjacent]
    groups = [list(range(len(frags)))]
    truth, w0 = workload.perturbed_group_poses(wl, 1, seed=args.seed + 1, rot_deg=0.1,
                                               trans_t=0.02)
    poses = list(w0[0])
    thick = np.array([fr.t for fr in frags])

    def step():
        t0 = time.perf_counter()
        pieces = [refine.RefinePiece(fr.t, fr.res, refine.fracture_cloud(
            ctx, v, f, c, fr.frac, fr.t, fr.res)) for fr, (v, f), c in zip(frags, meshes, cents)]
        t1 = time.perf_counter()
        out = refine.refine_joins(ctx, pieces, poses, groups, used)
        t2 = time.perf_counter()
        return pieces, out, t1 - t0, t2 - t1

    for _ in range(args.warmup):
        step()
    stats0 = ctx.stats()["methods"]
    sampler = ClockSampler(local)
    sampler.start()
    runs = [step() for _ in range(args.steps)]
    clocks = sampler.stop()
    stats1 = ctx.stats()["methods"]
    device_ms = {k: {"ms_per_step": (v["ms"] - stats0.get(k, {}).get("ms", 0.0)) / args.steps,
                     "calls_per_step": (v["calls"] - stats0.get(k, {}).get("calls", 0)) / args.steps,
                     "items_per_step": (v["items"] - stats0.get(k, {}).get("items", 0)) / args.steps}
                 for k, v in stats1.items()
                 if v["calls"] > stats0.get(k, {}).get("calls", 0)}
    pieces, out, _, _ = runs[-1]
    t_clouds = float(np.mean([r[2] for r in runs]))
    t_walk = float(np.mean([r[3] for r in runs]))
    n_joins = len(out.joins)
    point_passes = sum(len(pieces[j.moving].cloud) * (r.iterations + 1)
                       for j in out.joins for r in j.registrations)
    walked = [(j.fixed, j.moving) for j in out.joins]
    before = _edge_errors(poses, truth, walked, thick)
    after = _edge_errors(out.poses, truth, walked, thick)
    cpu = None
    if not args.no_cpu:
        oracle = importlib.import_module("oracle")
        first = out.joins[0]
        o_pieces = []
        t0 = time.perf_counter()
        for k in (first.fixed, first.moving):
            v, f = meshes[k]
            nrm = oracle.vertex_normals(v, f)
            o_pieces.append(oracle.cloud_from_indices(v, nrm, oracle.cap_selection(
                oracle.select_candidates(v, cents[k], frags[k].frac, frags[k].t, frags[k].res))))
        t_cloud_cpu = (time.perf_counter() - t0) / 2
        op = [None] * len(frags)
        op[first.fixed] = oracle.RefinePiece(frags[first.fixed].t, frags[first.fixed].res,
                                             o_pieces[0])
        op[first.moving] = oracle.RefinePiece(frags[first.moving].t, frags[first.moving].res,
                                              o_pieces[1])
        t0 = time.perf_counter()
        oj = oracle.refine_one(op, poses, first.fixed, first.moving, oracle.default_params())
        t_join_cpu = time.perf_counter() - t0
        assert oj.dist == first.dist
        vs = []
        for mine, theirs in zip(first.rungs, oj.rungs):
            r = mine[:3, :3].T @ theirs[:3, :3]
            vs.append([float(np.degrees(np.arccos(np.clip((np.trace(r) - 1) / 2, -1, 1)))),
                       float(np.linalg.norm(mine[:3, 3] - theirs[:3, 3]) / frags[first.moving].t)])
        cpu_stage = len(frags) * t_cloud_cpu + n_joins * t_join_cpu
        cpu = {"value": n_joins / cpu_stage, "unit": "joins/s",
               "cores": oracle.lib().or_default_threads(), "kind": "port",
               "sample": (f"the oracle on the walk's first join ({len(o_pieces[1].points)} source, "
                          f"{len(o_pieces[0].points)} target points; {t_join_cpu:.2f} s, each "
                          f"pass's searches on all threads) and its two fragments' clouds "
                          f"({t_cloud_cpu:.2f} s each, all threads), scaled to {len(frags)} "
                          f"clouds and {n_joins} joins"),
               "join_s": t_join_cpu, "cloud_s": t_cloud_cpu,
               "first_join_device_vs_oracle": {"rung_rot_deg_trans_t": vs,
                                               "fitness": [first.fitness, oj.fitness]}}
    line = {
        "metric": "refined joins/s (R 9 stage)", "value": n_joins / (t_clouds + t_walk),
        "unit": "joins/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * (t_clouds + t_walk), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": (f"{args.refine_workload}: {len(frags)} fragments "
                                f"({sum(len(f) for _, f in meshes)} faces), one group, "
                                f"{len(used)} joins in used order, poses perturbed 0.1 deg / 0.02 t"),
                   "cloud_points": [len(p.cloud) for p in pieces],
                   "timer": "host wall clock around the synchronous C-ABI calls (meshes and "
                            "clouds in from host memory, normals, indices and poses out)",
                   "generate_s": round(t_gen, 1)},
        "clouds_ms": 1000 * t_clouds, "walk_ms": 1000 * t_walk,
        "walk_joins_per_s": n_joins / t_walk,
        "point_passes_per_s": point_passes / t_walk,
        "iterations": [[r.iterations for r in j.registrations] for j in out.joins],
        "device_ms": device_ms,
        "perturbation": "0.1 deg about the fracture centroid and 0.02 t per fragment",
        "edge_error_before": {"rot_deg": before[0], "disp_t": before[1]},
        "edge_error_after": {"rot_deg": after[0], "disp_t": after[1]},
        "gpu_launches": int(args.steps * (device_ms.get("refine_join_rungs", {}).get(
            "items_per_step", 0) + 5 * n_joins + 3 * len(frags))),
        "gpu_launches_counts": ("k_wide_pass (one per pass), k_wide_reset and k_place_fused "
                                "(5 per join), k_incidence, k_vertex_normals and k_nn_below (3 per "
                                "fragment); the LBVH builds' and the radix sorts' own launches "
                                "are not counted"),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_stage1(args):
    """Stage 1 (R 5.1-5.5) of the reference's own slab pair (tests/golden/slab.npz, extracted
    from its fixture dump): 16 337 hypotheses scored on a 60-point probe, 250 kept and refined
    by two point-to-point rungs, re-scored, 10 kept. One step is the whole chain on the device
    (PairStage1.run with its own walk orders); the oracle runs the same chain on the CPU."""
    world, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    sherd = _pkg()
    st = _pkg("stage1")
    with np.load(ROOT / "tests" / "golden" / "slab.npz") as z:
        slab = {k: z[k] for k in z.files}

    def frames(name):
        g = lambda k: slab[f"{name}.{k}"]
        return st.Frames(p=g("brk_P"), ns=g("brk_ns"), f=g("brk_f"), dih=g("brk_dih"),
                         sub=g("brk_sub"))

    fa, fb = frames("pieceA"), frames("pieceB")
    ctx = sherd.Context(local)
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    pair = st.PairStage1(ctx, fa, fb, scales)
    for _ in range(args.warmup):
        pair.run(seed=args.seed)
    stats0 = ctx.stats()["methods"]
    sampler = ClockSampler(local)
    sampler.start()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = pair.run(seed=args.seed)
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    stats1 = ctx.stats()["methods"]
    device_ms = {k: (v["ms"] - stats0.get(k, {}).get("ms", 0.0)) / args.steps
                 for k, v in stats1.items() if v["calls"] > stats0.get(k, {}).get("calls", 0)}
    step = float(np.median(times))
    n_hyp = len(res.hypotheses)
    cpu = None
    if not args.no_cpu:
        oracle = importlib.import_module("oracle")
        a = {"p": fa.p, "ns": fa.ns, "f": fa.f, "dih": fa.dih}
        b = {"p": fb.p, "ns": fb.ns, "f": fb.f, "dih": fb.dih}
        osc = oracle.scales_from(slab["scales"])
        t0 = time.perf_counter()
        pa, pb, poses = oracle.hypotheses(a, b, fa.sub, fb.sub)
        idx = st.probe_draw(fb.sub, st.COARSE_POINTS, args.seed).astype(np.int64)
        target = oracle.Cloud(fa.p, fa.ns)
        cs = oracle.coarse_scores(target, fb.p[idx], fb.ns[idx], poses, osc.coarse)
        kept = oracle.nms(oracle.order_by_score(cs, oracle.COARSE_ORDER_LIMIT), poses, cs,
                          osc.nms, st.STAGE1, oracle.COARSE_FLOOR)
        sub = np.asarray(fb.sub, np.int64)
        refined = oracle.stage1_ladder(fb.p[sub], target, poses[kept.astype(np.int64)], osc)
        rescore = oracle.coarse_scores(target, fb.p[sub], fb.ns[sub], refined, osc.stage1)
        kept2 = oracle.nms(oracle.order_by_score(rescore), refined, rescore, osc.nms, st.STAGE2,
                           oracle.STAGE1_FLOOR)
        t_cpu = time.perf_counter() - t0
        same = (np.array_equal(kept, res.kept) and np.array_equal(kept2, res.kept2)
                and np.array_equal(cs, res.coarse))
        cpu = {"value": 1.0 / t_cpu, "unit": "pairs/s", "cores": oracle.lib().or_default_threads(),
               "kind": "port", "sample": f"the whole chain once, {t_cpu:.2f} s",
               "same_kept_lists_and_coarse_scores": bool(same)}
    line = {
        "metric": "stage-1 pairs/s (R 5.1-5.5)", "value": 1.0 / step, "unit": "pairs/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "the reference's slab fixture pair (tests/golden/slab.npz)",
        "config": {"workload": (f"slab pair: {n_hyp} hypotheses x {st.COARSE_POINTS} probe points, "
                                f"{len(res.kept)} refined (2 point-to-point rungs over "
                                f"{len(fb.sub)} points), {len(res.kept2)} starts"),
                   "timer": "host wall clock around the chain (median of the steps)"},
        "hypotheses_per_s": n_hyp / step,
        "device_ms": device_ms,
        "gpu_launches": args.steps * 8,
        "gpu_launches_counts": ("k_hyp_flags, the compaction, k_hyp_poses, k_coarse_scores, 2 "
                                "k_icp_rung, k_coarse_scores; the LBVH and cloud builds' own "
                                "launches not counted"),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_chain(args):
    """The matching stage from labelled meshes (pair.match_collection): every fragment's R 3.5
    arrays at its pairs' t, stage 1 per pair, one batched stage-2 call over every pair's starts,
    R 5.7 per pair, on a synthetic workload (default: the pot, all 28 pairs). One step is the
    whole stage. The line also scores the result against the generator's ground truth."""
    world, rank, local = _dist()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    sherd = _pkg()
    synth = _pkg("synth")
    pm = _pkg("pair")
    wl = synth.make(args.chain_workload, args.seed)
    frags = [pm.FragmentInput(fr.v.astype(np.float64), fr.f, fr.frac, float(fr.t), float(fr.res))
             for fr in wl.fragments]
    pairs = [(p.a, p.b) for p in wl.pairs]
    adjacent = np.array([p.adjacent for p in wl.pairs])
    ctx = sherd.Context(local)
    params = sherd.default_params()
    for _ in range(args.warmup):
        pm.match_collection(ctx, frags, pairs, params, seed=args.seed)
    sampler = ClockSampler(local)
    sampler.start()
    steps = []
    for _ in range(args.steps):
        timings = {}
        t0 = time.perf_counter()
        res = pm.match_collection(ctx, frags, pairs, params, seed=args.seed, timings=timings)
        steps.append((time.perf_counter() - t0, timings))
    clocks = sampler.stop()
    step = float(np.median([x for x, _ in steps]))
    phases = {k: float(np.median([t[k] for _, t in steps])) for k in steps[0][1]}
    accepted = np.array([bool(r.candidates) and bool(r.candidates[0].accepted) for r in res])
    errors = []
    for r, p in zip(res, wl.pairs):
        if p.adjacent and r.candidates and r.candidates[0].accepted:
            pose = np.array(r.candidates[0].rungs[3].transform[:]).reshape(4, 4)
            rr = pose[:3, :3].T @ p.truth[:3, :3]
            errors.append(float(np.degrees(np.arccos(np.clip((np.trace(rr) - 1) / 2, -1, 1)))))
    n_items = sum(len(r.stage1.starts) for r in res if r.stage1 is not None)
    line = {
        "metric": "pairs matched/s (R 3.5 + R 5, from labelled meshes)", "value": len(pairs) / step,
        "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": (f"{args.chain_workload}: {len(frags)} fragments, {len(pairs)} pairs, "
                                f"{n_items} stage-2 starts"),
                   "timer": "host wall clock around match_collection (median of the steps)"},
        "phases_s": phases,
        "accepted": {"true_joins": int((accepted & adjacent).sum()),
                     "adjacent_pairs": int(adjacent.sum()),
                     "false_joins": int((accepted & ~adjacent).sum()),
                     "best_rot_err_deg_median": float(np.median(errors)) if errors else None},
        "gpu_launches": None,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def _config_dict(wl, args):
    """The workload the line is quoted on; both arms print the same dictionary."""
    d = wl.describe()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"workload": f"{args.config}: {d['fragments']} fragments, {d['pairs']} pairs x "
                        f"{d['starts_per_pair']} starts = {d['items']} (pair, start) items",
            **d, "sched": args.sched,
            "l2": (f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MB write); the resident "
                   "fragment data also exceeds L2"),
            "parallelism": (f"{world} rank(s), one GPU each; the collection's pairs partitioned "
                            "over the ranks by estimated cost, each rank holding only its pairs' "
                            "fragments, one batched call per rank, one all-gather of candidate "
                            "records (strong scaling)")}


def _source_hash() -> str:
    """A digest of the CUDA sources, naming the build a recorded ncu capture belongs to."""
    import hashlib
    h = hashlib.sha256()
    for f in sorted((ROOT / "sherd-refit_b200" / "csrc").glob("*.cu*")):
        h.update(f.name.encode())
        h.update(f.read_bytes())
    return h.hexdigest()[:12]


def _plain_leg(ctx, sherd, dev, wl, params, n_pairs, full_cands):
    """SHERD_SCHED_PLAIN (one k_ladder + k_verify_items launch per pair, synchronised after each
    pair) on n_pairs pairs evenly spaced over the collection with all their starts, and the
    batched schedule on the same items, on the resident data (device time, CUDA events)."""
    workload = _pkg("workload")
    sub = np.unique(np.linspace(0, len(dev.pairs) - 1, n_pairs).round().astype(np.int64))
    pair, start, inits = workload.item_arrays(wl)
    where = np.full(len(dev.pairs), -1, np.int64)
    where[sub] = np.arange(len(sub))
    sel = np.flatnonzero(where[pair] >= 0)
    items = sherd.work_item_array(where[pair[sel]].astype(np.uint32), start[sel], inits[sel])
    pairs = [dev.pairs[k] for k in sub]
    out = {}
    for name, sched in (("plain", sherd.SCHED_PLAIN), ("batched", sherd.SCHED_BATCHED)):
        b = ctx.batch(pairs, items, params, sched)
        b.run()
        out[name] = (b.run()["total"], sherd.candidates(b.results()).copy())
        del b
    n = len(sel)
    plain_ms, plain_c = out["plain"]
    batched_ms, batched_c = out["batched"]
    want = full_cands[sel].copy()
    want["pair"] = where[want["pair"].astype(np.int64)]
    return {"value": n / (plain_ms / 1000.0), "unit": UNIT, "ms": plain_ms, "items": int(n),
            "pairs": int(len(sub)),
            "sample": (f"{len(sub)} of the {len(dev.pairs)} pairs, evenly spaced over the pair "
                       f"list, with all their starts ({n} items)"),
            "batched_same_items": {"value": n / (batched_ms / 1000.0), "ms": batched_ms},
            "batched_over_plain_same_items": plain_ms / batched_ms,
            "identical_candidates": bool(plain_c.tobytes() == batched_c.tobytes()
                                         == want.tobytes())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=("cuda", "reference"))
    ap.add_argument("--config", default="collection")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--sched", default="batched", choices=("batched", "plain"))
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-items", type=int, default=CPU_ITEMS)
    ap.add_argument("--plain-pairs", type=int, default=24)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--group-poses", type=int, default=4096)
    ap.add_argument("--refine-workload", default="scan")
    ap.add_argument("--chain-workload", default="pot")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.config == "group":
        run_group(args)
        return
    if args.config == "refine":
        run_refine(args)
        return
    if args.config == "stage1":
        run_stage1(args)
        return
    if args.config == "chain":
        run_chain(args)
        return

    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    sherd = _pkg()
    synth = _pkg("synth")
    workload = _pkg("workload")
    shard = _pkg("shard")
    t_gen = time.perf_counter()
    wl = synth.make(args.config, args.seed)
    t_gen = time.perf_counter() - t_gen
    mine = shard.rank_pairs(wl, rank, world) if world > 1 else None
    ctx = sherd.Context(local)
    params = sherd.default_params()
    t_up = time.perf_counter()
    dev = workload.to_device(ctx, wl, params, pairs=mine)
    t_up = time.perf_counter() - t_up
    sched = sherd.SCHED_BATCHED if args.sched == "batched" else sherd.SCHED_PLAIN
    batch = ctx.batch(dev.pairs, dev.items, params, sched)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        batch.run()

    sampler = ClockSampler(local)
    _barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    runs = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        runs.append(batch.run())
    torch.cuda.synchronize()
    _barrier(world)
    clocks = sampler.stop()
    stage_ms = {k: float(np.mean([r[k] for r in runs])) for k in runs[0]}
    step_ms = _max_over_ranks(world, stage_ms["total"])
    n_items = wl.n_items
    value = n_items / (step_ms / 1000.0)

    local_cands = sherd.candidates(batch.results()).copy()
    local_cands["pair"] = np.asarray(dev.pair_index)[local_cands["pair"].astype(np.int64)]
    sbytes = workload.stage_bytes(wl, local_cands)
    total_q = shard.sum_over_ranks(sbytes["ladder"] / 48.0, device="cuda")

    # End to end through the host-buffer C-ABI call: work items in from pinned host memory,
    # candidates out into pinned host memory (both buffers allocated once, as a caller that
    # runs step after step keeps them), then the one all-gather that puts every item's
    # candidate on every rank.
    def pinned(dtype, n):
        raw = torch.empty(max(n, 1) * dtype.itemsize, dtype=torch.uint8, pin_memory=True)
        return raw.numpy().view(dtype)[:n]

    items_host = pinned(sherd.WORK_ITEM, dev.n_items)
    items_host[:] = np.ctypeslib.as_array(dev.items)[:dev.n_items]
    cands_host = pinned(sherd.CANDIDATE, dev.n_items)
    e2e_ms = []
    for k in range(args.e2e_steps + 1):
        flush.zero_()
        torch.cuda.synchronize()
        _barrier(world)
        t0 = time.perf_counter()
        out = ctx.ladder_verify_batch(dev.pairs, items_host, params, sched, out=cands_host)
        full = shard.gather_candidates(wl, dev, out, device="cuda")
        t1 = time.perf_counter()
        if k:
            e2e_ms.append(1000 * (t1 - t0))
    e2e_step = _max_over_ranks(world, float(np.mean(e2e_ms)))
    h2d = dev.n_items * sherd.WORK_ITEM.itemsize
    d2h = dev.n_items * sherd.CANDIDATE.itemsize
    same = bytes(out) == bytes(batch.results())
    accepted = int(full["accepted"].sum())
    status_bad = int((full["status"] != 0).sum())

    peak, peak_kind = _peaks()
    kernel_of = {"ladder": "k_ladder", "verify": "k_verify_items", "pen_inside": "k_pen_inside",
                 "pen_min": "k_pen_seed + k_pen_min", "finalize": "k_pen_init + k_pen_finalize"}
    stages = {}
    for k, name in kernel_of.items():
        ms = stage_ms[k]
        stages[k] = {"kernel": name, "ms": ms, "algorithmic_bytes": sbytes[k],
                     "gbs": sbytes[k] / (ms / 1000.0) / 1e9 if ms > 0 else None}
    dom = max(("ladder", "verify", "pen_inside", "pen_min"), key=lambda k: stage_ms[k])
    achieved = stages[dom]["gbs"]
    src = _source_hash()
    rec = TRAFFIC.get((args.config, args.seed, kernel_of[dom], world))
    traffic = rec[0] if rec and rec[1] == src else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of the "
                                   f"stage's launches in one full-size step of this build (CUDA "
                                   f"sources {src})"
                                   if traffic else
                                   f"no ncu capture recorded for this build (CUDA sources {src})"),
                "kernel": stages[dom]["kernel"],
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "per_unit": ("48 B per ICP point-iteration (16 B source point + 32 B matched "
                             "target point and normal) over the passes each rung ran"
                             if dom == "ladder" else "24 B per query point"),
                "stages": stages}

    plain = None
    if world == 1 and not args.no_plain and sched == sherd.SCHED_BATCHED:
        plain = _plain_leg(ctx, sherd, dev, wl, params, args.plain_pairs, full)
        plain["value_over_plain"] = value / plain["value"]

    if rank != 0:
        ctx.close()
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    cpu, par = None, None
    if not args.no_cpu:
        cpu, par = cpu_baseline_and_parity(wl, args.cpu_items, full)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, sherd-refit_b200/synth.py)",
        "config": _config_dict(wl, args),
        "run": {"accepted": accepted, "item_errors": status_bad, "generate_s": round(t_gen, 1),
                "upload_s": round(t_up, 1),
                "rank_items": int(dev.n_items), "rank_pairs": len(dev.pairs)},
        "e2e": {"value": n_items / (e2e_step / 1000.0), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "timer": ("host wall clock around the synchronous C-ABI call (work items from "
                          "and candidates into pinned host buffers allocated once) and the "
                          "candidate all-gather (max over ranks); bytes per rank"),
                "matches_resident_run": same},
        "gpu_launches": 9 * args.steps,
        "gpu_launches_counts": ("per step: k_ladder once per point-count bucket (3), "
                                "k_verify_items, k_pen_init, k_pen_inside, k_pen_seed, k_pen_min, "
                                "k_pen_finalize"),
        "ladder_autotune": ctx.stats().get("ladder_autotune"),
        "nn_queries": nn_query_rates(sbytes, stage_ms, step_ms, total_q),
        "roofline": roofline,
        "plain": plain,
        "parity": par,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
