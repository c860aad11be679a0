"""R 3.5 (fragment/breakline.rs, fragment/samples.rs): breaklines, frames and samples of a labelled
working mesh, against the slab fixture's md.* arrays at the pair's t.

The oracle reproduces the fixture's breakline points, validity and subset exactly, the macro
normals, frames and dihedrals to 1e-12 (the reference summed its balls in an unspecified
order), and every sample array bit for bit: the reference draws from one numpy default_rng(seed)
per fragment (samples.rs:33-42), and so do the oracle and the package. On the device the
breakline arrays equal the oracle's bit for bit (dihedrals to the device's acos), and the whole
native chain (labelled meshes -> R 3.5 -> stage 1 -> stage 2 -> R 5.7) finds the fixture's
accepted join.
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest

from _slab import origin_t, piece, trace_deg

MD = ("t", "seed", "surface_points", "frac_per_t2", "min_frac_points", "max_frac_points",
      "margin_points", "macro_inner", "macro_outer", "brk_voxel")


def _md(p):
    return dict(zip(MD, (float(x) for x in p["md_params"])))


def _pre():
    return importlib.import_module("sherd-refit_b200.preprocess")


class _OracleDevice:
    """The Context calls preprocess.py and stage1.py make, answered by the oracle."""

    def __init__(self, oracle):
        self.o = oracle

    def face_geometry(self, v, f):
        return self.o.face_geometry(v, f)

    def breaklines(self, v, f, frac, t, macro_inner=0.15, macro_outer=0.6, brk_voxel=0.5):
        return self.o.breaklines(v, f, frac, t, macro_inner, macro_outer, brk_voxel)

    def cloud(self, p, n=None):
        return self.o.Cloud(p, n)

    def hypotheses_coarse(self, fa, fb, ia, ib, tol, target, q, qn, delta, agree=0.7):
        d = lambda fr: {"p": fr.p, "ns": fr.ns, "f": fr.f, "dih": fr.dih}
        pa, pb, poses = self.o.hypotheses(d(fa), d(fb), ia, ib, tol)
        return pa, pb, poses, self.o.coarse_scores(target, q, qn, poses, delta, agree)

    def icp_rung(self, source, target, inits, distance, max_iteration=30, estimation=1):
        A = importlib.import_module("sherd-refit_b200._abi")
        regs = self.o.icp_rung(source, target, inits, distance, max_iteration,
                               point_to_point=estimation == A.POINT_TO_POINT)
        return [A.Registration.from_buffer_copy(r) for r in regs]

    def icp_rung_array(self, *a, **k):
        regs = self.icp_rung(*a, **k)
        rec = importlib.import_module("sherd-refit_b200.backend").REGISTRATION
        return np.frombuffer(b"".join(bytes(r) for r in regs), rec)

    def coarse_scores(self, target, points, normals, poses, radius, normal_agree=0.7):
        return self.o.coarse_scores(target, points, normals, poses, radius, normal_agree)

    def ladder_verify_batch(self, pairs, items, params, sched=0):
        import ctypes as C
        A = importlib.import_module("sherd-refit_b200._abi")
        w = [self.o.WorkItem(p, s, (C.c_double * 16)(*np.ravel(t))) for p, s, t in items]
        out, _ = self.o.ladder_verify_batch(pairs, w, self.o.Params.from_buffer_copy(params))
        return [A.Candidate.from_buffer_copy(c) for c in out]


def _check_breaklines(b, p, exact_normals=False):
    assert np.array_equal(b["p"], p["brk_P"])
    assert np.array_equal(np.asarray(b["valid"]).astype(bool), p["brk_valid"].astype(bool))
    assert np.array_equal(np.sort(b["sub"]), np.sort(p["brk_sub"]))
    tol = 0.0 if exact_normals else 1e-12
    for k, ref in (("ns", "brk_ns"), ("nf", "brk_nf"), ("f", "brk_f")):
        assert np.abs(b[k] - p[ref]).max() <= tol, k
    assert np.abs(b["dih"] - p["brk_dih"]).max() <= 1e-9


# ---- the oracle, pinned ---------------------------------------------------------------------


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_oracle_breaklines_are_the_fixtures(oracle, slab, name):
    p = piece(slab, name)
    md = _md(p)
    b = oracle.breaklines(p["V"], p["F"], p["frac"], md["t"], md["macro_inner"],
                          md["macro_outer"], md["brk_voxel"])
    _check_breaklines(b, p)


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_oracle_samples_are_the_fixtures(oracle, slab, name):
    p = piece(slab, name)
    md = _md(p)
    s = oracle.samples(p["V"], p["F"], p["frac"], p["brk_P"], md["t"], int(md["seed"]),
                       int(md["surface_points"]), md["frac_per_t2"], int(md["min_frac_points"]),
                       int(md["max_frac_points"]), int(md["margin_points"]))
    assert np.array_equal(s["S"], p["S"]) and np.array_equal(s["Pf"], p["Pf"])
    assert np.array_equal(s["sp"], p["sp"]) and np.array_equal(s["fp"], p["fp"])
    assert np.array_equal(np.stack([s["S_u"], s["S_v"]]), p["S_uv"])
    assert np.array_equal(np.stack([s["Pf_u"], s["Pf_v"]]), p["Pf_uv"])
    assert np.array_equal(s["margin_idx"], p["margin_idx"])
    assert np.array_equal(s["S"][s["margin_idx"]], p["margin_p"])


def test_counts_and_splits():
    """samples.rs:250-268 and 601-618: the fracture count's clip (a NaN density takes the lower
    bound) and the registration split's round-half-even."""
    pre = _pre()
    assert pre.fracture_count(100.0, 1.0) == 12000 and pre.fracture_count(1.0, 1.0) == 5000
    assert pre.fracture_count(50.0, 1.0) == 7500
    assert pre.fracture_count(float("nan"), 1.0) == 5000
    assert pre.registration_split(10, 5, 0) == (10, 5)
    assert pre.registration_split(10, 5, 20) == (10, 5)
    assert pre.registration_split(5000, 6000, 6000) == (2727, 3273)
    assert pre.registration_split(3, 3, 3) == (2, 1)       # 1.5 rounds to even 2


def test_package_match_data_on_the_oracle(oracle, slab):
    """preprocess.match_data over an oracle-backed context: the fixture's samples and registration
    clouds bit for bit, and its breakline to 1e-12."""
    pre = _pre()
    dev = _OracleDevice(oracle)
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        md = pre.match_data(dev, p["V"], p["F"], p["frac"], _md(p)["t"], 0)
        assert np.array_equal(md.samples.pf, p["Pf"]) and np.array_equal(md.samples.s, p["S"])
        assert np.array_equal(md.margin_p, p["margin_p"]) and np.array_equal(md.margin_n, p["margin_n"])
        assert np.array_equal(md.reg_p, p["reg_p"]) and np.array_equal(md.reg_n, p["reg_n"])
        assert np.array_equal(md.pf_n, p["frac_n"])
        assert md.frac_area == float(p["frac_area"])
        _check_breaklines({"p": md.brk.p, "ns": md.brk.ns, "nf": md.brk.nf, "f": md.brk.f,
                           "valid": md.brk.valid, "sub": md.brk.sub, "dih": md.brk.dih}, p)


def test_native_stage1_on_the_oracle_finds_the_seam(sherd, oracle, slab):
    """From the labelled working meshes alone: R 3.5 at the pair's t, then stage 1 on the native
    frames (ascending subsets, stable orders) keeps the start the fixture's accepted join came
    from."""
    pre = _pre()
    st = importlib.import_module("sherd-refit_b200.stage1")
    dev = _OracleDevice(oracle)
    mds = [pre.match_data(dev, piece(slab, n)["V"], piece(slab, n)["F"], piece(slab, n)["frac"],
                          float(slab["scales"][0]), 0) for n in ("pieceA", "pieceB")]
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    res = st.PairStage1(dev, mds[0].frames, mds[1].frames, scales).run(seed=0)
    t = scales.t
    accepted = slab["starts"][int(np.argmax(slab["s2_accepted"]))]
    assert min(trace_deg(s, accepted) + origin_t(s, accepted, t) for s in res.starts) < 0.05


def test_native_pair_chain_on_the_oracle_accepts_the_fixtures_join(sherd, oracle, slab):
    """Labelled working meshes in, R 5.7's candidates out, every array built by the package over
    an oracle-backed context: the best candidate is the fixture's accepted join."""
    pre = _pre()
    st = importlib.import_module("sherd-refit_b200.stage1")
    pm = importlib.import_module("sherd-refit_b200.pair")
    dev = _OracleDevice(oracle)
    t = float(slab["scales"][0])
    mds, surf = [], []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        md = pre.match_data(dev, p["V"], p["F"], p["frac"], t, 0)
        mesh = oracle.Mesh(p["V"], p["F"])
        fm = mesh.subset(p["frac"])
        surf.append((mesh, fm, oracle.Surfaces(fm, mesh, int(p["watertight"]), md.frac_area,
                                               md.samples.pf, md.samples.s, md.brk.p, md.brk.ns,
                                               md.margin_p, md.margin_n)))
        mds.append(md)
    a, b = mds
    sc = oracle.scales_from(slab["scales"])
    pair = oracle.Pair(surf[0][2], surf[1][2], oracle.Cloud(a.reg_p, a.reg_n),
                       oracle.Cloud(a.samples.pf, a.pf_n), b.reg_p, b.samples.pf, sc)
    params = sherd.default_params()
    for k, val in zip(("min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n"), slab["params"]):
        setattr(params, k, float(val))
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    res = pm.match_pair(dev, pair, st.PairStage1(dev, a.frames, b.frames, scales), params)
    best = np.array(res.candidates[0].rungs[3].transform[:]).reshape(4, 4)
    assert res.candidates[0].accepted == 1
    assert trace_deg(best, slab["result_T"][0]) <= 0.05
    assert origin_t(best, slab["result_T"][0], t) <= 0.01


# ---- on the device -----------------------------------------------------------------------------


@pytest.mark.gpu
def test_device_breaklines_equal_the_oracles(gpu_ctx, oracle, slab):
    synth = importlib.import_module("sherd-refit_b200.synth")
    cases = [(piece(slab, n)["V"], piece(slab, n)["F"], piece(slab, n)["frac"],
              _md(piece(slab, n))["t"]) for n in ("pieceA", "pieceB")]
    fr = synth.make("pot", 0).fragments[1]
    cases.append((fr.v.astype(np.float64), fr.f, fr.frac, fr.t))
    for v, f, frac, t in cases:
        got = gpu_ctx.breaklines(v, f, frac, t)
        want = oracle.breaklines(v, f, frac, t)
        for k in ("p", "ns", "nf", "f", "sub"):
            assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(got["valid"], want["valid"])
        assert np.abs(got["dih"] - want["dih"]).max() <= 1e-12
    # The fixture's own arrays on the slab.
    p = piece(slab, "pieceB")
    _check_breaklines(gpu_ctx.breaklines(p["V"], p["F"], p["frac"], _md(p)["t"]), p)


@pytest.mark.gpu
def test_device_match_data_is_the_fixtures(gpu_ctx, slab):
    pre = _pre()
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        md = pre.match_data(gpu_ctx, p["V"], p["F"], p["frac"], _md(p)["t"], 0)
        assert np.array_equal(md.samples.pf, p["Pf"]) and np.array_equal(md.samples.s, p["S"])
        assert np.array_equal(md.reg_p, p["reg_p"]) and np.array_equal(md.margin_n, p["margin_n"])
        assert np.array_equal(np.sort(md.brk.sub), np.sort(p["brk_sub"]))


@pytest.mark.gpu
def test_device_native_pair_chain_accepts_the_fixtures_join(sherd, gpu_ctx, oracle, slab):
    """Labelled working meshes in, R 5.7's candidates out, every array built here: the best
    candidate is accepted and is the fixture's accepted join."""
    pre = _pre()
    st = importlib.import_module("sherd-refit_b200.stage1")
    pm = importlib.import_module("sherd-refit_b200.pair")
    t = float(slab["scales"][0])
    mds, surf = [], []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        md = pre.match_data(gpu_ctx, p["V"], p["F"], p["frac"], t, 0)
        mesh = gpu_ctx.mesh(p["V"], p["F"])
        fm = mesh.subset(p["frac"])
        surf.append((mesh, fm, gpu_ctx.surfaces(fm, mesh, int(p["watertight"]), md.frac_area,
                                                md.samples.pf, md.samples.s, md.brk.p,
                                                md.brk.ns, md.margin_p, md.margin_n)))
        mds.append(md)
    a, b = mds
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    reg_t = gpu_ctx.cloud(a.reg_p, a.reg_n)
    frac_t = gpu_ctx.cloud(a.samples.pf, a.pf_n)
    pair = gpu_ctx.pair(surf[0][2], surf[1][2], reg_t, frac_t, b.reg_p, b.samples.pf, scales)
    params = sherd.default_params()
    for k, val in zip(("min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n"), slab["params"]):
        setattr(params, k, float(val))
    res = pm.match_pair(gpu_ctx, pair, st.PairStage1(gpu_ctx, a.frames, b.frames, scales), params)
    best = np.array(res.candidates[0].rungs[3].transform[:]).reshape(4, 4)
    assert res.candidates[0].accepted == 1
    assert trace_deg(best, slab["result_T"][0]) <= 0.2 and origin_t(best, slab["result_T"][0], t) <= 0.05


@pytest.mark.gpu
def test_device_match_collection_accepts_the_fixtures_join(sherd, gpu_ctx, slab):
    """pair.match_collection on the device from the two labelled slab meshes: the pair's best
    candidate is the fixture's accepted join."""
    pm = importlib.import_module("sherd-refit_b200.pair")
    params = sherd.default_params()
    for k, val in zip(("min_tight", "max_gap", "max_pen", "min_seam", "min_cont_n"), slab["params"]):
        setattr(params, k, float(val))
    frags = []
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        frags.append(pm.FragmentInput(p["V"], p["F"], p["frac"], float(p["thick_t"]),
                                      float(p["res"]), bool(p["watertight"])))
    (res,) = pm.match_collection(gpu_ctx, frags, [(0, 1)], params)
    best = np.array(res.candidates[0].rungs[3].transform[:]).reshape(4, 4)
    t = float(slab["scales"][0])
    assert res.candidates[0].accepted == 1
    assert trace_deg(best, slab["result_T"][0]) <= 0.2 and origin_t(best, slab["result_T"][0], t) <= 0.05
