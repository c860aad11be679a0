"""The checker of the batched path's candidates (oracle/parity.py) on planted answers, on the CPU.

A check that cannot fail is no evidence: each planted difference below must be caught, and the
one-ULP chaos probe must excuse only what it is told is chaotic.
"""

from __future__ import annotations

import importlib

import numpy as np


def _cands(n, seed=0):
    backend = importlib.import_module("sherd-refit_b200.backend")
    rng = np.random.default_rng(seed)
    c = np.zeros(n, backend.CANDIDATE)
    for k in range(n):
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        th = rng.uniform(0, 0.5)
        kx = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        r = np.eye(3) + np.sin(th) * kx + (1 - np.cos(th)) * kx @ kx
        pose = np.eye(4)
        pose[:3, :3] = r
        pose[:3, 3] = rng.normal(size=3) * 50
        c["rungs"]["transform"][k, 3] = pose.reshape(16)
    c["pair"] = np.arange(n) // 8
    c["accepted"] = np.arange(n) % 3 == 0
    return c


def test_identical_candidates_pass_and_planted_differences_fail():
    parity = importlib.import_module("oracle.parity")
    ref = _cands(32)
    t = np.full(32, 8.0)
    centre = np.tile([10.0, -20.0, 5.0], (32, 1))
    res = parity.compare(ref.copy(), ref, t, centre, pair_ids=ref["pair"])
    assert res["ok"] and res["bit_identical_candidates"] == 32 and res["rot_rad"]["max"] == 0.0
    assert res["pairs_with_share"] == 4 and res["chaotic_share_worst_pair"] == 0.0
    # a translation 2e-4 t off at one item
    g = ref.copy()
    g["rungs"]["transform"][5, 3, 3] += 2e-4 * 8.0
    res = parity.compare(g, ref, t, centre, pair_ids=ref["pair"])
    assert not res["ok"] and res["determined_past_bound"] == 1
    # a rotation 2e-5 rad off
    g = ref.copy()
    th = 2e-5
    rz = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    pose = g["rungs"]["transform"][7, 3].reshape(4, 4).copy()
    pose[:3, :3] = rz @ pose[:3, :3]
    g["rungs"]["transform"][7, 3] = pose.reshape(16)
    res = parity.compare(g, ref, t, np.zeros((32, 3)), pair_ids=ref["pair"])
    assert not res["ok"] and res["rot_rad"]["max"] > 1e-5
    # a flipped verdict
    g = ref.copy()
    g["accepted"][3] ^= 1
    res = parity.compare(g, ref, t, centre, pair_ids=ref["pair"])
    assert not res["ok"] and res["determined_verdict_mismatch"] == 1


def test_the_chaos_probe_excuses_only_what_it_finds_chaotic():
    parity = importlib.import_module("oracle.parity")
    ref = _cands(32)
    t = np.full(32, 8.0)
    centre = np.zeros((32, 3))
    g = ref.copy()
    g["rungs"]["transform"][[1, 9, 17], 3, 3] += 1.0
    res = parity.compare(g, ref, t, centre, pair_ids=ref["pair"],
                         probe=lambda m: np.zeros(int(m.sum()), bool))
    assert res["ok"] and res["chaotic"] == 3 and res["chaotic_share_worst_pair"] == 1 / 8
    res = parity.compare(g, ref, t, centre, pair_ids=ref["pair"],
                         probe=lambda m: np.ones(int(m.sum()), bool))
    assert not res["ok"] and res["determined_past_bound"] == 3
    # more than 0.4 of a pair excused is a failure
    g = ref.copy()
    g["rungs"]["transform"][:4, 3, 3] += 1.0
    res = parity.compare(g, ref, t, centre, pair_ids=ref["pair"],
                         probe=lambda m: np.zeros(int(m.sum()), bool))
    assert not res["ok"] and res["chaotic_share_worst_pair"] == 0.5


def test_nudged_inits_move_one_entry_by_one_ulp():
    parity = importlib.import_module("oracle.parity")
    init = np.arange(16, dtype=np.float64).reshape(4, 4) + 0.5
    out = parity.nudged_inits(init)
    assert out.shape == (12, 4, 4)
    for k in range(12):
        i, j = divmod(k, 4)
        d = out[k] != init
        assert d.sum() == 1 and d[i, j] and out[k, i, j] == np.nextafter(init[i, j], np.inf)
