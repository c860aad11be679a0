"""R 3.4 segmentation on the device (sherd_segment) against the oracle and the fixture.

Every intermediate array is compared bit for bit with the oracle's sequential restatement:
the representatives and each face's, the smoothed normals, the votes, the raw, majority and
island masks, has_ref, and the final labels. On the slab the final labels also equal the
fixture's `seg.frac_final` face for face.
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest

from _slab import piece

pytestmark = pytest.mark.gpu

TRACE_KEYS = ("rep", "near", "ns", "good", "frac_raw", "frac_majority", "frac_islands", "has_ref")


def _compare(gpu, cpu):
    g_labels, g_info, g_tr = gpu
    c_labels, c_info, c_tr = cpu
    assert (g_info.votes, g_info.n_rep, g_info.smooth_radius, g_info.boundary_angle) == \
        (c_info.votes, c_info.n_rep, c_info.smooth_radius, c_info.boundary_angle)
    for k in TRACE_KEYS:
        assert np.array_equal(g_tr[k], c_tr[k]), k
    assert np.array_equal(g_labels, c_labels)


@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_segmentation_is_bit_exact_on_the_slab(sherd, gpu_ctx, oracle, slab, name):
    p = piece(slab, name)
    t, res = float(p["thick_t"]), float(p["res"])
    gpu = gpu_ctx.segment(gpu_ctx.mesh(p["V"], p["F"]), p["V"], p["F"], t, res, trace=True)
    cpu = oracle.segment(oracle.Mesh(p["V"], p["F"]), p["V"], p["F"], t, res)
    _compare(gpu, cpu)
    assert np.array_equal(gpu[0], p["frac"])


def test_segmentation_is_bit_exact_on_a_pot_fragment(sherd, gpu_ctx, oracle):
    synth = importlib.import_module("sherd-refit_b200.synth")
    wl = synth.make("pot", 0)
    for fr in wl.fragments[:2]:
        v = fr.v.astype(np.float64)
        gpu = gpu_ctx.segment(gpu_ctx.mesh(fr.v, fr.f), v, fr.f, fr.t, fr.res, trace=True)
        cpu = oracle.segment(oracle.Mesh(fr.v, fr.f), v, fr.f, fr.t, fr.res)
        _compare(gpu, cpu)
        # The generator's own fracture faces: the segmentation finds most of them.
        truth = fr.frac.astype(bool)
        assert np.mean(gpu[0].astype(bool) == truth) > 0.8


def test_segmentation_options_and_refusals(sherd, gpu_ctx, oracle, slab):
    p = piece(slab, "pieceA")
    mesh = gpu_ctx.mesh(p["V"], p["F"])
    t, res = float(p["thick_t"]), float(p["res"])
    params = sherd.seg_params_default()
    params.boundary_angle_auto = 1
    params.smoothed_hit_normal = 1
    gpu = gpu_ctx.segment(mesh, p["V"], p["F"], t, res, params, trace=True)
    o = oracle.seg_params(boundary_angle_auto=1, smoothed_hit_normal=1)
    cpu = oracle.segment(oracle.Mesh(p["V"], p["F"]), p["V"], p["F"], t, res, o)
    _compare(gpu, cpu)
    labels, info = gpu_ctx.segment(mesh, p["V"], p["F"], 0.0, res)
    assert not labels.any()
    with pytest.raises(sherd.SherdError):
        gpu_ctx.segment(mesh, p["V"], p["F"][:-1], t, res)
