"""The C ABI library on a host without a GPU: it loads, exports every symbol the header
declares, and its host-only functions answer (no compute call needs a device here)."""

from __future__ import annotations

import re
from pathlib import Path

import numpy as np

HEADER = Path(__file__).resolve().parent.parent / "include" / "sherd_cuda.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sherd_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(sherd):
    lib = sherd.lib()
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(sherd.exported_symbols()) == names


def test_the_backend_names_itself(sherd):
    assert sherd.lib().sherd_name() == b"cuda"


def test_scales_for_pair_reproduces_the_fixture_bit_for_bit(sherd, slab):
    """Scales::for_pair (scales.rs:72-88) at the slab pair's t and res gives scales.json."""
    p = sherd.default_params()
    sc = sherd.scales_for_pair(p, slab["scales"][0], slab["scales"][1])
    got = np.array([getattr(sc, k) for k, _ in sherd.Scales._fields_])
    assert np.array_equal(got, slab["scales"])


def test_thin_walls_activate_the_resolution_floor(sherd):
    """scales.rs:117-160: at 4-6 edges per t the m*res term wins."""
    p = sherd.default_params()
    t = 2.0
    res = t / 5.0
    sc = sherd.scales_for_pair(p, t, res)
    assert sc.tight == 0.15 * res and sc.tight > 0.01 * t
    assert sc.icp == (0.6 * res) / (0.04 * t) and sc.icp > 1.0
    thick = sherd.scales_for_pair(p, 39.0, 0.058 * 39.0)
    assert abs(thick.coarse - 0.15 * 39.0) < 1e-12 and thick.icp == 1.0


def test_accept_reads_the_five_limits(sherd):
    p = sherd.default_params()
    sc = sherd.scales_for_pair(p, 10.0, 0.5)
    s = sherd.Scores(tight=0.3, gap=0.01, pen=0.0, seam=4.0, cont_n=0.9)
    assert sherd.accept(s, p, sc)
    for field, value in (("tight", 0.2), ("gap", 0.05), ("pen", 0.01), ("seam", 2.0),
                         ("cont_n", 0.5), ("tight", float("nan"))):
        bad = sherd.Scores(tight=0.3, gap=0.01, pen=0.0, seam=4.0, cont_n=0.9)
        setattr(bad, field, value)
        assert not sherd.accept(bad, p, sc), field


def test_struct_layouts_match_the_header(sherd):
    """executor/batch.rs:591-653's layout assertions, for the ABI's POD types."""
    import ctypes as C
    assert C.sizeof(sherd.InsideOutcome) == 8
    assert C.sizeof(sherd.Registration) == 16 * 8 + 8 + 8 + 8 + 4 + 4
    assert C.sizeof(sherd.Scales) == 12 * 8
    assert C.sizeof(sherd.WorkItem) == 8 + 128
    assert C.sizeof(sherd.Scores) == 16 * 8 + 8 + 16


def test_opening_without_a_device_fails_loudly(sherd):
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(sherd.SherdError):
        sherd.Context(0)
