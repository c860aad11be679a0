"""Shared fixtures: the golden slab vectors, the oracle and (on a GPU host) the CUDA backend."""

from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

from _slab import piece

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden" / "slab.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def slab():
    """The reference's slab fixture, as extracted by tests/golden/make_golden.py."""
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle():
    return importlib.import_module("oracle")


def package():
    """The product package (its directory name carries a hyphen, so it is imported by name)."""
    return importlib.import_module("sherd-refit_b200")


@pytest.fixture(scope="session")
def sherd():
    return package()


@pytest.fixture(scope="session")
def gpu_ctx(sherd):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    return sherd.Context(0)


@pytest.fixture(scope="session")
def gpu_slab(sherd, gpu_ctx, slab):
    """Device meshes, surfaces, clouds and the pair of the slab, built once."""
    out = {}
    for name in ("pieceA", "pieceB"):
        p = piece(slab, name)
        mesh = gpu_ctx.mesh(p["V"], p["F"])
        frac = mesh.subset(p["frac"])
        surf = gpu_ctx.surfaces(frac, mesh, int(p["watertight"]), float(p["frac_area"]), p["Pf"],
                                p["S"], p["brk_P"], p["brk_ns"], p["margin_p"], p["margin_n"])
        out[name] = dict(mesh=mesh, frac=frac, surf=surf, arrays=p)
    a, b = out["pieceA"], out["pieceB"]
    reg_t = gpu_ctx.cloud(a["arrays"]["reg_p"], a["arrays"]["reg_n"])
    frac_t = gpu_ctx.cloud(a["arrays"]["frac_p"], a["arrays"]["frac_n"])
    scales = sherd.Scales(*[float(x) for x in slab["scales"]])
    pair = gpu_ctx.pair(a["surf"], b["surf"], reg_t, frac_t, b["arrays"]["reg_p"],
                        b["arrays"]["frac_p"], scales)
    return dict(a=a, b=b, reg_t=reg_t, frac_t=frac_t, scales=scales, pair=pair)
