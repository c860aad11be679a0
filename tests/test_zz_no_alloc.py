"""The allocation-free ICP rung (sherd_icp_rung_noalloc) against sherd_icp_rung.

Some callers cannot allocate device memory in the middle of a run: a worker held to a device
memory budget fixed up front, or code that must not call cudaMalloc/cudaFree while other
streams are in flight, because both can block or synchronise the whole device. For them the
rung keeps its per-point working memory in one fixed array inside the library and takes inputs
and outputs that already live on the device. Here the test itself allocates those buffers
(with torch) and checks two calls in a row against the allocating entry point, within the
tolerance the other ICP tests use (1e-6 t and 1e-4 degrees on at least 8 of the 10 starts).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from _slab import origin_t, piece, trace_deg

pytestmark = pytest.mark.gpu


def _call(sherd, ctx, src, n, target, inits, k, opt, out):
    return sherd.lib().sherd_icp_rung_noalloc(ctx.h, C.c_void_p(src), n, target.h,
                                              C.c_void_p(inits), k, opt, C.c_void_p(out))


@pytest.mark.parametrize("estimation", [1, 0], ids=["point_to_plane", "point_to_point"])
def test_the_allocation_free_rung_matches_the_allocating_one(sherd, gpu_ctx, slab, estimation):
    import torch

    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    target = gpu_ctx.cloud(a["reg_p"], a["reg_n"])
    t, icp = float(slab["scales"][0]), float(slab["scales"][11])
    dist = 0.2 * t * icp
    starts = np.ascontiguousarray(slab["starts"].reshape(-1, 16))
    k, n = len(starts), len(b["reg_p"])
    expected = gpu_ctx.icp_rung(b["reg_p"], target, starts, dist, 30, estimation=estimation)

    src = np.zeros((n, 4))
    src[:, :3] = b["reg_p"]
    d_src = torch.from_numpy(src).cuda()
    d_inits = torch.from_numpy(starts.copy()).cuda()
    d_out = torch.empty(C.sizeof(sherd.Registration) * k, dtype=torch.uint8, device="cuda")
    opt = sherd.IcpOptions(estimation, 30, dist)
    calls = []
    for _ in range(2):
        d_out.fill_(0xFF)
        torch.cuda.synchronize()
        rc = _call(sherd, gpu_ctx, d_src.data_ptr(), n, target, d_inits.data_ptr(), k, opt,
                   d_out.data_ptr())
        assert rc == 0, sherd.lib().sherd_last_error(gpu_ctx.h)
        host = d_out.cpu().numpy().tobytes()
        calls.append((sherd.Registration * k).from_buffer_copy(host))

    for regs in calls:
        close = 0
        for got, want in zip(regs, expected):
            pg, pw = got.pose(), want.pose()
            if origin_t(pg, pw, t) < 1e-6 and trace_deg(pg, pw) < 1e-4:
                close += 1
                assert got.correspondences == want.correspondences
        assert close >= 8, close
    assert bytes(calls[0]) == bytes(calls[1])


def test_the_allocation_free_rung_refuses_what_it_cannot_hold(sherd, gpu_ctx, slab):
    import torch

    a, b = piece(slab, "pieceA"), piece(slab, "pieceB")
    target = gpu_ctx.cloud(a["reg_p"], a["reg_n"])
    n = len(b["reg_p"])
    d_src = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    d_inits = torch.zeros((1, 16), dtype=torch.float64, device="cuda")
    d_out = torch.empty(C.sizeof(sherd.Registration), dtype=torch.uint8, device="cuda")
    opt = sherd.IcpOptions(1, 30, 1.0)
    too_many = (1 << 20) // n + 1  # the capacity is k * n_source <= 2^20
    rc = _call(sherd, gpu_ctx, d_src.data_ptr(), n, target, d_inits.data_ptr(), too_many, opt,
               d_out.data_ptr())
    assert rc == -1
    assert b"SHERD_NOALLOC_CAPACITY" in sherd.lib().sherd_last_error(gpu_ctx.h)
    rc = _call(sherd, gpu_ctx, d_src.data_ptr() + 8, n, target, d_inits.data_ptr(), 1, opt,
               d_out.data_ptr())
    assert rc == -1
    # Misaligned poses or records, and host memory, are refused on the host before a launch.
    rc = _call(sherd, gpu_ctx, d_src.data_ptr(), n, target, d_inits.data_ptr() + 4, 1, opt,
               d_out.data_ptr())
    assert rc == -1 and b"aligned" in sherd.lib().sherd_last_error(gpu_ctx.h)
    rc = _call(sherd, gpu_ctx, d_src.data_ptr(), n, target, d_inits.data_ptr(), 1, opt,
               d_out.data_ptr() + 4)
    assert rc == -1 and b"aligned" in sherd.lib().sherd_last_error(gpu_ctx.h)
    host_inits = np.zeros(16)
    rc = _call(sherd, gpu_ctx, d_src.data_ptr(), n, target, host_inits.ctypes.data, 1, opt,
               d_out.data_ptr())
    assert rc == -1 and b"device" in sherd.lib().sherd_last_error(gpu_ctx.h)
