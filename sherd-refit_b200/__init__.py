"""sherd-refit B200 backend: the geometry hot path of sherd-refit on sm_100a CUDA kernels.

The package wraps the C ABI of include/sherd_cuda.h (built into `_lib/libsherd_cuda.so`):
device LBVHs over fragment meshes and point clouds, first-hit and parity rays, bounded
point-to-mesh distances, exact nearest neighbours, the point-to-plane ICP ladder, the R 6
verification and the batched persistent stage-2 path, plus the differentiable pose objective
(`adjoint`). Around it, with the reference's names: `preprocess` (R 3.5 breaklines and samples
of a labelled mesh), `stage1` (R 5.1-5.5), `pair` (`match_pair` through R 5.7), `refine`
(R 9's join refinement) and `read_mesh` (PLY). There is no CPU fallback: if the library is
missing, using it raises.
"""

from ._abi import (AdjointOptions, Candidate, IcpOptions, InsideOutcome, Params, Registration,
                   Scales, Scores, SegInfo, SegParams, SherdError, WorkItem, REDUCE_ALL,
                   REDUCE_MIN, SCHED_BATCHED, SCHED_PLAIN, exported_symbols, lib)
from .backend import (CANDIDATE, WORK_ITEM, Batch, Cloud, CoarseBatch, Context, CudaExecutor,
                      DistBatch, IcpBatch, InsideBatch, Mesh, Pair, Surfaces, accept, candidates,
                      default_params, read_mesh, scales_for_pair, work_item_array, work_items)

__all__ = [
    "AdjointOptions", "Batch", "CANDIDATE", "WORK_ITEM", "candidates", "work_item_array",
    "Candidate", "Cloud", "CoarseBatch", "Context", "CudaExecutor", "DistBatch", "IcpBatch",
    "IcpOptions",
    "InsideBatch", "InsideOutcome", "Mesh", "Pair", "Params", "Registration", "Scales", "Scores",
    "SegInfo", "SegParams", "SherdError", "Surfaces", "WorkItem", "REDUCE_ALL", "REDUCE_MIN", "SCHED_BATCHED",
    "SCHED_PLAIN", "accept", "default_params", "exported_symbols", "lib", "read_mesh",
    "scales_for_pair",
    "seg_params_default", "work_items",
]


def seg_params_default() -> SegParams:
    """SegParams::default (fragment/segment.rs:107-118), from the library."""
    p = SegParams()
    lib().sherd_seg_params_default(p)
    return p
