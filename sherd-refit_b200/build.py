"""Build recipe of the CUDA backend: csrc/sherd.cu -> _lib/libsherd_cuda.so (sm_100a).

nvcc cross-compiles for the B200 without a GPU present. Flags:
  -gencode arch=compute_100a,code=sm_100a   Blackwell datacenter SASS only
  -fmad=false                               no multiply-add contraction anywhere: the hit
                                            distances, point-to-triangle distances and f64
                                            point loops are the same IEEE operations, in the
                                            same order, as the CPU oracle and the reference
  -lineinfo                                 source lines for ncu
The library is built in-tree so it travels with the repository to the GPU hosts.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
OUT = HERE / "_lib" / "libsherd_cuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
    "-Xptxas", "-v",
]


def sources():
    return sorted(SRC.glob("*.cu")) + sorted(SRC.glob("*.cuh")) + [
        HERE.parent / "include" / "sherd_cuda.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library unless it is newer than every source."""
    if not force and OUT.exists():
        newest = max(p.stat().st_mtime for p in sources())
        if OUT.stat().st_mtime >= newest:
            return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [NVCC, *FLAGS, str(SRC / "sherd.cu"), "-o", str(tmp)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    log = OUT.parent / "ptxas.log"
    log.write_text(proc.stdout + proc.stderr)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc failed ({proc.returncode}); see {log}")
    if verbose:
        sys.stdout.write(proc.stdout + proc.stderr)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
