"""Build recipe of the oracle: oracle.cpp -> oracle/_build/liboracle.so.

The oracle is test infrastructure (the checker the CUDA backend is compared against). It is
compiled with -ffp-contract=off so that, like the reference's Rust, it never fuses a multiply
into an add, and without -march=native so the library built here also loads on the GPU hosts.

The reference's own CPU backend is Rust (crates/sherd-core) and cannot be compiled in this
environment (no cargo/rustc, no network), so there is no oracle/_ref build.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "oracle.cpp"
OUT = HERE / "_build" / "liboracle.so"
FLAGS = ["-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-ffp-contract=off",
         "-fno-fast-math", "-Wall", "-Wextra"]


def build(force: bool = False) -> Path:
    """Compile the oracle unless the library is newer than its sources."""
    header = HERE.parent / "include" / "sherd_cuda.h"
    if not force and OUT.exists():
        newest = max(SOURCE.stat().st_mtime, header.stat().st_mtime)
        if OUT.stat().st_mtime >= newest:
            return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = ["g++", *FLAGS, str(SOURCE), "-o", str(tmp)]
    subprocess.run(cmd, check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
