"""io::load_mesh for PLY (io/mod.rs:114-137, io/ply.rs, mesh/clean.rs): sherd_mesh_read.

Checked on files written here in every PLY encoding (ASCII, binary little- and big-endian), with
float and double coordinates, extra properties and elements, polygons (fan-triangulated from the
first corner; faces under three corners dropped, io/ply.rs:1-16), and the three cleaning steps of
mesh/clean.rs:138-142 (duplicates merge onto their first occurrence with +0 = -0 and NaN never
equal, faces with a repeated corner dropped, unreferenced vertices removed). On the reference's
own slab input, when it is present, the result is the fixture's load.V0 / load.F0 exactly.
"""

from __future__ import annotations

import os
import struct
from pathlib import Path

import numpy as np
import pytest

# The reference's slab input directory (its fixtures/slab/input), named by SHERD_REFERENCE_ROOT:
# the test that reads it is skipped where the variable is unset or the files are absent.
_REF_ROOT = os.environ.get("SHERD_REFERENCE_ROOT")
REFERENCE_INPUT = Path(_REF_ROOT) / "fixtures" / "slab" / "input" if _REF_ROOT else None


def _write_ply(path, v, faces, fmt="binary_little_endian", vtype="double", extra=True):
    fmtc = {"binary_little_endian": "<", "binary_big_endian": ">"}.get(fmt)
    head = ["ply", f"format {fmt} 1.0", "comment written by the test",
            f"element vertex {len(v)}"]
    head += [f"property {vtype} {c}" for c in "xyz"]
    if extra:
        head += ["property float nx", "property uchar red"]
    head += [f"element face {len(faces)}", "property list uchar int vertex_indices"]
    if extra:
        head += ["element camera 1", "property float k"]
    head += ["end_header"]
    vf = {"double": "d", "float": "f"}[vtype]
    with open(path, "wb") as out:
        out.write(("\n".join(head) + "\n").encode())
        if fmtc is None:
            for p in v:
                out.write((" ".join(repr(float(x)) for x in p) + (" 0.5 7" if extra else "") + "\n").encode())
            for fc in faces:
                out.write((" ".join(str(x) for x in [len(fc), *fc]) + "\n").encode())
            if extra:
                out.write(b"1.5\n")
        else:
            for p in v:
                out.write(struct.pack(fmtc + vf * 3, *p))
                if extra:
                    out.write(struct.pack(fmtc + "fB", 0.5, 7))
            for fc in faces:
                out.write(struct.pack(fmtc + "B" + "i" * len(fc), len(fc), *fc))
            if extra:
                out.write(struct.pack(fmtc + "f", 1.5))


# A square split as a quad, a pentagon, a two-corner face, a face naming vertex 0 twice, a
# duplicate of vertex 1 (and -0.0 against +0.0 for vertex 0), a NaN vertex used twice and never
# merged, and an unreferenced vertex.
V = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0],
     [-0.0, 0.0, 0.0], [2.0, 0.5, 0.0], [9.0, 9.0, 9.0], [np.nan, 0.0, 0.0], [np.nan, 0.0, 0.0],
     [3.0, 3.0, 3.0]]
FACES = [[0, 1, 2, 3], [4, 6, 2, 3, 5], [0, 1], [0, 5, 2], [8, 9, 10]]


def _expected():
    """The same file read and cleaned by hand."""
    fan = []
    for fc in FACES:
        for k in range(2, len(fc)):
            fan.append([fc[0], fc[k - 1], fc[k]])
    # duplicates: 4 -> 1, 5 -> 0 (the -0.0 equals +0.0); NaN rows 8, 9 stay distinct.
    remap = {0: 0, 1: 1, 2: 2, 3: 3, 4: 1, 5: 0, 6: 4, 7: 5, 8: 6, 9: 7, 10: 8}
    verts = [V[i] for i in (0, 1, 2, 3, 6, 7, 8, 9, 10)]
    tri = [[remap[i] for i in t] for t in fan]
    tri = [t for t in tri if len(set(t)) == 3]
    used = sorted({i for t in tri for i in t})
    ren = {o: k for k, o in enumerate(used)}
    return np.array([verts[i] for i in used]), np.array([[ren[i] for i in t] for t in tri])


@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
@pytest.mark.parametrize("vtype", ["double", "float"])
def test_read_and_clean(sherd, tmp_path, fmt, vtype):
    path = tmp_path / "m.ply"
    _write_ply(path, V, FACES, fmt, vtype)
    v, f = sherd.read_mesh(path)
    want_v, want_f = _expected()
    assert np.array_equal(f, want_f)
    assert np.array_equal(v, want_v.astype(np.float32 if vtype == "float" else np.float64),
                          equal_nan=True)


def test_refusals(sherd, tmp_path):
    with pytest.raises(sherd.SherdError):
        sherd.read_mesh(tmp_path / "missing.ply")
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"not a ply\n")
    with pytest.raises(sherd.SherdError):
        sherd.read_mesh(bad)
    flat = tmp_path / "flat.ply"
    _write_ply(flat, [[0.0, 0, 0], [1.0, 0, 0]], [[0, 1]])
    with pytest.raises(sherd.SherdError):
        sherd.read_mesh(flat)
    short = tmp_path / "short.ply"
    _write_ply(short, V, FACES)
    short.write_bytes(short.read_bytes()[:-40])
    with pytest.raises(sherd.SherdError):
        sherd.read_mesh(short)
    out = tmp_path / "out_of_range.ply"
    _write_ply(out, V[:3], [[0, 1, 7]])
    with pytest.raises(sherd.SherdError):
        sherd.read_mesh(out)


@pytest.mark.skipif(REFERENCE_INPUT is None or not REFERENCE_INPUT.is_dir(),
                    reason="SHERD_REFERENCE_ROOT names no reference checkout with its slab input")
@pytest.mark.parametrize("name", ["pieceA", "pieceB"])
def test_the_reference_slab_input_reads_as_its_load_row(sherd, slab, name):
    v, f = sherd.read_mesh(REFERENCE_INPUT / f"{name}.ply")
    assert np.array_equal(v, slab[f"{name}.V0"]) and np.array_equal(f, slab[f"{name}.F"])
