"""The ctypes mirrors in ``uniphot_b200/_lib.py`` must lay out every public
struct of ``include/uniphot_b200.h`` exactly as a C compiler does: a field
at a wrong offset would hand the library a wrong pointer.  gcc compiles a
probe that prints ``offsetof`` of every field the ctypes class names and the
struct's size; the two must agree.  CPU only."""

import shutil
import subprocess
from pathlib import Path

import ctypes as C
import pytest

from uniphot_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
PAIRS = [(_lib.ClassDesc, "uph_class_desc"), (_lib.ChunkIn, "uph_chunk_in"),
         (_lib.ChunkOut, "uph_chunk_out"), (_lib.SparseBand, "uph_sparse_band"),
         (_lib.SparseOut, "uph_sparse_out"), (_lib.NoallocArgs, "uph_noalloc_args")]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_ctypes_structs_match_the_c_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "uniphot_b200.h"',
             "int main(void) {"]
    for cls, cname in PAIRS:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        cname, field, v = ln.split()
        got[(cname, field)] = int(v)
    for cls, cname in PAIRS:
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, f"{cname}.{f[0]}"
