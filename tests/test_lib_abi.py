"""The C-ABI library loads and exports every symbol the header declares
(no device calls)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    txt = (ROOT / "include" / "uniphot_b200.h").read_text()
    return sorted(set(re.findall(r"\b(uph_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_entry_points():
    d = _declared()
    for name in ("uph_create", "uph_run_chunk", "uph_job_solve", "uph_upload_field"):
        assert name in d


def test_library_exports_every_declared_symbol():
    from uniphot_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.fail(f"library not built: {_lib.LIB_PATH}")
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) <= set(_declared())


def test_binding_structs_match_header_fields():
    from uniphot_b200 import _lib
    txt = (ROOT / "include" / "uniphot_b200.h").read_text()
    for struct, cls in (("uph_class_desc", _lib.ClassDesc), ("uph_chunk_in", _lib.ChunkIn),
                        ("uph_chunk_out", _lib.ChunkOut)):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), txt, re.S).group(1)
        fields = re.findall(r"\b([a-z_0-9]+);", re.sub(r"/\*.*?\*/", "", body, flags=re.S))
        assert [f[0] for f in cls._fields_] == fields, struct
