"""The ctypes layer declares every C entry point with the parameter count and
return kind that include/dq.h gives it (a mismatch would pass garbage through
the boundary without any error). Loads the library; calls nothing."""
import ctypes as C
import os
import re
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dynaquant_b200 import _lib  # noqa: E402


def _declarations():
    text = open(os.path.join(ROOT, "include", "dq.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for m in re.finditer(r"DQ_API\s+([\w\s\*]+?)\b(dq_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        out[name] = (ret, n)
    return out


def test_header_and_ctypes_list_the_same_entry_points():
    decl = _declarations()
    assert len(decl) >= 50
    assert sorted(decl) == sorted(_lib.EXPORTS)


def test_ctypes_parameter_counts_and_return_kinds_match_the_header():
    L = _lib.load()
    for name, (ret, n) in _declarations().items():
        f = getattr(L, name)
        assert f.argtypes is not None, f"{name}: no argtypes"
        assert len(f.argtypes) == n, f"{name}: header has {n} parameters, ctypes {len(f.argtypes)}"
        if ret == "void":
            assert f.restype is None, name
        elif ret in ("dq_status", "int"):
            assert f.restype is C.c_int, name
        elif ret.endswith("*"):
            assert f.restype in (C.c_void_p, C.c_char_p), name
