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
    inc = os.path.join(ROOT, "include")
    text = "".join(open(os.path.join(inc, h)).read() for h in sorted(os.listdir(inc)) if h.endswith(".h"))
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for m in re.finditer(r"DQ_API\s+([\w\s\*]+?)\b(dq_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [q.strip() for q in params.split(",")]
        out[name] = (ret, len(plist), plist)
    return out


def _kind_of_param(p):
    if "*" in p:
        return "pointer"
    if re.match(r"(const\s+)?double\b", p):
        return "double"
    return "int"   # int and the enum/int-typed parameters


def _kind_of_ctype(t):
    if t in (C.c_void_p, C.c_char_p) or t.__name__.startswith("LP_"):
        return "pointer"
    if t is C.c_double:
        return "double"
    if t is C.c_int:
        return "int"
    return t.__name__


def test_header_and_ctypes_list_the_same_entry_points():
    decl = _declarations()
    assert len(decl) >= 50
    assert sorted(decl) == sorted(_lib.EXPORTS)


def test_ctypes_parameter_counts_and_return_kinds_match_the_header():
    L = _lib.load()
    for name, (ret, n, plist) in _declarations().items():
        f = getattr(L, name)
        assert f.argtypes is not None, f"{name}: no argtypes"
        assert len(f.argtypes) == n, f"{name}: header has {n} parameters, ctypes {len(f.argtypes)}"
        for i, (p, t) in enumerate(zip(plist, f.argtypes)):
            assert _kind_of_param(p) == _kind_of_ctype(t), f"{name} parameter {i} ({p}): ctypes {t.__name__}"
        if ret == "void":
            assert f.restype is None, name
        elif ret in ("dq_status", "int"):
            assert f.restype is C.c_int, name
        elif ret.endswith("*"):
            assert f.restype in (C.c_void_p, C.c_char_p), name
