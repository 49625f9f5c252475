"""The C++ host behind include/dq_host.h: the reference's input file and its run driver.

``parse_infile(path)`` reads a ``key = value`` file as systemClass::parseInFile does
(systemClass.cu:184-735) and returns the dq_infile fields as a dict; ``run_infile`` runs
the simulation it describes (propagate.cu:29-298) and writes the reference's output files.
The command-line form is ``dynaquant_b200/dq_propagate <infile>``.
"""
from __future__ import annotations

import ctypes as C

from . import _lib


def _as_dict(s):
    out = {}
    for name, _t in _lib.InFile._fields_:
        v = getattr(s, name)
        if isinstance(v, bytes):
            v = v.decode()
        elif name == "printpop":
            v = list(v)
        out[name] = v
    return out


def split_line(line: str):
    """(key, value) of one assignment line as the parser reads it; None for a line without '='
    or a key containing '!'."""
    L = _lib.load()
    k = C.create_string_buffer(4096)
    v = C.create_string_buffer(4096)
    rc = L.dq_infile_split_line(line.encode(), k, len(k), v, len(v))
    return (k.value.decode(), v.value.decode()) if rc == 1 else None


def parse_infile_struct(path) -> _lib.InFile:
    L = _lib.load()
    s = _lib.InFile()
    err = C.create_string_buffer(1024)
    rc = L.dq_infile_parse(str(path).encode(), C.byref(s), err, len(err))
    if rc != 0:
        raise _lib.DQError(rc, err.value.decode(errors="replace"))
    return s


def parse_infile(path) -> dict:
    return _as_dict(parse_infile_struct(path))


def defaults() -> dict:
    L = _lib.load()
    s = _lib.InFile()
    L.dq_infile_defaults(C.byref(s))
    return _as_dict(s)


def run_infile(path_or_struct, base_dir=None, device=0):
    """Runs an input file (a path, or a struct from parse_infile_struct); relative paths in it are
    taken from base_dir (None: the current directory, as the reference opens them)."""
    L = _lib.load()
    s = parse_infile_struct(path_or_struct) if not isinstance(path_or_struct, _lib.InFile) else path_or_struct
    err = C.create_string_buffer(1024)
    rc = L.dq_infile_run(C.byref(s), None if base_dir is None else str(base_dir).encode(), int(device), err,
                         len(err))
    if rc != 0:
        raise _lib.DQError(rc, err.value.decode(errors="replace"))
