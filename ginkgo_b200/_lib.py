"""Loads libginkgo_b200.so and binds every function declared in
include/ginkgo_b200.h through ctypes.

The prototypes are read from the header itself, so the binding and the C ABI
cannot drift apart.  Calls return the library's status code; ``call`` raises
``GinkgoError`` with ``b2s_last_error()`` for a negative one.  There is no
fallback: without the built library every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libginkgo_b200.so")
HEADERS = [os.path.join(ROOT, "include", "ginkgo_b200.h")]

_CTYPES = {
    "int": C.c_int,
    "int64_t": C.c_int64,
    "double": C.c_double,
    "float": C.c_float,
    "void": None,
}


class GinkgoError(RuntimeError):
    """A libginkgo_b200 entry point returned an error status."""

    def __init__(self, name, code, message):
        super().__init__(f"{name} failed with status {code}: {message}")
        self.code = code


def _ctype(decl: str):
    decl = decl.strip()
    if "*" in decl:
        return C.c_char_p if decl.replace(" ", "").startswith("constchar*") \
            else C.c_void_p
    base = decl.replace("const", "").split()[0]
    return _CTYPES[base]


def parse_header(path):
    """Returns {name: (restype, [argtypes])} for every prototype."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"#.*", "", text)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(b2s_\w+)\s*\(([^;{]*?)\)\s*;",
                         text, flags=re.S):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        argtypes = []
        if args.strip() not in ("", "void"):
            for a in args.split(","):
                a = " ".join(a.split())
                # drop the parameter name
                a = re.sub(r"\b\w+$", "", a) if not a.endswith("*") else a
                argtypes.append(_ctype(a))
        protos[name] = (_ctype(ret) if ret.strip() != "void" else None, argtypes)
    return protos


def declared_symbols():
    out = {}
    for h in HEADERS:
        out.update(parse_header(h))
    return out


_lib = None


def lib():
    """The loaded library (built lazily when the .so is missing and nvcc is
    available); raises if it cannot be loaded."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        lib_ = C.CDLL(LIB_PATH)
        for name, (res, args) in declared_symbols().items():
            f = getattr(lib_, name)
            f.restype = res
            f.argtypes = args
        _lib = lib_
    return _lib


def call(name, *args):
    """Calls an int-returning entry point and raises on a negative status."""
    rc = getattr(lib(), name)(*args)
    if rc < 0:
        msg = lib().b2s_last_error().decode(errors="replace")
        raise GinkgoError(name, rc, msg)
    return rc
