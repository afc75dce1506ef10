"""ctypes binding of libcudaring.so, generated from include/cudaring.h.

The header is the single source of truth: every ``int cr_*(...)`` prototype in
it is bound here with argument types derived from its C types, and
``declared_symbols()`` lists them so the tests can check that the library
exports each one.  Loading fails loudly when the library is missing: there is
no CPU fallback for the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HEADER = os.path.join(ROOT, "include", "cudaring.h")
LIBPATH = os.environ.get("CUDARING_LIBPATH") or os.path.join(HERE, "lib", "libcudaring.so")

_TYPES = {
    "int": C.c_int,
    "long": C.c_long,
    "double": C.c_double,
    "long long": C.c_longlong,
    "unsigned long long": C.c_ulonglong,
}


def _ctype(decl: str):
    decl = decl.strip()
    decl = re.sub(r"\bconst\b", "", decl).strip()
    if decl.count("*") == 2:
        return C.POINTER(C.c_void_p)
    if "*" in decl:
        return C.c_void_p
    base = re.sub(r"\s+[A-Za-z_]\w*$", "", decl).strip()
    return _TYPES[base]


def parse_header(path: str = HEADER) -> dict[str, tuple[str, list]]:
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(int|const char\*)\s+(cr_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3).strip()
        argtypes = [] if args in ("", "void") else [_ctype(a) for a in args.split(",")]
        out[name] = (ret, argtypes)
    return out


def declared_symbols() -> list[str]:
    return sorted(parse_header())


class CudaRingError(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


_LIB = None


def lib() -> C.CDLL:
    """Load libcudaring.so and bind every prototype of include/cudaring.h."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIBPATH):
        raise FileNotFoundError(
            f"{LIBPATH} is missing: build it with `python -m cudaring_b200.build` (there is no CPU fallback)")
    L = C.CDLL(LIBPATH)
    for name, (ret, argtypes) in parse_header().items():
        fn = getattr(L, name)
        fn.argtypes = argtypes
        fn.restype = C.c_char_p if ret.startswith("const char") else C.c_int
    _LIB = L
    return L
