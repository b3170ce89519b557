"""cffi (ABI mode) binding of libbempp_b200.so, declared from include/bempp_b200.h.

The reference binds its cdylib the same way (module ``bempp._bempprs``, cffi, see
pyproject.toml of bempp-rs); here the header is parsed at import time and the in-tree
library is opened directly.  There is no fallback: if the library is missing the import
fails with the build command to run.
"""

from __future__ import annotations

import os
import re

from cffi import FFI

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_ROOT = os.path.dirname(_PKG)
HEADER = os.path.join(_ROOT, "include", "bempp_b200.h")
LIBRARY = os.path.join(_PKG, "lib", "libbempp_b200.so")


def _cdef_source(path: str) -> str:
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    lines = [ln for ln in text.splitlines() if not ln.lstrip().startswith("#")]
    text = "\n".join(lines)
    text = text.replace('extern "C" {', "")
    # drop the closing brace of the extern "C" block (a lone "}" line)
    text = re.sub(r"^\}\s*$", "", text, flags=re.M)
    return text


ffi = FFI()
ffi.cdef(_cdef_source(HEADER))

if not os.path.exists(LIBRARY):
    raise ImportError(
        f"{LIBRARY} is missing: build it with `python bempp-rs_b200/build.py` "
        "(the assembler has no CPU fallback)")
lib = ffi.dlopen(LIBRARY)


def last_error() -> str:
    return ffi.string(lib.bempp_last_error()).decode()


def check(status: int, what: str = "bempp") -> None:
    if status != lib.BemppStatus_Ok:
        raise RuntimeError(f"{what} failed (status {status}): {last_error()}")
