"""Locates and loads the in-tree shared libraries of this package."""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
_cache: dict[str, ctypes.CDLL] = {}


def lib_path(name: str) -> str:
    return os.path.join(PKG_DIR, name)


def load_library(name: str) -> ctypes.CDLL:
    """Loads ``name`` from the package directory.  Raises if it was not built:
    there is no fallback implementation."""
    if name in _cache:
        return _cache[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python -m aretomo3_b200.build`")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
    _cache[name] = lib
    return lib
