"""Locating and loading the in-tree shared libraries of the package."""
import ctypes
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)

_cache = {}


def lib_path(name: str) -> str:
    return os.path.join(PKG_DIR, name)


def load(name: str) -> ctypes.CDLL:
    """Loads lamb_b200/<name>; raises with a build hint when it is missing."""
    if name in _cache:
        return _cache[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run `python -m lamb_b200.build` (or __graft_entry__.build())")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
    _cache[name] = lib
    return lib
