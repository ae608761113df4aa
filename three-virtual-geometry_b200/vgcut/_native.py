"""Loading of the in-tree native libraries.

``libvgcut.so`` is the sm_100a cull + LOD-cut engine; ``libvgbuild.so`` is the host DAG builder and scene
generators. Both are built in-tree by ``make`` (see the package Makefile). A missing library raises at once:
there is no CPU fallback for the cut.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
_libs: dict[str, ctypes.CDLL] = {}


def lib_path(name: str) -> str:
    return os.path.join(_HERE, name)


def build(targets: tuple[str, ...] = ("all",)) -> None:
    """Compiles the native libraries in-tree (nvcc for sm_100a, g++ for the host builder)."""
    subprocess.run(["make", "-C", PKG_ROOT, *targets], check=True)


def load(name: str) -> ctypes.CDLL:
    """Loads ``name`` from the package directory; raises ``OSError`` when it was never built."""
    lib = _libs.get(name)
    if lib is not None:
        return lib
    path = lib_path(name)
    if not os.path.exists(path):
        raise OSError(f"{name} is not built: run `make -C {PKG_ROOT}` (no fallback exists for this library)")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
    _libs[name] = lib
    return lib
