"""The C-ABI libraries load and export every entry point their headers declare (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header: str, prefix: str) -> list[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"\w+)\s*\(", text)))


@pytest.mark.parametrize("header,lib,prefix", [("vgcut.h", "libvgcut.so", "vgc_"), ("vgbuild.h", "libvgbuild.so", "vgb_")])
def test_exports(header, lib, prefix):
    from vgcut import _native
    L = _native.load(lib)
    names = declared(header, prefix)
    assert len(names) > 5
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_engine_reports_no_device_loudly():
    """Without a CUDA device the engine refuses to create a context: there is no CPU fallback."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from vgcut import engine
    with pytest.raises(engine.VgcError) as e:
        engine.VirtualGeometry()
    assert "no CUDA device" in str(e.value)


def test_version_string():
    from vgcut import engine
    assert b"sm_100a" in engine.lib().vgc_version()
