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


STRUCTS = [("engine", "Options", "vgc_options"), ("engine", "MeshData", "vgc_mesh_data"),
           ("engine", "MeshOpts", "vgc_mesh_opts"), ("engine", "View", "vgc_view"),
           ("engine", "TuneResult", "vgc_tune_result"), ("engine", "ServerOptions", "vgc_server_options"),
           ("engine", "ServerStats", "vgc_server_stats"), ("engine", "Output", "vgc_output"),
           ("engine", "Stats", "vgc_stats"), ("engine", "ServeResult", "vgc_serve_result"),
           ("build", "_Mesh", "vgb_mesh"), ("build", "_Options", "vgb_options"), ("build", "_Raw", "vgb_raw")]


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors in vgcut/engine.py and vgcut/build.py have the C structs' sizes and field offsets (a C
    program compiled against include/vgcut.h and include/vgbuild.h prints them)."""
    import importlib
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vgcut.h"', '#include "vgbuild.h"',
             "int main(void) {"]
    want = {}
    for mod, py, c in STRUCTS:
        cls = getattr(importlib.import_module("vgcut." + mod), py)
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        want[(py, "size")] = ctypes.sizeof(cls)
        for name, _ in cls._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
            want[(py, name)] = getattr(cls, name).offset
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        py, name, value = line.split()
        got[(py, name)] = int(value)
    assert got == want
