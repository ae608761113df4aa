"""Python side of the host DAG builder (``include/vgbuild.h``).

``build_virtual_mesh`` mirrors the reference's ``buildVirtualMesh(src, opts)``
(src/core/preprocess/buildVirtualMesh.ts:185) and returns a :class:`VirtualMeshData` with the same fields as the
reference's interface (buildVirtualMesh.ts:75-138), as numpy arrays. The generators produce the seeded synthetic
meshes the tests and the benchmark use.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native

MESHLET_BOUNDS_STRIDE = 16
MESHLET_INFO_STRIDE = 4
ERROR_INFINITY = 1e30
MAX_MESHLET_TRIANGLES = 128
MAX_MESHLET_VERTICES = 128


class _Mesh(C.Structure):
    _fields_ = [
        ("vertex_count", C.c_uint32), ("positions", C.POINTER(C.c_float)),
        ("index_count", C.c_uint32), ("indices", C.POINTER(C.c_uint32)),
        ("meshlet_count", C.c_uint32), ("meshlet_bounds", C.POINTER(C.c_float)),
        ("meshlet_info", C.POINTER(C.c_uint32)),
        ("meshlet_vertex_count", C.c_uint32), ("meshlet_vertices", C.POINTER(C.c_uint32)),
        ("meshlet_triangle_count", C.c_uint32), ("meshlet_triangles", C.POINTER(C.c_uint32)),
        ("level_count", C.c_uint32), ("level_ranges", C.POINTER(C.c_uint32)),
        ("level_errors", C.POINTER(C.c_float)), ("level_guard_errors", C.POINTER(C.c_float)),
        ("lod_bounds_sphere", C.c_float * 4), ("cull_bounds_sphere", C.c_float * 4),
        ("bounding_sphere", C.c_float * 4),
        ("replacement_group", C.POINTER(C.c_int32)), ("group_count", C.c_uint32),
        ("replacement_start", C.POINTER(C.c_uint32)), ("replacement_index_count", C.c_uint32),
        ("replacement_indices", C.POINTER(C.c_uint32)),
        ("leaf_triangles", C.c_uint32), ("leaf_meshlets", C.c_uint32), ("root_triangles", C.c_uint32),
        ("root_meshlets", C.c_uint32), ("lod_levels", C.c_uint32), ("build_ms", C.c_double),
    ]


class _Options(C.Structure):
    _fields_ = [
        ("group_size", C.c_uint32), ("max_lod_levels", C.c_uint32), ("simplify_ratio", C.c_float),
        ("max_group_keep_ratio", C.c_float), ("min_level_reduction", C.c_float),
        ("min_root_triangles", C.c_uint32), ("threads", C.c_uint32),
    ]


class _Raw(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("positions", C.POINTER(C.c_float)),
                ("index_count", C.c_uint32), ("indices", C.POINTER(C.c_uint32))]


_configured = False


def _lib() -> C.CDLL:
    global _configured
    lib = _native.load("libvgbuild.so")
    if not _configured:
        P = C.POINTER
        lib.vgb_build.argtypes = [P(C.c_float), C.c_uint32, P(C.c_uint32), C.c_uint32, P(_Options), P(P(_Mesh))]
        lib.vgb_mesh_free.argtypes = [P(_Mesh)]
        lib.vgb_default_options.argtypes = [P(_Options)]
        lib.vgb_last_error.restype = C.c_char_p
        lib.vgb_gen_icosphere.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_uint32, P(P(_Raw))]
        lib.vgb_gen_box_lattice.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, P(P(_Raw))]
        lib.vgb_gen_terrain.argtypes = [C.c_float, C.c_uint32, C.c_float, C.c_float, C.c_float, P(P(_Raw))]
        lib.vgb_raw_free.argtypes = [P(_Raw)]
        lib.vgb_gen_depth_image.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float,
                                            C.c_float, C.c_uint32, P(C.c_float)]
        lib.vgb_morton_order.argtypes = [P(C.c_float), C.c_uint32, P(C.c_float), P(C.c_uint32)]
        lib.vgb_vgeo_checksum.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64]
        lib.vgb_vgeo_checksum.restype = C.c_uint32
        lib.vgb_mulberry32_next.argtypes = [P(C.c_uint32)]
        lib.vgb_mulberry32_next.restype = C.c_uint32
        lib.vgb_perlin3.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float]
        lib.vgb_perlin3.restype = C.c_float
        _configured = True
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(_lib().vgb_last_error().decode())


def _arr(ptr, n, dtype) -> np.ndarray:
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


@dataclass
class VirtualMeshData:
    """Same fields as the reference's ``VirtualMeshData`` (buildVirtualMesh.ts:75-138), minus render attributes."""
    positions: np.ndarray
    indices: np.ndarray
    meshlet_count: int
    meshlet_bounds: np.ndarray
    meshlet_info: np.ndarray
    meshlet_vertices: np.ndarray
    meshlet_triangles: np.ndarray
    level_ranges: np.ndarray
    level_errors: np.ndarray
    level_guard_errors: np.ndarray
    lod_bounds_sphere: np.ndarray
    cull_bounds_sphere: np.ndarray
    bounding_sphere: np.ndarray
    replacement_group: np.ndarray
    replacement_start: np.ndarray
    replacement_indices: np.ndarray
    stats: dict = field(default_factory=dict)
    extra: dict = field(default_factory=dict)  # fields this builder does not produce (normals, colors, uvs, ...)

    @property
    def level_count(self) -> int:
        return len(self.level_ranges) // 2


def build_virtual_mesh(positions: np.ndarray, indices: np.ndarray, group_size: int = 12, max_lod_levels: int = 24,
                       threads: int = 0, **extra) -> VirtualMeshData:
    """Builds the cluster DAG of an indexed triangle mesh (positions: float32 (n, 3), indices: uint32 (3 m,))."""
    lib = _lib()
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    opts = _Options()
    lib.vgb_default_options(C.byref(opts))
    opts.group_size = group_size
    opts.max_lod_levels = max_lod_levels
    opts.threads = threads
    for k, v in extra.items():
        setattr(opts, k, v)
    out = C.POINTER(_Mesh)()
    _check(lib.vgb_build(pos.ctypes.data_as(C.POINTER(C.c_float)), len(pos) // 3,
                         idx.ctypes.data_as(C.POINTER(C.c_uint32)), len(idx), C.byref(opts), C.byref(out)))
    m = out.contents
    M, L = m.meshlet_count, m.level_count
    data = VirtualMeshData(
        positions=_arr(m.positions, m.vertex_count * 3, np.float32),
        indices=_arr(m.indices, m.index_count, np.uint32),
        meshlet_count=M,
        meshlet_bounds=_arr(m.meshlet_bounds, M * 16, np.float32),
        meshlet_info=_arr(m.meshlet_info, M * 4, np.uint32),
        meshlet_vertices=_arr(m.meshlet_vertices, m.meshlet_vertex_count, np.uint32),
        meshlet_triangles=_arr(m.meshlet_triangles, m.meshlet_triangle_count, np.uint32),
        level_ranges=_arr(m.level_ranges, L * 2, np.uint32),
        level_errors=_arr(m.level_errors, L * 2, np.float32),
        level_guard_errors=_arr(m.level_guard_errors, L * 2, np.float32),
        lod_bounds_sphere=np.array(list(m.lod_bounds_sphere), np.float32),
        cull_bounds_sphere=np.array(list(m.cull_bounds_sphere), np.float32),
        bounding_sphere=np.array(list(m.bounding_sphere), np.float32),
        replacement_group=_arr(m.replacement_group, M, np.int32),
        replacement_start=_arr(m.replacement_start, m.group_count + 1, np.uint32),
        replacement_indices=_arr(m.replacement_indices, m.replacement_index_count, np.uint32),
        stats=dict(leafTriangles=m.leaf_triangles, leafMeshlets=m.leaf_meshlets, rootTriangles=m.root_triangles,
                   rootMeshlets=m.root_meshlets, lodLevels=m.lod_levels, buildMs=m.build_ms),
    )
    lib.vgb_mesh_free(out)
    return data


def _raw(fn, *args) -> tuple[np.ndarray, np.ndarray]:
    lib = _lib()
    out = C.POINTER(_Raw)()
    _check(fn(*args, C.byref(out)))
    r = out.contents
    pos = _arr(r.positions, r.vertex_count * 3, np.float32).reshape(-1, 3)
    idx = _arr(r.indices, r.index_count, np.uint32)
    lib.vgb_raw_free(out)
    return pos, idx


def gen_icosphere(n: int, radius: float = 1.0, amplitude: float = 0.02, frequency: float = 3.0, seed: int = 1):
    """Geodesic icosphere with 20 n^2 triangles, Perlin-displaced by ``amplitude * radius``."""
    return _raw(_lib().vgb_gen_icosphere, n, radius, amplitude, frequency, seed)


def gen_box_lattice(boxes: int, k: int, extent: float = 1.0, seed: int = 1):
    """Ruins-like set of ``boxes`` closed boxes, each face a k x k grid (12 k^2 triangles per box)."""
    return _raw(_lib().vgb_gen_box_lattice, boxes, k, extent, seed)


def gen_terrain(size: float = 400.0, segments: int = 96, amplitude: float = 30.0, fx: float = 0.05, fz: float = 0.04):
    """Height-field terrain; defaults are the reference cut test's terrain (tests/cut.test.ts:14-19)."""
    return _raw(_lib().vgb_gen_terrain, size, segments, amplitude, fx, fz)


def gen_depth_image(width: int, height: int, quads: int, dmin: float, dmax: float, p10: float, p14: float,
                    seed: int) -> np.ndarray:
    out = np.empty((height, width), np.float32)
    _check(_lib().vgb_gen_depth_image(width, height, quads, dmin, dmax, p10, p14, seed,
                                      out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def morton_order(matrices: np.ndarray, sphere: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(matrices, dtype=np.float32).reshape(-1)
    s = np.ascontiguousarray(sphere, dtype=np.float32)
    out = np.empty(len(m) // 16, np.uint32)
    _check(_lib().vgb_morton_order(m.ctypes.data_as(C.POINTER(C.c_float)), len(m) // 16,
                                   s.ctypes.data_as(C.POINTER(C.c_float)), out.ctypes.data_as(C.POINTER(C.c_uint32))))
    return out


class Mulberry32:
    """Seeded PRNG shared with the C generators (same stream for the same seed)."""

    def __init__(self, seed: int):
        self._state = C.c_uint32(seed & 0xFFFFFFFF)

    def next_u32(self) -> int:
        return _lib().vgb_mulberry32_next(C.byref(self._state))

    def __call__(self) -> float:
        return self.next_u32() / 4294967296.0
