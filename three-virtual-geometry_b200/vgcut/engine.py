"""Python mirror of the reference's runtime API over the C ABI of ``include/vgcut.h``.

``VirtualGeometry`` mirrors src/core/runtime/VirtualGeometry.ts (levers :78-183, ``createMesh`` :231,
``update`` :392, ``readStats`` :591) and ``VirtualMesh`` mirrors src/core/runtime/VirtualMesh.ts
(``maxDrawDistance``/``minPixelRadius`` :137-152, ``setMatrixAt``/``commitInstances`` :305-314, ``dispose`` :320).
Every cut runs on the GPU through ``libvgcut.so``; without a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _native
from .budget import GlideController, stats_drawn_and_use
from .camera import Camera

VGC_OK = 0
STATUS = {0: "OK", -1: "INVALID_ARG", -2: "OOM", -3: "OVER_BUDGET", -4: "TIMEOUT", -5: "DEVICE_ERROR", -6: "NOT_FOUND"}
COUNTER_HEADER = 24
NO_DRAW_DISTANCE = 1e30
LOD_FADE_STEPS = 255
FULL_FADE_BITS = LOD_FADE_STEPS << 16


class VgcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("max_triangles", C.c_uint32), ("max_shadow_triangles", C.c_uint32), ("max_meshlets", C.c_uint32),
                ("output_slots", C.c_uint32), ("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64)]


class MeshData(C.Structure):
    _fields_ = [("meshlet_count", C.c_uint32), ("meshlet_bounds", C.POINTER(C.c_float)),
                ("meshlet_info", C.POINTER(C.c_uint32)), ("meshlet_triangle_count", C.c_uint32),
                ("meshlet_triangles", C.POINTER(C.c_uint32)), ("level_count", C.c_uint32),
                ("level_ranges", C.POINTER(C.c_uint32)), ("level_errors", C.POINTER(C.c_float)),
                ("level_guard_errors", C.POINTER(C.c_float)), ("lod_bounds_sphere", C.c_float * 4),
                ("cull_bounds_sphere", C.c_float * 4), ("bounding_sphere", C.c_float * 4),
                ("positions", C.POINTER(C.c_float)), ("vertex_count", C.c_uint32),
                ("meshlet_vertices", C.POINTER(C.c_uint32)), ("meshlet_vertex_count", C.c_uint32)]


class MeshOpts(C.Structure):
    _fields_ = [("max_draw_distance", C.c_float), ("min_pixel_radius", C.c_float), ("enabled", C.c_uint32),
                ("shadow", C.c_uint32), ("occlusion", C.c_uint32), ("occluder", C.c_uint32)]


class View(C.Structure):
    _fields_ = [("view", C.c_double * 16), ("proj", C.c_double * 16), ("near_", C.c_double),
                ("viewport_height", C.c_double), ("error_threshold", C.c_double), ("lod_blend", C.c_double),
                ("min_pixel_radius", C.c_double), ("shadow_error_scale", C.c_double),
                ("max_error_threshold", C.c_double), ("shadow_sweep", C.c_double * 3),
                ("triangle_budget", C.c_double), ("threshold_range", C.c_double * 2),
                ("frustum_culling", C.c_uint32), ("hzb", C.c_int32), ("state_slot", C.c_uint32),
                ("flags", C.c_uint32), ("depth", C.c_void_p), ("depth_width", C.c_uint32),
                ("depth_height", C.c_uint32), ("cascade_clip", C.c_double * 16)]


class TuneResult(C.Structure):
    _fields_ = [("instances_blocks_per_sm", C.c_uint32), ("chunks_blocks_per_sm", C.c_uint32), ("ms", C.c_float),
                ("chunk_meshlets", C.c_uint32)]


class ServerOptions(C.Structure):
    _fields_ = [("streams", C.c_uint32), ("max_batch", C.c_uint32), ("slots_per_scene", C.c_uint32),
                ("hbm_budget_bytes", C.c_uint64), ("linger_us", C.c_uint32), ("max_batch_instances", C.c_uint64),
                ("cross_scene", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("views_launched", C.c_uint64), ("bytes_in_use", C.c_uint64), ("max_bytes_in_use", C.c_uint64),
                ("max_in_flight", C.c_uint32), ("multi_scene_batches", C.c_uint64)]


VIS_EMPTY = 0x3F800000FFFFFFFF  # visibility-buffer pixel where nothing is drawn (VGC_VIS_EMPTY)


class Output(C.Structure):
    _fields_ = [("draw_list", C.c_void_p * 2), ("draw_args", C.c_void_p), ("counters", C.c_void_p),
                ("max_drawn", C.c_uint32), ("mesh_slots", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("visible_cells", C.c_uint32), ("occluded_instances", C.c_uint32), ("selected", C.c_uint32 * 2),
                ("drawn", C.c_uint32 * 2), ("survived", C.c_uint32 * 2), ("work", C.c_uint32 * 2),
                ("requested_indices", C.c_uint32 * 2), ("rounds", C.c_uint32), ("overflow", C.c_uint32),
                ("threshold_scale", C.c_float * 2), ("fill", C.c_float * 2), ("effective_threshold", C.c_float),
                ("instances_tested", C.c_uint32), ("meshlets_tested", C.c_uint32), ("fast_emitted", C.c_uint32),
                ("levels_read", C.c_uint32), ("predicted_triangles", C.c_uint64),
                ("meshlets_queued", C.c_uint32), ("faults", C.c_uint32)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class ServeResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("scene", C.c_uint32), ("slot", C.c_uint32), ("status", C.c_int32),
                ("batch_views", C.c_uint32), ("submit_us", C.c_double), ("start_us", C.c_double),
                ("done_us", C.c_double), ("batch_gpu_ms", C.c_float), ("stats", Stats), ("batch_scenes", C.c_uint32)]


_configured = False


def lib() -> C.CDLL:
    """The engine library with argument types set (raises OSError when it is not built)."""
    global _configured
    L = _native.load("libvgcut.so")
    if _configured:
        return L
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "vgc_last_error": ([], C.c_char_p), "vgc_version": ([], C.c_char_p),
        "vgc_default_options": ([P(Options)], None),
        "vgc_context_create": ([P(Options), P(vp)], C.c_int),
        "vgc_context_destroy": ([vp], C.c_int),
        "vgc_context_footprint": ([vp, P(C.c_uint64)], C.c_int),
        "vgc_mesh_add": ([vp, P(MeshData), P(C.c_float), C.c_uint32, P(MeshOpts), P(C.c_uint32), P(C.c_uint32)], C.c_int),
        "vgc_mesh_set_flags": ([vp, C.c_uint32, P(MeshOpts)], C.c_int),
        "vgc_instances_update": ([vp, C.c_uint32, C.c_uint32, C.c_uint32, P(C.c_float)], C.c_int),
        "vgc_mesh_remove": ([vp, C.c_uint32], C.c_int),
        "vgc_mesh_slots": ([vp, P(C.c_uint32), P(C.c_uint32)], C.c_int),
        "vgc_hzb_build": ([vp, C.c_int32, vp, C.c_uint32, C.c_uint32, C.c_int, vp], C.c_int),
        "vgc_cut": ([vp, P(View), C.c_uint32, C.c_uint32, vp], C.c_int),
        "vgc_cut_noalloc": ([vp, P(View), C.c_uint32, vp], C.c_int),
        "vgc_batch_create": ([vp, C.c_uint32, P(vp)], C.c_int),
        "vgc_batch_run": ([vp, P(View), C.c_uint32, C.c_uint32, vp], C.c_int),
        "vgc_batch_destroy": ([vp], C.c_int),
        "vgc_batch_autotune": ([vp, P(View), C.c_uint32, C.c_uint32, vp, C.c_uint32, P(TuneResult)], C.c_int),
        "vgc_batch_set_tuning": ([vp, P(TuneResult)], C.c_int),
        "vgc_get_output": ([vp, C.c_uint32, P(Output)], C.c_int),
        "vgc_read_stats": ([vp, C.c_uint32, P(Stats), vp], C.c_int),
        "vgc_read_draw_list": ([vp, C.c_uint32, C.c_uint32, P(C.c_uint32), C.c_uint32, P(C.c_uint32), vp], C.c_int),
        "vgc_state_access": ([vp, C.c_uint32, P(C.c_uint32), C.c_int, vp], C.c_int),
        "vgc_expand": ([vp, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp], C.c_int),
        "vgc_select_cut": ([vp, C.c_uint32, C.c_uint32, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double),
                            C.c_double, C.c_double, P(C.c_uint8), P(C.c_uint8)], C.c_int),
        "vgc_hzb_info": ([vp, C.c_int32, P(C.c_uint32), P(C.c_uint32), P(C.c_uint32), P(C.c_uint32), P(vp)], C.c_int),
        "vgc_set_profiling": ([vp, C.c_int], C.c_int),
        "vgc_kernel_times": ([vp, P(C.c_double), P(C.c_uint32), C.c_int], C.c_int),
        "vgc_debug_scene": ([vp, P(C.c_float), C.c_uint32, P(C.c_float), C.c_uint32, P(C.c_uint32), P(C.c_uint32)], C.c_int),
        "vgc_debug_cells_device": ([vp, P(C.c_float), C.c_uint32, P(C.c_uint32)], C.c_int),
        "vgc_debug_wait_probe": ([vp, C.c_uint32, P(C.c_uint32), P(C.c_uint64)], C.c_int),
        "vgc_occluder_depth": ([vp, C.c_uint32, P(View), vp, C.c_uint32, C.c_uint32, vp], C.c_int),
        "vgc_occluder_depth_batch": ([vp, C.c_uint32, P(C.c_uint32), P(View), P(vp), C.c_uint32, C.c_uint32, vp],
                                     C.c_int),
        "vgc_instances_resort": ([vp, C.c_uint32, P(C.c_uint32)], C.c_int),
        "vgc_visibility": ([vp, C.c_uint32, C.c_uint32, P(View), P(View), vp, C.c_uint64, vp, C.c_uint32, C.c_uint32,
                            C.c_uint32, vp], C.c_int),
        "vgc_server_default_options": ([P(ServerOptions)], None),
        "vgc_server_create": ([P(vp), C.c_uint32, P(ServerOptions), P(vp)], C.c_int),
        "vgc_server_submit": ([vp, C.c_uint32, P(View), P(C.c_uint64)], C.c_int),
        "vgc_server_wait": ([vp, C.c_uint64, C.c_uint32, P(ServeResult)], C.c_int),
        "vgc_server_release": ([vp, C.c_uint64], C.c_int),
        "vgc_server_drain": ([vp, C.c_uint32], C.c_int),
        "vgc_server_stats_get": ([vp, P(ServerStats)], C.c_int),
        "vgc_server_destroy": ([vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _configured = True
    return L


def check(rc: int) -> None:
    if rc != VGC_OK:
        raise VgcError(rc, lib().vgc_last_error().decode())


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _up(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def mesh_struct(data, with_vertices: bool = False) -> tuple[MeshData, list]:
    """C view of a VirtualMeshData (keeps the numpy arrays alive in the returned list); `with_vertices` adds the
    positions and meshlet vertex ids the occluder depth pass draws from."""
    keep = [np.ascontiguousarray(data.meshlet_bounds, np.float32), np.ascontiguousarray(data.meshlet_info, np.uint32),
            np.ascontiguousarray(data.meshlet_triangles, np.uint32), np.ascontiguousarray(data.level_ranges, np.uint32),
            np.ascontiguousarray(data.level_errors, np.float32),
            np.ascontiguousarray(data.level_guard_errors, np.float32)]
    m = MeshData()
    m.meshlet_count = data.meshlet_count
    m.meshlet_bounds = _fp(keep[0])
    m.meshlet_info = _up(keep[1])
    m.meshlet_triangle_count = len(keep[2])
    m.meshlet_triangles = _up(keep[2])
    m.level_count = len(keep[3]) // 2
    m.level_ranges = _up(keep[3])
    m.level_errors = _fp(keep[4])
    m.level_guard_errors = _fp(keep[5])
    for k in range(4):
        m.lod_bounds_sphere[k] = float(data.lod_bounds_sphere[k])
        m.cull_bounds_sphere[k] = float(data.cull_bounds_sphere[k])
        m.bounding_sphere[k] = float(data.bounding_sphere[k])
    if with_vertices:
        pos = np.ascontiguousarray(data.positions, np.float32).reshape(-1)
        mv = np.ascontiguousarray(data.meshlet_vertices, np.uint32)
        keep += [pos, mv]
        m.positions, m.vertex_count = _fp(pos), len(pos) // 3
        m.meshlet_vertices, m.meshlet_vertex_count = _up(mv), len(mv)
    return m, keep


@dataclass
class ViewParams:
    """Levers of one cut (VirtualGeometry.ts:78-183 defaults)."""
    error_threshold: float = 1.0
    lod_blend: float = 2.0
    min_pixel_radius: float = 0.7
    shadow_error_scale: float = 3.0
    max_error_threshold: float = 64.0
    shadow_sweep: tuple = (0.0, 0.0, 0.0)
    triangle_budget: float = 0.0
    threshold_range: tuple = (0.5, 3.0)
    frustum_culling: bool = True
    hzb: int = -1
    state_slot: int = 0
    fresh_state: bool = False  # VGC_VIEW_FRESH_STATE: the capacity controller starts from its initial state
    cascade_clip: object = None  # VGC_VIEW_CASCADE: 16 floats, the cascade's world -> clip matrix (column-major)
    depth_as_mip0: bool = False  # VGC_VIEW_DEPTH_AS_MIP0: an HZB built from `depth` reads its mip 0 from it (no copy)


VGC_VIEW_FRESH_STATE = 1
VGC_VIEW_CASCADE = 2
VGC_VIEW_DEPTH_AS_MIP0 = 4


def make_view(camera: Camera, p: ViewParams | None = None, depth=None) -> View:
    """View struct for a camera. `depth`: optional (device pointer, width, height) of this frame's occluder depth,
    from which the cut builds HZB slot `p.hzb` first."""
    p = p or ViewParams()
    v = View()
    for k in range(16):
        v.view[k] = float(camera.view[k])
        v.proj[k] = float(camera.proj[k])
    v.near_ = float(camera.near)
    v.viewport_height = float(camera.height)
    v.error_threshold = p.error_threshold
    v.lod_blend = p.lod_blend
    v.min_pixel_radius = p.min_pixel_radius
    v.shadow_error_scale = p.shadow_error_scale
    v.max_error_threshold = p.max_error_threshold
    for k in range(3):
        v.shadow_sweep[k] = float(p.shadow_sweep[k])
    v.triangle_budget = p.triangle_budget
    v.threshold_range[0], v.threshold_range[1] = p.threshold_range
    v.frustum_culling = 1 if p.frustum_culling else 0
    v.hzb = p.hzb
    v.state_slot = p.state_slot
    v.flags = (VGC_VIEW_FRESH_STATE if p.fresh_state else 0) | (VGC_VIEW_CASCADE if p.cascade_clip is not None else 0) | \
        (VGC_VIEW_DEPTH_AS_MIP0 if p.depth_as_mip0 else 0)
    if p.cascade_clip is not None:
        for k in range(16):
            v.cascade_clip[k] = float(p.cascade_clip[k])
    if depth is not None:
        v.depth, v.depth_width, v.depth_height = depth
    return v


class VirtualMesh:
    """An instanced virtual mesh resident on the GPU (VirtualMesh.ts:91-331)."""

    def __init__(self, vg: "VirtualGeometry", data, matrices: np.ndarray, max_draw_distance: float = math.inf,
                 min_pixel_radius: float = 0.0, cast_shadow: bool = False, occlusion_culling: bool = False,
                 occluder: bool = False, vertex_data: bool = False):
        """`vertex_data`: upload the mesh's positions and meshlet vertices (always done for an occluder), which the
        visibility pass (VirtualGeometry.visibility) pulls its vertices from."""
        self.vg = vg
        self.data = data
        m = np.ascontiguousarray(matrices, np.float32).reshape(-1, 16)
        self.instance_count = len(m)
        self.full_detail_triangles = int(data.stats.get("leafTriangles", 0)) * self.instance_count
        self._flags = dict(max_draw_distance=max_draw_distance, min_pixel_radius=min_pixel_radius, visible=True,
                           cast_shadow=cast_shadow, occlusion_culling=occlusion_culling, occluder=occluder)
        md, keep = mesh_struct(data, with_vertices=occluder or vertex_data)
        self.gpu_to_input = np.zeros(self.instance_count, np.uint32)
        slot = C.c_uint32()
        check(lib().vgc_mesh_add(vg.handle, C.byref(md), _fp(m), self.instance_count, C.byref(self._opts()),
                                 C.byref(slot), _up(self.gpu_to_input)))
        self.slot = slot.value
        self.gpu_index_of = np.empty_like(self.gpu_to_input)
        self.gpu_index_of[self.gpu_to_input] = np.arange(self.instance_count, dtype=np.uint32)
        self._matrices = m[self.gpu_to_input].copy()  # GPU (Morton) order
        self._dirty: set[int] = set()

    def _opts(self) -> MeshOpts:
        f = self._flags
        o = MeshOpts()
        d = f["max_draw_distance"]
        o.max_draw_distance = float(d) if math.isfinite(d) else 0.0
        o.min_pixel_radius = float(f["min_pixel_radius"])
        o.enabled = 1 if f["visible"] else 0
        o.shadow = 1 if f["cast_shadow"] else 0
        o.occlusion = 1 if f["occlusion_culling"] else 0
        o.occluder = 1 if f["occluder"] else 0
        return o

    def _set(self, **kw):
        self._flags.update(kw)
        check(lib().vgc_mesh_set_flags(self.vg.handle, self.slot, C.byref(self._opts())))

    max_draw_distance = property(lambda s: s._flags["max_draw_distance"], lambda s, v: s._set(max_draw_distance=max(0.0, v)))
    min_pixel_radius = property(lambda s: s._flags["min_pixel_radius"], lambda s, v: s._set(min_pixel_radius=max(0.0, v)))
    visible = property(lambda s: s._flags["visible"], lambda s, v: s._set(visible=bool(v)))
    cast_shadow = property(lambda s: s._flags["cast_shadow"], lambda s, v: s._set(cast_shadow=bool(v)))
    occlusion_culling = property(lambda s: s._flags["occlusion_culling"], lambda s, v: s._set(occlusion_culling=bool(v)))

    def set_matrix_at(self, index: int, matrix: np.ndarray) -> None:
        """Updates one instance (caller index). Call ``commit_instances`` afterwards (VirtualMesh.ts:305-309)."""
        g = int(self.gpu_index_of[index])
        self._matrices[g] = np.asarray(matrix, np.float32).reshape(16)
        self._dirty.add(g)

    def set_matrices(self, matrices: np.ndarray) -> None:
        """Updates every instance (caller order, (n, 16)); ``commit_instances`` uploads them in one call."""
        m = np.ascontiguousarray(matrices, np.float32).reshape(self.instance_count, 16)
        self._matrices[:] = m[self.gpu_to_input]
        if self.instance_count:
            self._dirty.update((0, self.instance_count - 1))

    def commit_instances(self) -> None:
        if not self._dirty:
            return
        lo, hi = min(self._dirty), max(self._dirty)
        block = np.ascontiguousarray(self._matrices[lo:hi + 1])
        check(lib().vgc_instances_update(self.vg.handle, self.slot, lo, hi - lo + 1, _fp(block)))
        self._dirty.clear()

    def resort(self) -> np.ndarray:
        """Morton re-sort of the instances at their current positions (vgc_instances_resort), after pending
        set_matrix_at calls are committed; returns new_to_old (previous GPU index of each new GPU index)."""
        self.commit_instances()
        new_to_old = np.zeros(self.instance_count, np.uint32)
        check(lib().vgc_instances_resort(self.vg.handle, self.slot, _up(new_to_old)))
        self.gpu_to_input = self.gpu_to_input[new_to_old]
        self.gpu_index_of[self.gpu_to_input] = np.arange(self.instance_count, dtype=np.uint32)
        self._matrices = self._matrices[new_to_old]
        return new_to_old

    def dispose(self) -> None:
        check(lib().vgc_mesh_remove(self.vg.handle, self.slot))
        self.vg.meshes.remove(self)


class VirtualGeometry:
    """GPU culling + LOD-cut context (VirtualGeometry.ts:77-633), one resident scene."""

    def __init__(self, max_triangles: int = 10_000_000, max_shadow_triangles: int = 4_000_000,
                 max_meshlets: int = 1 << 20, output_slots: int = 1, device: int = 0, hbm_budget_bytes: int = 0,
                 budget_mode: str = "search"):
        """budget_mode: how `triangle_budget` steers the threshold in `update` — "search" (the device histogram
        search of each frame's own cut) or "glide" (the reference's CPU controller over stats readbacks)."""
        o = Options()
        lib().vgc_default_options(C.byref(o))
        o.max_triangles, o.max_shadow_triangles = max_triangles, max_shadow_triangles
        o.max_meshlets = min(max_meshlets, 1 << 24)
        o.output_slots, o.device, o.hbm_budget_bytes = output_slots, device, hbm_budget_bytes
        h = C.c_void_p()
        check(lib().vgc_context_create(C.byref(o), C.byref(h)))
        self.handle = h
        self.options = o
        self.meshes: list[VirtualMesh] = []
        self.params = ViewParams()
        self.last_stats: dict | None = None
        self._batches: dict[int, C.c_void_p] = {}
        if budget_mode not in ("search", "glide"):
            raise ValueError("budget_mode is 'search' or 'glide'")
        self.budget_mode = budget_mode
        self.glide: GlideController | None = None

    # ------------------------------------------------------------------ levers (VirtualGeometry.ts:78-183)
    def __getattr__(self, name):
        p = self.__dict__.get("params")
        if p is not None and hasattr(p, name):
            return getattr(p, name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        p = self.__dict__.get("params")
        if p is not None and name in ViewParams.__dataclass_fields__:
            setattr(p, name, value)
        else:
            super().__setattr__(name, value)

    # ------------------------------------------------------------------ scene
    def create_mesh(self, data, matrices: np.ndarray, **options) -> VirtualMesh:
        m = VirtualMesh(self, data, matrices, **options)
        self.meshes.append(m)
        return m

    def build_hzb(self, slot: int, depth: np.ndarray) -> None:
        d = np.ascontiguousarray(depth, np.float32)
        h, w = d.shape
        check(lib().vgc_hzb_build(self.handle, slot, d.ctypes.data, w, h, 0, None))

    def hzb_info(self, slot: int) -> dict:
        levels = C.c_uint32()
        off, w, h = (C.c_uint32 * 16)(), (C.c_uint32 * 16)(), (C.c_uint32 * 16)()
        data = C.c_void_p()
        check(lib().vgc_hzb_info(self.handle, slot, C.byref(levels), off, w, h, C.byref(data)))
        return dict(levels=levels.value, offset=list(off), width=list(w), height=list(h), data=data.value)

    # ------------------------------------------------------------------ the cut
    def update(self, camera: Camera, slot: int = 0, stream=None, **overrides) -> None:
        """Runs the cut for `camera` into output slot `slot` (VirtualGeometry.update, :392). With a triangle budget
        and budget_mode "glide", the reference's controller steps the threshold first and reads the stats back every
        few frames (budget.GlideController)."""
        p = ViewParams(**{**self.params.__dict__, **overrides})
        glide = self.budget_mode == "glide" and p.triangle_budget > 0
        if glide:
            g = self.glide
            if g is None:
                g = self.glide = GlideController(p.error_threshold, p.triangle_budget, p.threshold_range)
            elif g.written != p.error_threshold:
                g.error_threshold = p.error_threshold  # the user's value (step() then drops the glide)
            g.triangle_budget, g.threshold_range = p.triangle_budget, tuple(p.threshold_range)
            p.error_threshold = self.params.error_threshold = g.step()
            p.triangle_budget = 0.0
        v = make_view(camera, p)
        check(lib().vgc_cut(self.handle, C.byref(v), 1, slot, stream))
        if glide and self.glide.end_frame():
            drawn, use = stats_drawn_and_use(self.read_stats(slot), self.options.max_triangles,
                                             self.options.max_shadow_triangles, self.options.max_meshlets)
            self.glide.adapt(drawn, use)

    def cut(self, views: list[View], first_slot: int = 0, stream=None, graph: bool = False) -> None:
        arr = (View * len(views))(*views)
        if not graph:
            check(lib().vgc_cut(self.handle, arr, len(views), first_slot, stream))
            return
        b = self._batches.get(len(views))
        if b is None:
            b = C.c_void_p()
            check(lib().vgc_batch_create(self.handle, len(views), C.byref(b)))
            self._batches[len(views)] = b
        check(lib().vgc_batch_run(b, arr, len(views), first_slot, stream))

    def autotune(self, views: list[View], first_slot: int = 0, stream=None, reps: int = 3) -> dict:
        """Picks the persistent grid sizes of the batched launch for `len(views)` views (vgc_batch_autotune); later
        `cut(..., graph=True)` calls with that many views use them."""
        arr = (View * len(views))(*views)
        b = self._batches.get(len(views))
        if b is None:
            b = C.c_void_p()
            check(lib().vgc_batch_create(self.handle, len(views), C.byref(b)))
            self._batches[len(views)] = b
        r = TuneResult()
        check(lib().vgc_batch_autotune(b, arr, len(views), first_slot, stream, reps, C.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def set_tuning(self, count: int, instances_blocks_per_sm: int = 0, chunks_blocks_per_sm: int = 0,
                   chunk_meshlets: int = 512) -> None:
        """Applies a tuning to the batched launch of `count` views (vgc_batch_set_tuning): blocks per SM of the
        instance and meshlet kernels (0: occupancy default) and meshlets per chunk (256, 512 or 1024)."""
        b = self._batches.get(count)
        if b is None:
            b = C.c_void_p()
            check(lib().vgc_batch_create(self.handle, count, C.byref(b)))
            self._batches[count] = b
        t = TuneResult(instances_blocks_per_sm, chunks_blocks_per_sm, 0.0, chunk_meshlets)
        check(lib().vgc_batch_set_tuning(b, C.byref(t)))

    def cut_noalloc(self, view: View, slot: int = 0, stream=None) -> None:
        """The single-view cut that allocates nothing on the call (see vgc_cut_noalloc in include/vgcut.h)."""
        check(lib().vgc_cut_noalloc(self.handle, C.byref(view), slot, stream))

    def read_stats(self, slot: int = 0) -> dict:
        s = Stats()
        check(lib().vgc_read_stats(self.handle, slot, C.byref(s), None))
        self.last_stats = s.as_dict()
        return self.last_stats

    def draw_list(self, slot: int = 0, cut: int = 0) -> np.ndarray:
        """The drawn (instance, meshlet, firstIndex, packed) entries of a cut, copied to host memory."""
        n = C.c_uint32()
        check(lib().vgc_read_draw_list(self.handle, slot, cut, None, 0, C.byref(n), None))
        out = np.zeros((n.value, 4), np.uint32)
        if n.value:
            check(lib().vgc_read_draw_list(self.handle, slot, cut, _up(out), n.value, C.byref(n), None))
        return out

    def output(self, slot: int = 0) -> Output:
        o = Output()
        check(lib().vgc_get_output(self.handle, slot, C.byref(o)))
        return o

    def state(self, state_slot: int = 0, words: np.ndarray | None = None) -> np.ndarray:
        w = np.zeros(8, np.uint32) if words is None else np.ascontiguousarray(words, np.uint32)
        check(lib().vgc_state_access(self.handle, state_slot, _up(w), 0 if words is None else 1, None))
        return w

    KERNEL_KINDS = ("reset", "cells", "select0", "retry", "finish", "hzb", "chunks0", "budget")

    def set_profiling(self, enable: bool) -> None:
        check(lib().vgc_set_profiling(self.handle, 1 if enable else 0))

    def kernel_times(self, reset: bool = True) -> dict:
        """Per kernel kind: (summed device ms, launches) of the plain path since the last reset."""
        ms = (C.c_double * 8)()
        n = (C.c_uint32 * 8)()
        check(lib().vgc_kernel_times(self.handle, ms, n, 1 if reset else 0))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNEL_KINDS)}

    def footprint(self) -> int:
        b = C.c_uint64()
        check(lib().vgc_context_footprint(self.handle, C.byref(b)))
        return b.value

    def debug_scene(self) -> tuple[np.ndarray, np.ndarray]:
        nc, ni = C.c_uint32(), C.c_uint32()
        check(lib().vgc_debug_scene(self.handle, None, 0, None, 0, C.byref(nc), C.byref(ni)))
        cells = np.zeros((nc.value, 8), np.float32)
        mats = np.zeros((ni.value, 16), np.float32)
        check(lib().vgc_debug_scene(self.handle, _fp(cells), nc.value, _fp(mats), ni.value, None, None))
        return cells, mats

    def occluder_depth(self, src_slot: int, camera: Camera, depth_ptr: int, width: int, height: int, stream=None) -> None:
        """The occluder depth pass (vgc_occluder_depth): slot `src_slot`'s camera cut drawn with `camera` into the
        device buffer at `depth_ptr` (width x height float32), ready to be this frame's view depth."""
        v = make_view(camera, self.params)
        check(lib().vgc_occluder_depth(self.handle, src_slot, C.byref(v), C.c_void_p(depth_ptr), width, height, stream))

    def occluder_depth_batch(self, src_slots, cameras, depth_ptrs, width: int, height: int, stream=None) -> None:
        """vgc_occluder_depth_batch: image i draws slot src_slots[i] with cameras[i] into depth_ptrs[i]."""
        OccluderBatch(self, src_slots, cameras, depth_ptrs).run(width, height, stream)

    def expand(self, slot: int, cut: int, index_ptr: int, capacity: int, stream=None) -> None:
        """Index expansion (vgc_expand) of output slot `slot`'s cut `cut` into the device buffer at `index_ptr`."""
        check(lib().vgc_expand(self.handle, slot, cut, C.c_void_p(index_ptr), capacity, stream))

    def visibility(self, slot: int, cut: int, camera: Camera, index_ptr: int, capacity: int, vis_ptr: int, width: int,
                   height: int, frame: int = 0, fade_camera: Camera | None = None, stream=None) -> None:
        """Visibility buffer of slot `slot`'s cut `cut` from its expanded index buffer (vgc_visibility): per pixel of
        the device buffer at `vis_ptr` (height x width uint64), depth bits << 32 | drawSlot << 7 | triangle."""
        v = make_view(camera, self.params)
        f = make_view(fade_camera, self.params) if fade_camera is not None else None
        check(lib().vgc_visibility(self.handle, slot, cut, C.byref(v), C.byref(f) if f is not None else None,
                                   C.c_void_p(index_ptr), capacity, C.c_void_p(vis_ptr), width, height, frame, stream))

    def debug_cells_device(self) -> np.ndarray:
        """The device's cell records (8 floats each), as the kernels read them."""
        n = C.c_uint32()
        check(lib().vgc_debug_cells_device(self.handle, None, 0, C.byref(n)))
        cells = np.zeros((n.value, 8), np.float32)
        check(lib().vgc_debug_cells_device(self.handle, _fp(cells), n.value, C.byref(n)))
        return cells

    def wait_probe(self, limit_us: int) -> tuple[int, int]:
        """The device's bounded mbarrier wait run out on purpose: (completed, nanoseconds waited)."""
        done, ns = C.c_uint32(), C.c_uint64()
        check(lib().vgc_debug_wait_probe(self.handle, limit_us, C.byref(done), C.byref(ns)))
        return done.value, ns.value

    def select_cut(self, slot: int, viewmodels: np.ndarray, proj_scale, near, scale, threshold: float,
                   blend: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
        """selectCut / selectBlendCut (cut.ts:26-77) on the GPU for many view-model matrices of one mesh."""
        vm = np.ascontiguousarray(viewmodels, np.float64).reshape(-1, 16)
        n = len(vm)
        ps = np.ascontiguousarray(np.broadcast_to(np.asarray(proj_scale, np.float64), (n,)))
        nr = np.ascontiguousarray(np.broadcast_to(np.asarray(near, np.float64), (n,)))
        sc = np.ascontiguousarray(np.broadcast_to(np.asarray(scale, np.float64), (n,)))
        mcount = next(m for m in self.meshes if m.slot == slot).data.meshlet_count
        lo = np.zeros((n, mcount), np.uint8)
        hi = np.zeros((n, mcount), np.uint8)
        D = C.POINTER(C.c_double)
        check(lib().vgc_select_cut(self.handle, slot, n, vm.ctypes.data_as(D), ps.ctypes.data_as(D),
                                   nr.ctypes.data_as(D), sc.ctypes.data_as(D), threshold, blend,
                                   lo.ctypes.data_as(C.POINTER(C.c_uint8)), hi.ctypes.data_as(C.POINTER(C.c_uint8))))
        return lo, hi

    def dispose(self) -> None:
        h = self.__dict__.get("handle")
        if h:
            for b in self._batches.values():
                lib().vgc_batch_destroy(b)
            self._batches.clear()
            lib().vgc_context_destroy(h)
            self.handle = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


class OccluderBatch:
    """The arguments of one vgc_occluder_depth_batch call, packed once for a caller that repeats it every frame."""

    def __init__(self, vg: "VirtualGeometry", src_slots, cameras, depth_ptrs):
        n = len(src_slots)
        self.vg, self.n = vg, n
        self.slots = (C.c_uint32 * n)(*src_slots)
        self.views = (View * n)(*[make_view(c, vg.params) for c in cameras])
        self.ptrs = (C.c_void_p * n)(*depth_ptrs)

    def run(self, width: int, height: int, stream=None) -> None:
        check(lib().vgc_occluder_depth_batch(self.vg.handle, self.n, self.slots, self.views, self.ptrs, width, height,
                                             stream))


class Server:
    """The serving loop over several resident scenes (vgc_server_* in include/vgcut.h): requests (scene index, view)
    are submitted from any thread, admitted by free output slots and HBM budget, batched oldest first (across scenes
    with `cross_scene`) and run on `streams` CUDA streams with continuous batching. Results stay in the scene's
    output slot until released."""

    def __init__(self, scenes: list, streams: int = 2, max_batch: int = 64, slots_per_scene: int = 0,
                 hbm_budget_bytes: int = 0, linger_us: int = 0, max_batch_instances: int | None = None,
                 cross_scene: bool = True):
        self.scenes = list(scenes)
        o = ServerOptions()
        lib().vgc_server_default_options(C.byref(o))
        o.streams, o.max_batch, o.slots_per_scene = streams, max_batch, slots_per_scene
        o.hbm_budget_bytes, o.linger_us = hbm_budget_bytes, linger_us
        o.cross_scene = 1 if cross_scene else 0
        if max_batch_instances is not None:
            o.max_batch_instances = max_batch_instances
        arr = (C.c_void_p * len(self.scenes))(*[vg.handle for vg in self.scenes])
        self.handle = C.c_void_p()
        check(lib().vgc_server_create(arr, len(self.scenes), C.byref(o), C.byref(self.handle)))

    def submit(self, scene: int, view: View) -> int:
        t = C.c_uint64()
        check(lib().vgc_server_submit(self.handle, scene, C.byref(view), C.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60_000) -> dict:
        r = ServeResult()
        self.wait_into(ticket, r, timeout_ms)
        return self.result_dict(r)

    def wait_into(self, ticket: int, out: "ServeResult", timeout_ms: int = 60_000) -> None:
        """wait() into a caller's result struct, without building a dict (for callers that keep up with a fast
        server: read the struct later with result_dict)."""
        check(lib().vgc_server_wait(self.handle, ticket, timeout_ms, C.byref(out)))

    @staticmethod
    def result_dict(r: "ServeResult") -> dict:
        out = {k: getattr(r, k) for k, _ in ServeResult._fields_ if k != "stats"}
        out["stats"] = r.stats.as_dict()
        return out

    def release(self, ticket: int) -> None:
        check(lib().vgc_server_release(self.handle, ticket))

    def drain(self, timeout_ms: int = 60_000) -> None:
        check(lib().vgc_server_drain(self.handle, timeout_ms))

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().vgc_server_stats_get(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            lib().vgc_server_destroy(self.handle)
            self.handle = C.c_void_p()
