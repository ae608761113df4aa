"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference arm may import this module. It
loads ``oracle/liboracle.so`` (the C restatement of the reference's cut evaluator and per-frame passes, see
vg_oracle.h) and builds it with ``make`` when missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    P = C.POINTER
    D16 = C.c_double * 16
    L.vgo_lod_fade_range.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, P(C.c_int), P(C.c_int)]
    L.vgo_select_cut.argtypes = [P(C.c_float), C.c_uint32, D16, C.c_double, C.c_double, C.c_double, C.c_double, P(C.c_uint8)]
    L.vgo_select_blend_cut.argtypes = [P(C.c_float), C.c_uint32, D16, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, P(C.c_uint8), P(C.c_uint8)]
    L.vgo_verify_overlap.argtypes = [C.c_uint32, P(C.c_int32), P(C.c_uint32), P(C.c_uint32), P(C.c_uint8), P(C.c_uint32)]
    L.vgo_verify_overlap.restype = C.c_uint32
    L.vgo_verify_coverage.argtypes = [C.c_uint32, P(C.c_uint32), P(C.c_int32), P(C.c_uint32), P(C.c_uint32),
                                      P(C.c_uint8), P(C.c_uint32)]
    L.vgo_verify_coverage.restype = C.c_uint32
    L.vgo_instance_meshlet_range.argtypes = [P(C.c_uint32), P(C.c_float), C.c_uint32, P(C.c_float), D16, C.c_double,
                                             C.c_double, C.c_double, C.c_double, C.c_double, P(C.c_uint32), P(C.c_uint32)]
    L.vgo_instance_guaranteed_range.argtypes = [P(C.c_uint32), P(C.c_float), P(C.c_float), C.c_uint32, P(C.c_float),
                                                D16, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                                P(C.c_uint32), P(C.c_uint32)]
    L.vgo_cull_pass_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    U32, F32 = P(C.c_uint32), P(C.c_float)
    L.vgo_blend_keep.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32]
    L.vgo_visibility.argtypes = [U32, C.c_uint64, U32, C.c_uint32, U32, C.c_uint32, F32, C.c_uint32, U32, U32, F32,
                                 U32, C.c_uint32, U32, C.c_uint32, F32, C.c_uint32, P(C.c_double), P(C.c_double),
                                 P(C.c_double), C.c_uint32, C.c_uint32, C.c_uint32, P(C.c_uint64)]
    L.vgo_cull_pass_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.vgo_explain_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32]
    L.vgo_explain_f64.restype = C.c_double
    L.vgo_hzb_build.argtypes = [P(C.c_float), C.c_uint32, C.c_uint32, P(C.c_float), C.c_uint64, P(C.c_uint32),
                                P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
    L.vgo_hzb_build.restype = C.c_int64
    L.vgo_cut_invariant.argtypes = [C.c_void_p, P(C.c_uint32), C.c_uint32, P(C.c_uint32), C.c_uint32, P(C.c_uint32),
                                     C.c_uint64, P(C.c_uint32), C.c_uint32, C.c_int, P(C.c_uint64)]
    L.vgo_cut_invariant.restype = C.c_uint64
    L.vgo_frustum_planes.argtypes = [C.c_double * 16, C.c_double * 24]
    L.vgo_logf.argtypes = [C.c_float]
    L.vgo_logf.restype = C.c_float
    _lib = L
    return L


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _u(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _b(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _v16(view):
    return (C.c_double * 16)(*[float(x) for x in view])


# ------------------------------------------------------------------ Part A: cut.ts (double)
def lod_fade_range(own, parent, threshold, blend):
    lo, hi = C.c_int(), C.c_int()
    ok = lib().vgo_lod_fade_range(own, parent, threshold, blend, C.byref(lo), C.byref(hi))
    return (lo.value, hi.value) if ok else None


def select_cut(data, view16, proj_scale, near, threshold, scale=1.0) -> np.ndarray:
    out = np.zeros(data.meshlet_count, np.uint8)
    b = np.ascontiguousarray(data.meshlet_bounds, np.float32)
    lib().vgo_select_cut(_f(b), data.meshlet_count, _v16(view16), proj_scale, near, scale, threshold, _b(out))
    return out


def select_blend_cut(data, view16, proj_scale, near, threshold, blend, scale=1.0):
    lo = np.zeros(data.meshlet_count, np.uint8)
    hi = np.zeros(data.meshlet_count, np.uint8)
    b = np.ascontiguousarray(data.meshlet_bounds, np.float32)
    lib().vgo_select_blend_cut(_f(b), data.meshlet_count, _v16(view16), proj_scale, near, scale, threshold, blend,
                               _b(lo), _b(hi))
    return lo, hi


def _links(data):
    return (np.ascontiguousarray(data.replacement_group, np.int32), np.ascontiguousarray(data.replacement_start, np.uint32),
            np.ascontiguousarray(data.replacement_indices, np.uint32))


def verify_cut_overlap(data, selected) -> np.ndarray:
    g, s, l = _links(data)
    sel = np.ascontiguousarray(selected, np.uint8)
    out = np.zeros(data.meshlet_count, np.uint32)
    n = lib().vgo_verify_overlap(data.meshlet_count, g.ctypes.data_as(C.POINTER(C.c_int32)), _u(s), _u(l), _b(sel), _u(out))
    return out[:n]


def verify_cut_coverage(data, selected) -> np.ndarray:
    g, s, l = _links(data)
    sel = np.ascontiguousarray(selected, np.uint8)
    info = np.ascontiguousarray(data.meshlet_info, np.uint32)
    out = np.zeros(data.meshlet_count, np.uint32)
    n = lib().vgo_verify_coverage(data.meshlet_count, _u(info), g.ctypes.data_as(C.POINTER(C.c_int32)), _u(s), _u(l),
                                  _b(sel), _u(out))
    return out[:n]


def instance_meshlet_range(data, view16, proj_scale, near, threshold, blend=1.0, scale=1.0):
    r = np.ascontiguousarray(data.level_ranges, np.uint32)
    e = np.ascontiguousarray(data.level_errors, np.float32)
    L = np.ascontiguousarray(data.lod_bounds_sphere, np.float32)
    s, t = C.c_uint32(), C.c_uint32()
    lib().vgo_instance_meshlet_range(_u(r), _f(e), len(r) // 2, _f(L), _v16(view16), proj_scale, near, scale, threshold,
                                     blend, C.byref(s), C.byref(t))
    return s.value, t.value


def instance_guaranteed_range(data, view16, proj_scale, near, threshold, blend=1.0, scale=1.0):
    r = np.ascontiguousarray(data.level_ranges, np.uint32)
    e = np.ascontiguousarray(data.level_errors, np.float32)
    g = np.ascontiguousarray(data.level_guard_errors, np.float32)
    L = np.ascontiguousarray(data.lod_bounds_sphere, np.float32)
    s, t = C.c_uint32(), C.c_uint32()
    ok = lib().vgo_instance_guaranteed_range(_u(r), _f(e), _f(g), len(r) // 2, _f(L), _v16(view16), proj_scale, near,
                                             scale, threshold, blend, C.byref(s), C.byref(t))
    return (s.value, t.value) if ok else None


def frustum_planes(m16) -> np.ndarray:
    """three's Frustum.setFromProjectionMatrix(m, WebGPUCoordinateSystem) as the oracle computes it: (6, 4) planes in
    the order right, left, bottom, top, far, near."""
    out = (C.c_double * 24)()
    lib().vgo_frustum_planes(_v16(m16), out)
    return np.array(list(out)).reshape(6, 4)


class _Dag(C.Structure):
    _fields_ = [("meshlet_count", C.c_uint32), ("info", C.POINTER(C.c_uint32)), ("group", C.POINTER(C.c_int32)),
                ("start", C.POINTER(C.c_uint32)), ("list", C.POINTER(C.c_uint32))]


def cut_invariant(meshes, instance_slots, entries, steps=(0,), threads: int = 0) -> tuple[int, int]:
    """verifyCutCoverage + verifyCutOverlap (cut.ts:83-122) for every drawn instance of one cut at every blend step
    in `steps`: meshes in slot order, instance_slots (I,) mesh slot per GPU-order instance, entries (n, 3)
    (instance, pool-global meshlet, packed). Returns (failing (instance, step) pairs, instances checked)."""
    keep = []
    dags = (_Dag * max(1, len(meshes)))()
    base = np.zeros(max(1, len(meshes)), np.uint32)
    b = 0
    for k, d in enumerate(meshes):
        arrs = [np.ascontiguousarray(d.meshlet_info, np.uint32), np.ascontiguousarray(d.replacement_group, np.int32),
                np.ascontiguousarray(d.replacement_start, np.uint32),
                np.ascontiguousarray(d.replacement_indices, np.uint32)]
        keep += arrs
        dags[k].meshlet_count = d.meshlet_count
        dags[k].info = _u(arrs[0])
        dags[k].group = arrs[1].ctypes.data_as(C.POINTER(C.c_int32))
        dags[k].start, dags[k].list = _u(arrs[2]), _u(arrs[3])
        base[k] = b
        b += d.meshlet_count
    slots = np.ascontiguousarray(instance_slots, np.uint32)
    e = np.ascontiguousarray(entries, np.uint32).reshape(-1, 3)
    st = np.ascontiguousarray(steps, np.uint32)
    checked = C.c_uint64()
    bad = lib().vgo_cut_invariant(C.addressof(dags), _u(base), len(meshes), _u(slots), len(slots), _u(e), len(e),
                                  _u(st), len(st), threads, C.byref(checked))
    return int(bad), int(checked.value)


def logf(x: float) -> float:
    return lib().vgo_logf(x)


# ------------------------------------------------------------------ Part B: per-frame passes
class _Scene(C.Structure):
    P, F, U = C.POINTER, C.POINTER(C.c_float), C.POINTER(C.c_uint32)
    _fields_ = [("mesh_count", C.c_uint32), ("mesh_sphere", F), ("mesh_lod_bounds", F), ("mesh_cull_bounds", F),
                ("mesh_max_draw_distance", F), ("mesh_min_pixel_radius", F), ("mesh_level_count", U),
                ("mesh_level_base", U), ("mesh_enabled", U), ("mesh_shadow", U), ("mesh_occlusion", U),
                ("level_first", U), ("level_size", U), ("level_errors", F), ("level_guard_errors", F),
                ("meshlet_count", C.c_uint32), ("meshlet_bounds", F), ("meshlet_tri_count", U),
                ("instance_count", C.c_uint32), ("instance_matrices", F), ("cell_count", C.c_uint32), ("cell_data", F)]


class _View(C.Structure):
    _fields_ = [("view", C.c_double * 16), ("proj", C.c_double * 16), ("near_", C.c_double),
                ("viewport_height", C.c_double), ("error_threshold", C.c_double), ("lod_blend", C.c_double),
                ("min_pixel_radius", C.c_double), ("shadow_error_scale", C.c_double),
                ("max_error_threshold", C.c_double), ("shadow_sweep", C.c_double * 3), ("frustum_culling", C.c_uint32),
                ("occlusion_active", C.c_uint32), ("hzb", C.POINTER(C.c_float)), ("hzb_levels", C.c_uint32),
                ("hzb_offset", C.c_uint32 * 16), ("hzb_width", C.c_uint32 * 16), ("hzb_height", C.c_uint32 * 16),
                ("max_drawn", C.c_uint32), ("index_capacity", C.c_uint32 * 2), ("state", C.c_uint32 * 8),
                ("triangle_budget", C.c_double), ("threshold_range", C.c_double * 2),
                ("chosen_threshold", C.c_double), ("predicted_triangles", C.c_uint64), ("cascade", C.c_uint32),
                ("cascade_clip", C.c_double * 16), ("cut_state", (C.c_uint32 * 2) * 2), ("pin_state", C.c_uint32)]


class _Result(C.Structure):
    _fields_ = [("entry_capacity", C.c_uint32), ("entries", C.POINTER(C.c_uint32) * 2), ("entry_count", C.c_uint32 * 2),
                ("counters", C.c_uint32 * 12), ("mesh_counts", C.POINTER(C.c_uint32)),
                ("draw_args", C.POINTER(C.c_uint32)), ("rounds", C.c_uint32), ("max_selected", C.c_uint32 * 2)]


class OracleScene:
    """The pool-global scene arrays the oracle reads, built from meshes, GPU-ordered matrices and cell records.

    meshes: list of (VirtualMeshData, dict of flags). matrices: (I, 16) float32 in GPU order (Morton per mesh, meshes
    concatenated in slot order). cells: (C, 8) float32 (centre, radius, max radius, slot, first, count).
    """

    def __init__(self, meshes, matrices: np.ndarray, cells: np.ndarray):
        n = len(meshes)
        self.keep = []
        k = self.keep.append
        sph, lodb, cullb = (np.zeros((n, 4), np.float32) for _ in range(3))
        mdd, mpr = np.zeros(n, np.float32), np.zeros(n, np.float32)
        lcount, lbase, en, sh, oc = (np.zeros(n, np.uint32) for _ in range(5))
        lf, ls, le, lg, mb, mt = [], [], [], [], [], []
        meshlet_base = 0
        level_base = 0
        for i, (d, f) in enumerate(meshes):
            sph[i], lodb[i], cullb[i] = d.bounding_sphere, d.lod_bounds_sphere, d.cull_bounds_sphere
            dd = f.get("max_draw_distance", 0.0)
            mdd[i] = dd if (dd > 0 and dd < 1e30) else 1e30
            mpr[i] = f.get("min_pixel_radius", 0.0)
            en[i] = 1 if f.get("enabled", True) else 0
            sh[i] = 1 if f.get("shadow", False) else 0
            oc[i] = 1 if f.get("occlusion", False) else 0
            L = len(d.level_ranges) // 2
            lcount[i], lbase[i] = L, level_base
            lr = d.level_ranges.reshape(-1, 2)
            lf.append(lr[:, 0] + meshlet_base)
            ls.append(lr[:, 1])
            le.append(d.level_errors)
            lg.append(d.level_guard_errors)
            mb.append(d.meshlet_bounds)
            mt.append(d.meshlet_info.reshape(-1, 4)[:, 0])
            meshlet_base += d.meshlet_count
            level_base += L
        arrs = dict(sph=sph, lodb=lodb, cullb=cullb, mdd=mdd, mpr=mpr, lcount=lcount, lbase=lbase, en=en, sh=sh, oc=oc,
                    lf=np.concatenate(lf).astype(np.uint32), ls=np.concatenate(ls).astype(np.uint32),
                    le=np.concatenate(le).astype(np.float32), lg=np.concatenate(lg).astype(np.float32),
                    mb=np.concatenate(mb).astype(np.float32), mt=np.concatenate(mt).astype(np.uint32),
                    mats=np.ascontiguousarray(matrices, np.float32).reshape(-1), cells=np.ascontiguousarray(cells, np.float32).reshape(-1))
        for v in arrs.values():
            k(v)
        s = _Scene()
        s.mesh_count = n
        s.mesh_sphere, s.mesh_lod_bounds, s.mesh_cull_bounds = _f(arrs["sph"]), _f(arrs["lodb"]), _f(arrs["cullb"])
        s.mesh_max_draw_distance, s.mesh_min_pixel_radius = _f(arrs["mdd"]), _f(arrs["mpr"])
        s.mesh_level_count, s.mesh_level_base = _u(arrs["lcount"]), _u(arrs["lbase"])
        s.mesh_enabled, s.mesh_shadow, s.mesh_occlusion = _u(arrs["en"]), _u(arrs["sh"]), _u(arrs["oc"])
        s.level_first, s.level_size = _u(arrs["lf"]), _u(arrs["ls"])
        s.level_errors, s.level_guard_errors = _f(arrs["le"]), _f(arrs["lg"])
        s.meshlet_count = meshlet_base
        s.meshlet_bounds, s.meshlet_tri_count = _f(arrs["mb"]), _u(arrs["mt"])
        s.instance_count = len(arrs["mats"]) // 16
        s.instance_matrices = _f(arrs["mats"])
        s.cell_count = len(arrs["cells"]) // 8
        s.cell_data = _f(arrs["cells"])
        self.struct = s
        self.mesh_count = n


def hzb_build(depth: np.ndarray):
    """Returns (mips as one float32 array, levels, offsets, widths, heights)."""
    d = np.ascontiguousarray(depth, np.float32)
    h, w = d.shape
    out = np.zeros(int(w * h * 1.5) + 64, np.float32)
    levels = C.c_uint32()
    off, ww, hh = (C.c_uint32 * 16)(), (C.c_uint32 * 16)(), (C.c_uint32 * 16)()
    n = lib().vgo_hzb_build(_f(d), w, h, _f(out), len(out), C.byref(levels), off, ww, hh)
    assert n >= 0
    return out[:n].copy(), levels.value, list(off), list(ww), list(hh)


def make_view(camera, params, max_drawn=1 << 20, index_capacity=(30_000_000, 12_000_000), hzb=None, state=None,
              pin_state: bool = False) -> _View:
    """The oracle's view of a camera and levers. `pin_state`: one round at `state` (no capacity check, retry or
    steer), to assess a cut's decisions at the controller state another run's final round used."""
    v = _View()
    v.pin_state = 1 if pin_state else 0
    for i in range(16):
        v.view[i] = float(camera.view[i])
        v.proj[i] = float(camera.proj[i])
    v.near_ = float(camera.near)
    v.viewport_height = float(camera.height)
    v.error_threshold = params.error_threshold
    v.lod_blend = params.lod_blend
    v.min_pixel_radius = params.min_pixel_radius
    v.shadow_error_scale = params.shadow_error_scale
    v.max_error_threshold = params.max_error_threshold
    for i in range(3):
        v.shadow_sweep[i] = float(params.shadow_sweep[i])
    v.frustum_culling = 1 if params.frustum_culling else 0
    v.max_drawn = max_drawn
    v.index_capacity[0], v.index_capacity[1] = index_capacity
    st = state if state is not None else [10000, 10000, 0, 0, 0, 0, 0, 0]
    for i in range(8):
        v.state[i] = int(st[i])
    v.triangle_budget = float(getattr(params, "triangle_budget", 0.0))
    clip = getattr(params, "cascade_clip", None)
    v.cascade = 1 if clip is not None else 0
    if clip is not None:
        for k in range(16):
            v.cascade_clip[k] = float(clip[k])
    tr = getattr(params, "threshold_range", (0.5, 3.0))
    v.threshold_range[0], v.threshold_range[1] = float(tr[0]), float(tr[1])
    v.occlusion_active = 0
    if hzb is not None:
        mips, levels, off, ww, hh = hzb
        v._hzb_keep = mips
        v.hzb = _f(mips)
        v.hzb_levels = levels
        for i in range(16):
            v.hzb_offset[i], v.hzb_width[i], v.hzb_height[i] = off[i], ww[i], hh[i]
        v.occlusion_active = 1
    return v


def cut_state_words(view: _View, state, cut: int) -> list:
    """The state words a pinned run of cut `cut` starts from: `state` with the scales that cut's final computation
    in `view`'s pass ran with."""
    st = list(state)
    st[0], st[1] = int(view.cut_state[cut][0]), int(view.cut_state[cut][1])
    return st


def pinned_reference(scene: OracleScene, make, mirror_view: _View, state, threads: int = 0):
    """The double restatement of each cut at the controller scales its final computation in the mirror's pass ran
    with (one pinned round per cut). `make(state)` builds the pinned view. Returns (entries per cut, view per cut):
    the views are what `explain` takes for that cut."""
    entries, views = [], []
    for cut in (0, 1):
        v = make(cut_state_words(mirror_view, state, cut))
        v.pin_state = 1
        r = cull_pass(scene, v, "f64", threads=threads)
        entries.append(r["entries"][cut])
        views.append(v)
    return entries, views


def cull_pass(scene: OracleScene, view: _View, precision: str = "f32", threads: int = 0, capacity: int | None = None):
    """Runs the full per-frame pass; returns dict with entries per cut ((n, 3) u32), counters, mesh_counts, args."""
    cap = capacity if capacity is not None else view.max_drawn
    e0 = np.zeros((cap, 3), np.uint32)
    e1 = np.zeros((cap, 3), np.uint32)
    mc = np.zeros(scene.mesh_count * 4, np.uint32)
    args = np.zeros(scene.mesh_count * 4 * 5, np.uint32)
    r = _Result()
    r.entry_capacity = cap
    r.entries[0], r.entries[1] = _u(e0), _u(e1)
    r.mesh_counts, r.draw_args = _u(mc), _u(args)
    fn = lib().vgo_cull_pass_f32 if precision == "f32" else lib().vgo_cull_pass_f64
    fn(C.addressof(scene.struct), C.addressof(view), C.addressof(r), threads)
    return dict(entries=[e0[:r.entry_count[0]].copy(), e1[:r.entry_count[1]].copy()], counters=list(r.counters),
                mesh_counts=mc.reshape(2, scene.mesh_count, 2), draw_args=args.reshape(2, scene.mesh_count, 2, 5),
                rounds=r.rounds, state=list(view.state), threshold=view.chosen_threshold,
                predicted=view.predicted_triangles, max_selected=list(r.max_selected))


def explain(scene: OracleScene, view: _View, cut: int, instance: int, meshlet: int) -> float:
    return lib().vgo_explain_f64(C.addressof(scene.struct), C.addressof(view), cut, instance, meshlet)


# ------------------------------------------------------------------ scene layout restated (host side of the reference)
def _spread10(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint32) & 0x3FF
    v = (v | (v << 16)) & 0x030000FF
    v = (v | (v << 8)) & 0x0300F00F
    v = (v | (v << 4)) & 0x030C30C3
    v = (v | (v << 2)) & 0x09249249
    return v


def instance_spheres(matrices: np.ndarray, sphere) -> np.ndarray:
    """instanceSphere (GeometryPool.ts:1171-1180) in double for every instance: (n, 4)."""
    m = np.asarray(matrices, np.float64).reshape(-1, 16)
    sx, sy, sz, sr = (float(x) for x in sphere)
    out = np.empty((len(m), 4))
    out[:, 0] = m[:, 0] * sx + m[:, 4] * sy + m[:, 8] * sz + m[:, 12]
    out[:, 1] = m[:, 1] * sx + m[:, 5] * sy + m[:, 9] * sz + m[:, 13]
    out[:, 2] = m[:, 2] * sx + m[:, 6] * sy + m[:, 10] * sz + m[:, 14]
    c = [np.sqrt(m[:, k] ** 2 + m[:, k + 1] ** 2 + m[:, k + 2] ** 2) for k in (0, 4, 8)]
    out[:, 3] = sr * np.maximum(c[0], np.maximum(c[1], c[2]))
    return out


def morton_codes(matrices: np.ndarray, sphere) -> np.ndarray:
    """The 30-bit Morton codes mortonOrder (GeometryPool.ts:1263-1284) sorts by: sphere centres quantised to 1024
    steps of the largest extent over the instances."""
    s = instance_spheres(matrices, sphere)
    if len(s) == 0:
        return np.zeros(0, np.uint32)
    lo, hi = s[:, :3].min(0), s[:, :3].max(0)
    extent = max(float((hi - lo).max()), 1e-9)
    q = np.clip(np.floor((s[:, :3] - lo) / extent * 1024), 0, 1023).astype(np.uint32)
    return _spread10(q[:, 0]) | (_spread10(q[:, 1]) << 1) | (_spread10(q[:, 2]) << 2)


def morton_order(matrices: np.ndarray, sphere) -> np.ndarray:
    """mortonOrder (GeometryPool.ts:1263-1284): stable sort by 30-bit Morton code of the sphere centres."""
    return np.argsort(morton_codes(matrices, sphere), kind="stable").astype(np.uint32)


def compute_cells(matrices_gpu: np.ndarray, sphere, slot: int, instance_base: int, cell_size: int = 128) -> np.ndarray:
    """computeCell (GeometryPool.ts:519-545) for every cell of one mesh: (cells, 8) float32."""
    s = instance_spheres(matrices_gpu, sphere)
    n = len(s)
    out = []
    for first in range(0, n, cell_size):
        t = s[first:first + cell_size]
        lo = (t[:, :3] - t[:, 3:4]).min(0)
        hi = (t[:, :3] + t[:, 3:4]).max(0)
        c = (lo + hi) / 2
        radius = float((np.sqrt(((t[:, :3] - c) ** 2).sum(1)) + t[:, 3]).max())
        max_r = float(t[:, 3].max())
        out.append([c[0], c[1], c[2], radius * (1 + 1e-4) + 1e-3, max_r * (1 + 1e-4) + 1e-4, slot,
                    instance_base + first, len(t)])
    return np.array(out, np.float32).reshape(-1, 8)


def scene_from_spec(meshes, instances, flags=None, orders_in=None) -> tuple[OracleScene, np.ndarray, list]:
    """OracleScene for meshes added in order (slot i = mesh i); returns it, the GPU-order matrices and the per-mesh
    Morton orders. `orders_in`: GPU orders to keep (a scene whose instances moved after it was added keeps the order
    it was added with)."""
    flags = flags or [{} for _ in meshes]
    mats, cells, orders = [], [], []
    base = 0
    for slot, (d, m) in enumerate(zip(meshes, instances)):
        m = np.asarray(m, np.float32).reshape(-1, 16)
        order = morton_order(m, d.bounding_sphere) if orders_in is None else np.asarray(orders_in[slot])
        g = m[order]
        mats.append(g)
        cells.append(compute_cells(g, d.bounding_sphere, slot, base))
        orders.append(order)
        base += len(g)
    allm = np.concatenate(mats) if mats else np.zeros((0, 16), np.float32)
    allc = np.concatenate(cells) if cells else np.zeros((0, 8), np.float32)
    return OracleScene(list(zip(meshes, flags)), allm, allc), allm, orders


def _pool_arrays(meshes, vertex_flags):
    """The engine's pool layout of the meshes (add order): meshlet info with pool-global triangle and
    meshlet-vertex offsets, packed triangles, and the meshlet vertices / positions of the meshes flagged in
    `vertex_flags` (pool-global vertex ids)."""
    infos, tris, mverts, pos = [], [], [], []
    tri_base = mv_base = v_base = 0
    for d, occ in zip(meshes, vertex_flags):
        info = np.asarray(d.meshlet_info, np.uint32).reshape(-1, 4).copy()
        info[:, 1] += np.uint32(tri_base * 3)
        info[:, 3] += np.uint32(mv_base)
        infos.append(info)
        t = np.asarray(d.meshlet_triangles, np.uint32)
        tris.append(t)
        tri_base += len(t)
        if occ:
            mv = np.asarray(d.meshlet_vertices, np.uint32) + np.uint32(v_base)
            p = np.asarray(d.positions, np.float32).reshape(-1, 3)
            mverts.append(mv)
            pos.append(p)
            mv_base += len(mv)
            v_base += len(p)
    m_info = np.ascontiguousarray(np.concatenate(infos), np.uint32)
    m_tris = np.ascontiguousarray(np.concatenate(tris), np.uint32)
    m_verts = np.ascontiguousarray(np.concatenate(mverts) if mverts else np.zeros(1, np.uint32), np.uint32)
    positions = np.ascontiguousarray(np.concatenate(pos) if pos else np.zeros((1, 3), np.float32), np.float32)
    return m_info, m_tris, m_verts, positions


def occluder_depth(meshes, occluder_flags, gpu_mats, inst_slot, entries, camera, width: int, height: int) -> np.ndarray:
    """The occluder depth pass restated (vg_raster.c) over the same pool layout the engine builds: meshes in add
    order, meshlet / triangle / meshlet-vertex / vertex ids rebased to pool-global, vertex data only for occluders.
    `entries`: (n, 4) uint32 draw-list entries of the source cut; returns the (height, width) float32 depth."""
    m_info, m_tris, m_verts, positions = _pool_arrays(meshes, occluder_flags)
    e = np.ascontiguousarray(entries, np.uint32).reshape(-1, 4)
    mats = np.ascontiguousarray(gpu_mats, np.float32)
    slots = np.ascontiguousarray(inst_slot, np.uint32)
    flags = np.ascontiguousarray([1 if f else 0 for f in occluder_flags], np.uint32)
    view = np.ascontiguousarray(camera.view, np.float64)
    proj = np.ascontiguousarray(camera.proj, np.float64)
    out = np.zeros((height, width), np.float32)
    L = lib()
    L.vgo_occluder_depth(_u(e), len(e), _f(mats), _u(slots), _u(flags), _u(m_info), _u(m_tris), _u(m_verts),
                         _f(positions), view.ctypes.data_as(C.POINTER(C.c_double)),
                         proj.ctypes.data_as(C.POINTER(C.c_double)), width, height, _f(out))
    return out


def blend_keep(px: int, py: int, frame: int, lo: int, hi: int) -> bool:
    """lodBlendMask (lodBlend.ts:36-45) at pixel (px, py), as vg_raster.c computes it."""
    return bool(lib().vgo_blend_keep(px, py, frame, lo, hi))


def visibility(meshes, vertex_flags, max_draw_distance, gpu_mats, inst_slot, indices, draw_list, args, camera,
               width: int, height: int, frame: int = 0, fade_camera=None) -> np.ndarray:
    """The visibility pass restated (vg_raster.c) over the engine's pool layout: `vertex_flags` per mesh, whether its
    vertex data was uploaded; `indices` the expanded index buffer, `draw_list` the output slot's entries of both cuts
    ((2 max_drawn, 4) u32), `args` the cut's draw args ((regions, 5) u32), `max_draw_distance` per mesh (as given to
    the engine; inf = none). Returns the (height, width) uint64 image."""
    has_vertices = [bool(f) for f in vertex_flags]
    m_info, _, m_verts, positions = _pool_arrays(meshes, has_vertices)
    n_verts = sum(len(np.asarray(d.meshlet_vertices)) for d, f in zip(meshes, has_vertices) if f)
    n_pos = sum(len(np.asarray(d.positions)) // 3 for d, f in zip(meshes, has_vertices) if f)
    maxd = np.array([np.float32(x) if (x > 0 and x < 1e30) else np.float32(1e30) for x in max_draw_distance],
                    np.float32)
    idx = np.ascontiguousarray(indices, np.uint32)
    dl = np.ascontiguousarray(draw_list, np.uint32).reshape(-1, 4)
    a = np.ascontiguousarray(args, np.uint32).reshape(-1, 5)
    mats = np.ascontiguousarray(gpu_mats, np.float32)
    slots = np.ascontiguousarray(inst_slot, np.uint32)
    flags = np.ascontiguousarray([1 if f else 0 for f in has_vertices], np.uint32)
    fc = fade_camera if fade_camera is not None else camera
    view = np.ascontiguousarray(camera.view, np.float64)
    proj = np.ascontiguousarray(camera.proj, np.float64)
    fview = np.ascontiguousarray(fc.view, np.float64)
    out = np.zeros((height, width), np.uint64)
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    lib().vgo_visibility(_u(idx), len(idx), _u(dl), len(dl), _u(a), len(a), _f(mats), len(mats), _u(slots), _u(flags),
                         _f(maxd), _u(m_info), len(m_info), _u(m_verts), n_verts, _f(positions), n_pos, dp(view),
                         dp(proj), dp(fview), width, height, frame, out.ctypes.data_as(C.POINTER(C.c_uint64)))
    return out
