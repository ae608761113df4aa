"""Shared helpers for comparing the GPU cut with the oracle (test infrastructure)."""
from __future__ import annotations

import numpy as np

import oracle as O
from vgcut import engine, scenes

MARGIN = 1e-5  # relative margin of the parity contract: decisions closer than this to a threshold are reported


def small_ruins(seed=3, meshes=6, instances=3000, extent=220.0, poses=6, tri_lo=2_000, tri_hi=30_000, quads=24,
                width=960, height=540):
    return scenes.ruins(seed=seed, mesh_count=meshes, tri_lo=tri_lo, tri_hi=tri_hi, instances=instances, extent=extent,
                        poses=poses, width=width, height=height, target_full_detail=instances * 8_000, quads=quads)


def grid_matrices(n: int, spacing: float, seed: int) -> np.ndarray:
    """n instances on a square grid (column-major 4x4), seeded yaw and lognormal scale."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(max(n, 1))))
    out = np.zeros((n, 16), np.float32)
    for i in range(n):
        yaw, s = rng.uniform(0, 2 * np.pi), np.exp(rng.normal(0.0, 0.2))
        c, sn = np.cos(yaw) * s, np.sin(yaw) * s
        out[i] = [c, 0, -sn, 0, 0, s, 0, 0, sn, 0, c, 0, (i % side) * spacing, 0, (i // side) * spacing, 1]
    return out


def d2h(ptr, count: int, dtype=np.uint32) -> np.ndarray:
    """Copies `count` elements from a device pointer (cudaMemcpy through the CUDA runtime the engine loaded)."""
    import ctypes
    rt = ctypes.CDLL("libcudart.so.12")
    out = np.zeros(count, dtype)
    rc = rt.cudaMemcpy(out.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(ptr), ctypes.c_size_t(out.nbytes), 2)
    assert rc == 0, f"cudaMemcpy failed ({rc})"
    return out


def key_set(entries: np.ndarray, cols=(0, 1, 2)) -> set:
    e = np.asarray(entries)
    return set(map(tuple, e[:, list(cols)].tolist())) if len(e) else set()


def check_index_tiling(entries: np.ndarray, inst_slot: np.ndarray, mesh_counts: np.ndarray, cut: int) -> None:
    """firstIndex values of each (slot, part) tile [0, requested) exactly (atomic order is free, the packing is not)."""
    e = np.asarray(entries)
    if len(e) == 0:
        return
    part = np.where((e[:, 3] & 0xFFFF00) == (255 << 16), 0, 1)
    slot = inst_slot[e[:, 0]]
    tris = e[:, 3] & 255
    for s in np.unique(slot):
        for p in (0, 1):
            m = (slot == s) & (part == p)
            if not m.any():
                continue
            order = np.argsort(e[m, 2], kind="stable")
            first = e[m, 2][order].astype(np.int64)
            size = 3 * tris[m][order].astype(np.int64)
            assert first[0] == 0
            assert np.all(first[1:] == first[:-1] + size[:-1]), "index regions overlap or leave gaps"
            assert first[-1] + size[-1] == mesh_counts[cut, s, p]


class Harness:
    """One scene resident on the GPU and in the oracle."""

    def __init__(self, spec, flags=None, max_meshlets=1 << 16, max_triangles=2_000_000, max_shadow=1_000_000,
                 output_slots=8):
        self.spec = spec
        self.flags = flags or [{} for _ in spec.meshes]
        self.vg = engine.VirtualGeometry(max_triangles=max_triangles, max_shadow_triangles=max_shadow,
                                         max_meshlets=max_meshlets, output_slots=output_slots)
        for d, m, f in zip(spec.meshes, spec.instances, self.flags):
            self.vg.create_mesh(d, m, max_draw_distance=f.get("max_draw_distance", float("inf")),
                                min_pixel_radius=f.get("min_pixel_radius", 0.0), cast_shadow=f.get("shadow", False),
                                occlusion_culling=f.get("occlusion", False), occluder=f.get("occluder", False),
                                vertex_data=f.get("vertex_data", False))
        self.scene, self.mats, self.orders = O.scene_from_spec(spec.meshes, spec.instances, self.flags)
        self.inst_slot = np.concatenate([np.full(len(m), i, np.uint32) for i, m in enumerate(spec.instances)])
        self.max_meshlets, self.caps = max_meshlets, (max_triangles * 3, max_shadow * 3)
        self.order_dependent = 0  # compared views whose draw list overflowed in some round (see compare)

    def check_layout(self):
        cells, mats = self.vg.debug_scene()
        assert np.array_equal(mats, self.mats), "instance order (Morton) differs from the oracle's"
        ocells = np.asarray(self.scene.keep[-1]).reshape(-1, 8)
        assert np.array_equal(cells, ocells), "cell records differ from the oracle's computeCell"

    def oracle(self, cam, params, hzb=None, precision="f32", state=None):
        v = O.make_view(cam, params, self.max_meshlets, self.caps, hzb=hzb, state=state)
        return O.cull_pass(self.scene, v, precision), v

    def reference(self, cam, params, hzb=None):
        """The double restatement of the reference's cut, each cut at the controller scales its final computation
        in the last compared run used (pinned: one round, no capacity check). The controller's own arithmetic is
        checked bit for bit against the float mirror; pinning keeps one margin decision in an early round from
        moving a retried cut's scale, which would shift every decision of the view. Returns (entries per cut,
        oracle view per cut)."""
        if getattr(params, "triangle_budget", 0.0) > 0:  # assess the cut at the threshold the search picked
            import dataclasses
            params = dataclasses.replace(params, triangle_budget=0.0,
                                         error_threshold=float(self.last_view.chosen_threshold))
        make = lambda st: O.make_view(cam, params, self.max_meshlets, self.caps, hzb=hzb, state=st)
        return O.pinned_reference(self.scene, make, self.last_view, self.last_state)

    def gpu(self, cam, params, slot=0, graph=False):
        v = engine.make_view(cam, params)
        self.vg.cut([v], first_slot=slot, graph=graph)
        stats = self.vg.read_stats(slot)
        lists = [self.vg.draw_list(slot, c) for c in (0, 1)]
        return stats, lists

    def compare(self, cam, params, hzb_oracle=None, slot=0, graph=False):
        """GPU result == float mirror (sets, counters, args); returns (gpu lists, oracle result)."""
        state = list(self.vg.state(params.state_slot))  # the controller state both start from
        if getattr(params, "fresh_state", False):
            state = [10000, 10000, 0, 0, 0, 0, 0, 0]
        res, self.last_view = self.oracle(cam, params, hzb_oracle, "f32", state)
        self.last_state = state
        stats, lists = self.gpu(cam, params, slot, graph)
        c = res["counters"]
        assert stats["faults"] == 0, "a kernel gave up waiting"
        assert stats["visible_cells"] == c[0]
        if any(m > self.max_meshlets for m in res["max_selected"]):
            # A round selected more meshlets than the draw list holds: the GPU kept the subset its atomics reached
            # first, and the capacity controller's fill (the kept entries' index count) - so the next round's scale,
            # the final state and everything after - follows from that order (as in the reference, whose controller
            # counts kept entries too). Only the order-independent part is compared; tests keep this count at 0.
            self.order_dependent += 1
            return lists, res
        assert stats["occluded_instances"] == c[1]
        for cut in (0, 1):
            k = c[2 + cut * 5: 7 + cut * 5]
            got = [stats["selected"][cut], stats["drawn"][cut], stats["survived"][cut], stats["work"][cut],
                   stats["requested_indices"][cut]]
            assert got == k, f"cut {cut} counters gpu {got} oracle {k}"
            g = key_set(lists[cut], (0, 1, 3))
            o = key_set(res["entries"][cut], (0, 1, 2))
            assert g == o, f"cut {cut}: {len(g - o)} only on GPU, {len(o - g)} only in the oracle"
            check_index_tiling(lists[cut], self.inst_slot, res["mesh_counts"], cut)
        assert stats["rounds"] == res["rounds"]
        out = self.vg.output(slot)
        args = d2h(out.draw_args, 2 * out.mesh_slots * 2 * 5).reshape(2, out.mesh_slots, 2, 5)
        n = len(self.spec.meshes)
        for cut in (0, 1):
            assert np.array_equal(args[cut, :n], res["draw_args"][cut]), "drawIndexedIndirect args differ"
        st = self.vg.state(params.state_slot)
        assert list(st) == res["state"], f"controller state gpu {list(st)} oracle {res['state']}"
        return lists, res


# ------------------------------------------------------------------ the hand-derived pass scene (tests/golden)
def tiny_dag_mesh(t: dict):
    """The golden vectors' three-meshlet DAG as a VirtualMeshData-shaped record (LOD, cull and bounding spheres
    (0, 0, 0, 1))."""
    from types import SimpleNamespace
    return SimpleNamespace(
        meshlet_count=3, meshlet_bounds=np.array(t["bounds"], np.float32).reshape(-1),
        meshlet_info=np.array(t["info"], np.uint32).reshape(-1), level_ranges=np.array(t["level_ranges"], np.uint32),
        level_errors=np.array(t["level_errors"], np.float32),
        level_guard_errors=np.array(t["level_guard_errors"], np.float32),
        lod_bounds_sphere=np.array(t["lod_bounds_sphere"], np.float32),
        cull_bounds_sphere=np.array([0, 0, 0, 1], np.float32), bounding_sphere=np.array([0, 0, 0, 1], np.float32),
        meshlet_triangles=np.array([0x020100, 0x030201, 0x020100, 0x030201, 0x020100], np.uint32),
        replacement_group=np.array(t["replacement_group"], np.int32),
        replacement_start=np.array(t["replacement_start"], np.uint32),
        replacement_indices=np.array(t["replacement_indices"], np.uint32), stats={"leafTriangles": 4})


def golden_pass_scene(vectors: dict):
    """(spec, flags, camera, names) of the golden pass scene: one tiny-DAG mesh per instance, camera at the origin
    looking down -z with fov 90, near 1, far 100 and a 200 x 200 viewport (projScale 100)."""
    from types import SimpleNamespace
    from vgcut.camera import Camera, compose
    g = vectors["pass_scene"]
    mesh = tiny_dag_mesh(vectors["tiny_dag"])
    a = -100.0 / 99.0
    proj = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, a, -1, 0, 0, a, 0], float)
    cam = Camera(view=np.eye(4).reshape(-1), proj=proj, near=1.0, height=200.0, width=200.0)
    instances, flags = [], []
    for inst in g["instances"]:
        instances.append(np.array([compose(inst["at"], 0.0, inst["s"])], np.float32))
        flags.append(dict(max_draw_distance=inst.get("max_draw_distance", float("inf")),
                          min_pixel_radius=inst.get("min_pixel_radius", 0.0), shadow=inst.get("shadow", False),
                          occlusion=inst.get("occlusion", False), enabled=inst.get("enabled", True)))
    spec = SimpleNamespace(meshes=[mesh] * len(instances), instances=instances)
    return spec, flags, cam, [inst["name"] for inst in g["instances"]]


def check_golden_view(view: dict, names: list, cuts: list, counters: dict) -> None:
    """Asserts a golden pass view's expectations. cuts[c]: (n, 3) (instance, pool-global meshlet, packed);
    counters: visible_cells, work0, occluded_instances and (GPU only) fast_emitted."""
    e = view["expect"]
    idx = {n: i for i, n in enumerate(names)}
    by_inst = [dict() for _ in range(2)]
    for c in (0, 1):
        for inst, m, packed in np.asarray(cuts[c]).reshape(-1, 3).tolist():
            by_inst[c].setdefault(names[inst], set()).add((m - 3 * inst, packed))
    for name, want in e.get("cut0", {}).items():
        assert by_inst[0].get(name, set()) == set(map(tuple, want)), f"view {view['name']}: {name} in the camera cut"
    for name in e.get("present0", []):
        assert by_inst[0].get(name), f"view {view['name']}: {name} must be drawn"
    for name in e.get("absent0", []):
        assert name not in by_inst[0], f"view {view['name']}: {name} must not be drawn"
    if "only" not in e and "cut0" in e and "present0" in e:  # the full camera cut is listed
        listed = set(e["cut0"]) | set(e["present0"])
        assert set(by_inst[0]) == listed, f"view {view['name']}: drawn {sorted(by_inst[0])}"
    if "cut1" in e:
        got = {(names[i], m - 3 * i, p) for i, m, p in np.asarray(cuts[1]).reshape(-1, 3).tolist()}
        assert got == set(map(tuple, e["cut1"])), f"view {view['name']}: shadow cut {got}"
    for k in ("visible_cells", "work0", "occluded_instances", "fast_emitted"):
        if k in e and k in counters:
            assert counters[k] == e[k], f"view {view['name']}: {k} {counters[k]} != {e[k]}"
