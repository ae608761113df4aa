"""The oracle's float mirror (the kernels' arithmetic) against its double restatement (the reference's semantics):
every difference is a decision within the 1e-5 relative margin, and the DAG-cut invariant (every leaf covered
exactly once) holds per instance in both precisions."""
import math

import numpy as np
import pytest

import oracle as O
from vgcut import engine, scenes
from vgcut.camera import Camera
from parity_util import MARGIN, key_set, small_ruins


@pytest.fixture(scope="module")
def small_plain():
    spec = scenes.plain_small(n=40, seed=1)
    scene, mats, _ = O.scene_from_spec(spec.meshes, spec.instances)
    return spec, scene


def cameras(n, radius, height, seed):
    r = np.random.default_rng(seed)
    return [Camera.perspective_look_at((math.cos(a) * d, height * h, math.sin(a) * d), (0, 0, 0), 60, 1920, 1080,
                                       0.1, 1000)
            for a, d, h in zip(r.uniform(0, 2 * math.pi, n), radius * r.uniform(0.3, 1.5, n), r.uniform(0.05, 1.5, n))]


def differences_explained(scene, cam, params, hzb=None):
    """Float mirror vs the double restatement, the latter at the controller state the mirror's final round used."""
    v32 = O.make_view(cam, params, hzb=hzb)
    a = O.cull_pass(scene, v32, "f32")
    b, views = O.pinned_reference(scene, lambda st: O.make_view(cam, params, hzb=hzb, state=st), v32,
                                  [10000, 10000, 0, 0, 0, 0, 0, 0])
    near = 0
    for cut in (0, 1):
        ka, kb = key_set(a["entries"][cut]), key_set(b[cut])
        for inst, m, _ in ka ^ kb:
            s = O.explain(scene, views[cut], cut, inst, m)
            assert s <= MARGIN, f"cut {cut} ({inst}, {m}) differs between float and double with slack {s}"
            near += 1
    return near, len(key_set(b[0]))


@pytest.mark.parametrize("threshold", [0.5, 1.0, 2.0, 3.0])
def test_float_mirror_within_margin(small_plain, threshold):
    spec, scene = small_plain
    near = total = 0
    for cam in cameras(10, 30, 10, seed=int(threshold * 10)):
        n, t = differences_explained(scene, cam, engine.ViewParams(error_threshold=threshold))
        near, total = near + n, total + t
    assert total > 0
    assert near <= max(3, total // 1000)


def test_float_mirror_ruins_features():
    spec = small_ruins(poses=3)
    flags = [dict(shadow=(i % 2 == 0), occlusion=True) for i in range(len(spec.meshes))]
    scene, _, _ = O.scene_from_spec(spec.meshes, spec.instances, flags)
    for k, cam in enumerate(spec.cameras):
        hzb = O.hzb_build(spec.depth_images[k])
        p = engine.ViewParams(shadow_sweep=(20.0, -50.0, 5.0))
        differences_explained(scene, cam, p, hzb)


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("threshold,blend", [(1.0, 2.0), (2.0, 2.0), (3.0, 3.0), (0.5, 1.0)])
def test_dag_cut_invariant_per_instance(small_plain, precision, threshold, blend):
    """With culling off (frustum, size, distance, occlusion), each instance's drawn meshlets form a complete,
    overlap-free cut at every blend step (cut.test.ts invariants, applied to the full pass)."""
    spec, scene = small_plain
    d = spec.meshes[0]
    for cam in cameras(4, 25, 8, seed=3):
        p = engine.ViewParams(error_threshold=threshold, lod_blend=blend, frustum_culling=False, min_pixel_radius=0.0)
        r = O.cull_pass(scene, O.make_view(cam, p), precision)
        e = r["entries"][0]
        assert r["counters"][2] == len(e)
        for inst in np.unique(e[:, 0]):
            rows = e[e[:, 0] == inst]
            lo = np.zeros(d.meshlet_count, np.int64)
            hi = np.zeros(d.meshlet_count, np.int64)
            lo[rows[:, 1]] = (rows[:, 2] >> 8) & 255
            hi[rows[:, 1]] = (rows[:, 2] >> 16) & 255
            steps = range(0, 255, 17) if blend > 1 else [0]
            for s in steps:
                sel = ((lo <= s) & (s < hi)).astype(np.uint8)
                assert len(O.verify_cut_coverage(d, sel)) == 0, f"hole at step {s}"
                assert len(O.verify_cut_overlap(d, sel)) == 0, f"overlap at step {s}"
        # every instance is drawn (nothing is culled)
        assert len(np.unique(e[:, 0])) == spec.instance_count


def test_capacity_controller_mirror(small_plain):
    """Retry rounds and steering behave the same in float and double on an overflowing cut."""
    spec, scene = small_plain
    cam = cameras(1, 12, 4, seed=7)[0]
    p = engine.ViewParams(error_threshold=0.5)
    va = O.make_view(cam, p, max_drawn=200, index_capacity=(60_000, 30_000))
    vb = O.make_view(cam, p, max_drawn=200, index_capacity=(60_000, 30_000))
    a = O.cull_pass(scene, va, "f32", capacity=1 << 16)
    b = O.cull_pass(scene, vb, "f64", capacity=1 << 16)
    assert a["rounds"] == b["rounds"] >= 2
    assert a["state"][0] > 10000, "the camera cut was coarsened"
