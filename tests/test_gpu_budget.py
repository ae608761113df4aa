"""triangleBudget on the GPU against the oracle's float mirror.

The reference picks errorThreshold each frame so that the plain camera cut fits `triangleBudget` triangles
(VirtualGeometry.ts triangleBudget / thresholdRange levers). The engine builds a 256-bin histogram of the triangles
entering and leaving the cut over thresholdRange in one pass on the device, prefix-scans it and takes the smallest
threshold whose cut fits. The chosen bin, the predicted triangle count and the resulting draw lists must equal the
oracle's on the same inputs, plain and inside the batched CUDA graph, with occlusion and the shadow cut on.
"""
import numpy as np
import pytest

import oracle as O
from parity_util import Harness, key_set, small_ruins
from vgcut import engine, scenes
from vgcut.camera import Camera

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain():
    spec = scenes.plain_small(n=40, seed=1)
    return Harness(spec)


def check_budget(h, cam, params, hzb_oracle=None, graph=False):
    lists, res = h.compare(cam, params, hzb_oracle=hzb_oracle, graph=graph)
    s = h.vg.last_stats
    assert s["predicted_triangles"] == res["predicted"], f"prediction gpu {s['predicted_triangles']} oracle {res['predicted']}"
    assert s["effective_threshold"] == np.float32(res["threshold"]), "chosen threshold differs"
    drawn = s["requested_indices"][0] // 3
    if res["threshold"] < params.threshold_range[1]:  # the search found a threshold whose cut fits
        # the prediction counts the blend band, so the drawn camera cut (both parts) stays within the budget
        assert drawn <= s["predicted_triangles"] <= params.triangle_budget, \
            f"drawn {drawn} predicted {s['predicted_triangles']} budget {params.triangle_budget}"
    return lists, res


@pytest.mark.parametrize("blend", [1.0, 1.5])
def test_budget_plain_small(plain, blend):
    h = plain
    cams = [h.spec.cameras[0], Camera.perspective_look_at((14, 6, -9), (0, 0, 0), 60, 1920, 1080, 0.1, 1000)]
    for cam in cams:
        full, _ = h.oracle(cam, engine.ViewParams(error_threshold=0.5, lod_blend=1.0))
        full_tris = full["counters"][2 + 4] // 3
        for frac in (0.0001, 0.3, 0.7, 2.0):  # below the coarsest cut, in between, above the finest
            p = engine.ViewParams(lod_blend=blend, triangle_budget=max(1.0, full_tris * frac), threshold_range=(0.5, 3.0))
            lists, res = check_budget(h, cam, p)
            if blend == 1.0:  # without blend steps the prediction is the cut's drawn triangles
                assert h.vg.last_stats["requested_indices"][0] == 3 * res["predicted"]


def test_budget_ruins_with_occlusion_shadow_and_graph():
    spec = small_ruins(seed=7, poses=3)
    flags = [dict(shadow=(i % 2 == 0), occlusion=True) for i in range(len(spec.meshes))]
    h = Harness(spec, flags)
    for k, cam in enumerate(spec.cameras):
        h.vg.build_hzb(k, spec.depth_images[k])
        hzb = O.hzb_build(spec.depth_images[k])
        for graph in (False, True):
            p = engine.ViewParams(hzb=k, shadow_sweep=(30.0, -60.0, 10.0), triangle_budget=150_000.0,
                                  threshold_range=(0.25, 4.0))
            check_budget(h, cam, p, hzb_oracle=hzb, graph=graph)


def test_budget_mixed_batch(plain):
    """Views with and without a budget in one launch: each gets its own threshold, as when run alone."""
    h = plain
    cams = [Camera.perspective_look_at((10 + 3 * i, 5, -8 + 2 * i), (0, 0, 0), 60, 1280, 720, 0.1, 1000)
            for i in range(4)]
    params = [engine.ViewParams(error_threshold=1.0, state_slot=i) if i % 2 else
              engine.ViewParams(triangle_budget=20_000.0 * (i + 1), threshold_range=(0.5, 3.0), state_slot=i)
              for i in range(4)]
    fresh = np.array([10000, 10000, 0, 0, 0, 0, 0, 0], np.uint32)
    for i in range(4):
        h.vg.state(i, fresh)
    views = [engine.make_view(c, p) for c, p in zip(cams, params)]
    for graph in (False, True):
        for i in range(4):
            h.vg.state(i, fresh)
        h.vg.cut(views, first_slot=0, graph=graph)
        for i, (cam, p) in enumerate(zip(cams, params)):
            res, _ = h.oracle(cam, p, state=list(fresh))
            s = h.vg.read_stats(i)
            assert s["effective_threshold"] == np.float32(res["threshold"])
            assert s["predicted_triangles"] == (res["predicted"] if p.triangle_budget > 0 else 0)
            assert key_set(h.vg.draw_list(i, 0), (0, 1, 3)) == key_set(res["entries"][0], (0, 1, 2))


def test_reference_glide_controller_on_the_gpu(plain):
    """budget_mode="glide": the reference's CPU controller steers the threshold over frames from stats readbacks
    until the camera cut's triangles sit inside its +-15% band around the budget."""
    spec = plain.spec
    cam = spec.cameras[0]
    target_t = 1.5
    res, _ = plain.oracle(cam, engine.ViewParams(error_threshold=target_t))
    budget = float(res["counters"][2 + 4] // 3)
    vg = engine.VirtualGeometry(max_meshlets=1 << 16, budget_mode="glide")
    try:
        scenes.load_into(vg, spec)
        vg.error_threshold = 0.5
        vg.triangle_budget = budget
        vg.threshold_range = (0.5, 3.0)
        ts = []
        for _ in range(400):
            vg.update(cam)
            ts.append(vg.error_threshold)
        drawn = vg.read_stats(0)["requested_indices"][0] / 3
        assert abs(drawn / budget - 1) < 0.15, f"drawn {drawn} budget {budget} threshold {ts[-1]}"
        assert ts[0] == 0.5 and all(b <= a * 1.03 + 1e-9 for a, b in zip(ts, ts[1:]))  # glided, never jumped
    finally:
        vg.dispose()
