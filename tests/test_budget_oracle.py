"""triangleBudget histogram search in the oracle: the predicted triangles equal the cut's drawn triangles at the
chosen threshold (blend off, no occlusion), and one bin finer the cut exceeds the budget; with the LOD-blend band open
the prediction counts the band, so the drawn cut stays within the budget and within a few percent of the
prediction (meshlets at the band's edges whose blend range rounds to empty are predicted but not drawn)."""
import dataclasses

import numpy as np
import pytest

import oracle as O
from vgcut import engine, scenes
from vgcut.camera import Camera


@pytest.fixture(scope="module")
def small():
    spec = scenes.plain_small(n=40, seed=1)
    scene, _, _ = O.scene_from_spec(spec.meshes, spec.instances)
    return spec, scene


def drawn_triangles(scene, cam, p, precision):
    r = O.cull_pass(scene, O.make_view(cam, p), precision)
    return r["counters"][2 + 4] // 3, r


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_budget_prediction_is_exact_without_blend(small, precision):
    spec, scene = small
    cams = [spec.cameras[0], Camera.perspective_look_at((14, 6, -9), (0, 0, 0), 60, 1920, 1080, 0.1, 1000)]
    for cam in cams:
        full, _ = drawn_triangles(scene, cam, engine.ViewParams(error_threshold=0.5, lod_blend=1.0), precision)
        for frac in (0.2, 0.5, 0.9):
            budget = full * frac
            p = engine.ViewParams(lod_blend=1.0, triangle_budget=budget, threshold_range=(0.5, 3.0))
            got, r = drawn_triangles(scene, cam, p, precision)
            t = r["threshold"]
            assert 0.5 <= t <= 3.0
            assert got == r["predicted"], "histogram prediction equals the cut at the chosen threshold"
            if t < 3.0:
                assert got <= budget
            if t > 0.5:  # one bin finer would not fit
                finer = 0.5 + (3.0 - 0.5) * (round((t - 0.5) / 2.5 * 255) - 1) / 255
                over, _ = drawn_triangles(scene, cam, engine.ViewParams(error_threshold=finer, lod_blend=1.0), precision)
                assert over > budget


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_budget_bounds_the_blended_cut(small, precision):
    spec, scene = small
    cams = [spec.cameras[0], Camera.perspective_look_at((14, 6, -9), (0, 0, 0), 60, 1920, 1080, 0.1, 1000)]
    thresholds = []
    for cam in cams:
        full, _ = drawn_triangles(scene, cam, engine.ViewParams(error_threshold=0.5, lod_blend=1.0), precision)
        for frac in (0.1, 0.3, 0.6):
            budget = full * frac
            p = engine.ViewParams(lod_blend=2.0, triangle_budget=budget, threshold_range=(0.5, 8.0))
            got, r = drawn_triangles(scene, cam, p, precision)
            assert r["threshold"] < 8.0, "the range reaches the budget"
            assert got <= r["predicted"] <= budget, f"drawn {got} predicted {r['predicted']} budget {budget}"
            assert got >= 0.95 * r["predicted"], f"drawn {got} far below the prediction {r['predicted']}"
            thresholds.append(r["threshold"])
    assert max(thresholds) > 2.5, "cases run with the blend band fully open"
