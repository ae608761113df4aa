"""The GPU cut on the hand-built golden pass scene (tests/golden/vectors.json "pass_scene"), through the C ABI:
every hand-derived decision (frustum planes of three's WebGPU convention, cell size and draw-distance rejections,
fast path vs work item, the exact projectedError switch, blend steps, HZB occlusion, the swept shadow frustum) must
hold on the device, and the device must equal the oracle's float mirror bit for bit on the same views."""
import json
import os

import numpy as np
import pytest

import oracle as O
from parity_util import Harness, check_golden_view, golden_pass_scene
from vgcut import engine

pytestmark = pytest.mark.gpu

V = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "vectors.json")))


def test_pass_scene_on_the_gpu():
    spec, flags, cam, names = golden_pass_scene(V)
    h = Harness(spec, flags, max_meshlets=1 << 10, max_triangles=100_000, max_shadow=100_000)
    for k, f in enumerate(flags):
        if not f["enabled"]:
            h.vg.meshes[k].visible = False
    h.check_layout()
    depth = np.array(V["pass_scene"]["hzb"], np.float32)
    h.vg.build_hzb(0, depth)
    hzb = O.hzb_build(depth)
    fresh = np.array([10000, 10000, 0, 0, 0, 0, 0, 0], np.uint32)
    try:
        for view in V["pass_scene"]["views"]:
            h.vg.state(0, fresh)
            p = engine.ViewParams(error_threshold=view["t"], lod_blend=view["blend"],
                                  shadow_sweep=tuple(view["sweep"]), hzb=0 if view["hzb"] else -1)
            lists, _ = h.compare(cam, p, hzb_oracle=hzb if view["hzb"] else None)
            s = h.vg.last_stats
            check_golden_view(view, names, [lists[c][:, [0, 1, 3]] for c in (0, 1)],
                              dict(visible_cells=s["visible_cells"], occluded_instances=s["occluded_instances"],
                                   work0=s["work"][0], fast_emitted=s["fast_emitted"]))
    finally:
        h.vg.dispose()
