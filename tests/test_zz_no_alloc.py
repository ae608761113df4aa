"""vgc_cut_noalloc, the single-view cut that allocates no device memory on the call, against vgc_cut.

Callers that cannot allocate while they run, such as a renderer's real-time frame thread that must not stall on
cudaMalloc or a host that reserves all of its GPU memory up front, use this entry point; its scratch is a fixed device array inside the library. The results must be the
ones vgc_cut produces for the same view, call after call (the array keeps the previous call's contents, so a
second call checks that everything that must start at zero is cleared). This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from vgcut import engine, scenes
from vgcut.camera import Camera

pytestmark = pytest.mark.gpu


def entries(vg, slot, cut):
    e = vg.draw_list(slot, cut)
    return set(map(tuple, e[:, [0, 1, 3]].tolist()))


def counters(vg, slot):
    s = vg.read_stats(slot)
    return [s["visible_cells"], s["occluded_instances"], s["selected"], s["drawn"], s["survived"], s["work"],
            s["requested_indices"], s["rounds"]]


@pytest.fixture(scope="module")
def scene():
    spec = scenes.plain_small(n=40, seed=4)
    vg = engine.VirtualGeometry(max_meshlets=1 << 16, output_slots=4)
    scenes.load_into(vg, spec, cast_shadow=True)
    # one allocating call publishes the scene and sizes every buffer the no-alloc call will use
    vg.update(spec.cameras[0], slot=0)
    vg.read_stats(0)
    yield spec, vg
    vg.dispose()


def test_noalloc_matches_vgc_cut_twice(scene):
    spec, vg = scene
    cams = [spec.cameras[0], Camera.perspective_look_at((9.0, 4.0, -7.0), (0.0, 0.0, 1.0), 60, 1920, 1080, 0.1, 1000)]
    fresh = np.array([10000, 10000, 0, 0, 0, 0, 0, 0], np.uint32)
    for call, (cam, t) in enumerate(zip(cams, [1.0, 2.5])):
        vg.state(0, fresh)  # both calls start from the same capacity-controller state
        vg.state(1, fresh)
        params = engine.ViewParams(error_threshold=t, shadow_sweep=(5.0, -20.0, 3.0))
        vg.cut([engine.make_view(cam, params)], first_slot=0)
        want_counters = counters(vg, 0)
        want = [entries(vg, 0, c) for c in (0, 1)]
        params.state_slot = 1
        vg.cut_noalloc(engine.make_view(cam, params), slot=1)
        assert counters(vg, 1) == want_counters, f"call {call}: counters differ from vgc_cut"
        for c in (0, 1):
            assert entries(vg, 1, c) == want[c], f"call {call}: cut {c} differs from vgc_cut"
        assert len(want[0]) > 0 and len(want[1]) > 0


def test_noalloc_rejects_what_it_cannot_hold(scene):
    spec, vg = scene
    view = engine.make_view(spec.cameras[0])
    with pytest.raises(engine.VgcError, match="not allocated"):
        vg.cut_noalloc(view, slot=99)  # output slot beyond the context's output_slots
    view.state_slot = 100000
    with pytest.raises(engine.VgcError, match="state slot"):
        vg.cut_noalloc(view, slot=1)
