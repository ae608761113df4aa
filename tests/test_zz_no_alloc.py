"""vgc_cut_noalloc, the single-view cut that allocates no device memory on the call, against vgc_cut.

Callers that cannot allocate while they run, such as a renderer's real-time frame thread that must not stall on
cudaMalloc or a host that reserves all of its GPU memory up front, use this entry point; its scratch is a fixed device
array inside the library. The results must be the ones vgc_cut produces for the same view, call after call (the array
keeps the previous call's contents, so a second call checks that everything that must start at zero is cleared), also
when the view's work overflows the fixed meshlet queue (items tested in place) and with a triangle budget, and the
calls must leave the device's free memory unchanged. This file is collected last on purpose.
"""
import ctypes
import dataclasses
from types import SimpleNamespace

import numpy as np
import pytest

from parity_util import Harness, grid_matrices, key_set
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


def device_free_bytes() -> int:
    rt = ctypes.CDLL("libcudart.so.12")
    assert rt.cudaDeviceSynchronize() == 0
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def test_noalloc_allocates_nothing(scene):
    spec, vg = scene
    view = engine.make_view(spec.cameras[0], engine.ViewParams(error_threshold=1.5, state_slot=1))
    vg.cut_noalloc(view, slot=1)  # the first call on a device looks the array's address up
    free, footprint = device_free_bytes(), vg.footprint()
    for _ in range(3):
        vg.cut_noalloc(view, slot=1)
    assert device_free_bytes() == free, "a no-alloc call changed the device's free memory"
    assert vg.footprint() == footprint, "a no-alloc call grew the context"
    assert vg.read_stats(1)["selected"][0] > 0


CROWD = 100_000          # instances of one small mesh on a grid 1.5 m apart
FIXED_QUEUE_SPANS = 49_152  # span entries of the no-alloc call's fixed meshlet queue (3/4 of 65,536)


@pytest.fixture(scope="module")
def crowd():
    """A crowd whose view queues more spans than the fixed queue holds: at 2.5 px the blend band is fully open, so
    almost no instance takes the fast path and nearly every visible one becomes a work item."""
    spec = SimpleNamespace(meshes=[scenes.icosphere_mesh(24, seed=2)], instances=[grid_matrices(CROWD, 1.5, 11)])
    h = Harness(spec, [dict(shadow=True)], max_meshlets=1 << 18, max_triangles=12_000_000, max_shadow=4_000_000)
    yield h
    h.vg.dispose()


@pytest.mark.parametrize("budget", [0.0, 2_000_000.0])
def test_noalloc_queue_overflow_matches_vgc_cut_and_oracle(crowd, budget):
    h = crowd
    side = float(np.ceil(np.sqrt(CROWD))) * 1.5
    cam = Camera.perspective_look_at((-5.0, 12.0, -5.0), (side / 2, 0.0, side / 2), 60, 1920, 1080, 0.1, 5000.0)
    p = engine.ViewParams(error_threshold=2.5, shadow_sweep=(5.0, -20.0, 3.0), triangle_budget=budget,
                          threshold_range=(0.5, 4.0))
    fresh = np.array([10000, 10000, 0, 0, 0, 0, 0, 0], np.uint32)
    for _ in range(2):  # vgc_cut grows its own queue after its first call; the no-alloc queue stays fixed
        h.vg.state(0, fresh)
        lists, res = h.compare(cam, p)  # vgc_cut == the oracle's float mirror
    want = h.vg.read_stats(0)
    assert want["work"][0] + want["work"][1] > FIXED_QUEUE_SPANS, "the view must overflow the fixed queue"
    for call in range(2):
        h.vg.state(1, fresh)
        h.vg.cut_noalloc(engine.make_view(cam, dataclasses.replace(p, state_slot=1)), slot=1)
        got = h.vg.read_stats(1)
        assert counters(h.vg, 1) == counters(h.vg, 0), f"call {call}: counters differ from vgc_cut"
        assert got["effective_threshold"] == want["effective_threshold"]
        assert got["predicted_triangles"] == want["predicted_triangles"]
        for c in (0, 1):
            g = entries(h.vg, 1, c)
            assert g == entries(h.vg, 0, c), f"call {call}: cut {c} differs from vgc_cut"
            assert g == key_set(res["entries"][c], (0, 1, 2)), f"call {call}: cut {c} differs from the oracle"
