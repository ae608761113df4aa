"""Batching many uneven views in one launch: cameras at 720p / 1080p / 4K with thresholds 0.5 / 1 / 2 px (2 px opens
the LOD-blend band), each with four orthographic shadow cascades (VGC_VIEW_CASCADE), all in one CUDA-graph launch,
before and after the autotuner picks the launch's grid sizes. Every view must equal the oracle's float mirror, and
the batched results must equal each view cut alone."""
import numpy as np
import pytest

from parity_util import Harness, key_set, small_ruins
from vgcut import engine
from vgcut.camera import Camera, cascade_clips

pytestmark = pytest.mark.gpu

LIGHT = (0.35, -1.0, 0.25)
SPLITS = [0.1, 8.0, 30.0, 90.0, 250.0]


@pytest.fixture(scope="module")
def ruins():
    spec = small_ruins(seed=5, poses=3)
    flags = [dict(shadow=(i % 3 != 2), occlusion=False) for i in range(len(spec.meshes))]
    h = Harness(spec, flags, max_meshlets=1 << 16)
    return h


def view_set(h):
    rng = np.random.default_rng(3)
    out = []
    sizes = [(1280, 720), (1920, 1080), (3840, 2160)]
    for i, base in enumerate(h.spec.cameras):
        eye = base.extra["eye"]
        w, hh = sizes[i % 3]
        t = [0.5, 1.0, 2.0][(i + 1) % 3]
        yaw = rng.uniform(0, 2 * np.pi)
        cam = Camera.perspective_look_at(tuple(eye), (eye[0] + np.cos(yaw), eye[1], eye[2] + np.sin(yaw)), 60, w, hh,
                                         0.1, 2000)
        out.append((cam, engine.ViewParams(error_threshold=t, shadow_sweep=(20.0, -40.0, 10.0))))
        for clip in cascade_clips(cam, LIGHT, SPLITS):
            out.append((cam, engine.ViewParams(error_threshold=t, cascade_clip=clip)))
    return out


def test_cascades_match_the_oracle(ruins):
    h = ruins
    casters = 0
    for k, (cam, p) in enumerate(view_set(h)):
        lists, res = h.compare(cam, p)
        if p.cascade_clip is not None:
            assert len(lists[0]) == 0, "a cascade has no camera cut"
            casters += len(lists[1])
    assert casters > 0


def test_uneven_batch_equals_alone_and_autotune_keeps_results(ruins):
    h = ruins
    vs = view_set(h)
    n = len(vs)
    fresh = np.array([10000, 10000, 0, 0, 0, 0, 0, 0], np.uint32)
    views = []
    for k, (cam, p) in enumerate(vs):
        p = engine.ViewParams(**{**p.__dict__, "state_slot": k, "fresh_state": True})
        views.append(engine.make_view(cam, p))
    # alone, one plain launch per view
    alone = []
    for k, v in enumerate(views):
        h.vg.cut([v], first_slot=k)
        alone.append([key_set(h.vg.draw_list(k, c), (0, 1, 3)) for c in (0, 1)] + [h.vg.read_stats(k)["selected"]])
    for tuned in (False, True):
        if tuned:
            best = h.vg.autotune(views, reps=2)
            assert best["instances_blocks_per_sm"] >= 1 and best["chunks_blocks_per_sm"] >= 1 and best["ms"] > 0
        h.vg.cut(views, first_slot=0, graph=True)
        for k in range(n):
            got = [key_set(h.vg.draw_list(k, c), (0, 1, 3)) for c in (0, 1)] + [h.vg.read_stats(k)["selected"]]
            assert got[2] == alone[k][2], f"view {k}: selected counts differ in the batch (tuned={tuned})"
            for c in (0, 1):  # a draw list that overflowed keeps an atomic-order-dependent subset
                if got[2][c] <= h.max_meshlets:
                    assert got[c] == alone[k][c], f"view {k} cut {c} differs in the batch (tuned={tuned})"


@pytest.mark.parametrize("chunk", [256, 512, 1024])
def test_every_chunk_size_gives_the_same_cuts(ruins, chunk):
    """The autotuner's candidates only cut the meshlet work into different windows (chunks of 256, 512 or 1024
    meshlets) and spread it over different grids: each must give every view's cut exactly."""
    h = ruins
    vs = view_set(h)
    views = [engine.make_view(cam, engine.ViewParams(**{**p.__dict__, "state_slot": k, "fresh_state": True}))
             for k, (cam, p) in enumerate(vs)]
    h.vg.set_tuning(len(views), 0, 0, 512)
    h.vg.cut(views, first_slot=0, graph=True)
    want = [([key_set(h.vg.draw_list(k, c), (0, 1, 3)) for c in (0, 1)], h.vg.read_stats(k)) for k in range(len(vs))]
    h.vg.set_tuning(len(views), 1, 2, chunk)
    h.vg.cut(views, first_slot=0, graph=True)
    for k in range(len(vs)):
        s = h.vg.read_stats(k)
        assert s["selected"] == want[k][1]["selected"] and s["work"] == want[k][1]["work"]
        assert s["requested_indices"] == want[k][1]["requested_indices"]
        for c in (0, 1):
            if s["selected"][c] <= h.max_meshlets:
                assert key_set(h.vg.draw_list(k, c), (0, 1, 3)) == want[k][0][c], f"view {k} cut {c}, chunk {chunk}"
    with pytest.raises(engine.VgcError, match="chunk_meshlets"):
        h.vg.set_tuning(len(views), 0, 0, 300)
