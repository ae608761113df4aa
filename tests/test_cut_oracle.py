"""The reference's LOD-cut tests (tests/cut.test.ts:5-117) ported to the oracle, on the same terrain recipe.

The terrain is built by this repository's builder (the reference's needs meshoptimizer), so the numbers differ
from the reference's run while the asserted invariants are the same."""
import numpy as np

import oracle as O
from vgcut.camera import Camera


def test_cut_covers_every_leaf_once(terrain, park_miller):
    d = terrain
    assert len(d.replacement_group) == d.meshlet_count
    rand = park_miller(7)
    views = []
    for _ in range(12):
        eye = ((rand() - 0.5) * 300, 2 + rand() * 80, (rand() - 0.5) * 300)
        target = ((rand() - 0.5) * 200, 0, (rand() - 0.5) * 200)
        views.append(Camera.perspective_look_at(eye, target, 60, 16, 9, 0.1, 5000))
    worst = 0
    for cam in views:
        ps = cam.proj[5] * 1080 * 0.5
        for t in (0.5, 1, 3):
            sel = O.select_cut(d, cam.view, ps, 0.1, t)
            holes = O.verify_cut_coverage(d, sel)
            worst = max(worst, len(holes))
            assert len(holes) == 0
            assert len(O.verify_cut_overlap(d, sel)) == 0
            start, end = O.instance_meshlet_range(d, cam.view, ps, 0.1, t)
            idx = np.nonzero(sel)[0]
            assert np.all((idx >= start) & (idx < end)), "level range contains every selected meshlet"
    # far away the range shrinks to a few coarse levels (cut.test.ts:55-64)
    cam = Camera.perspective_look_at((0, 2000, 8000), (0, 0, 0), 60, 16, 9, 0.1, 50000)
    start, end = O.instance_meshlet_range(d, cam.view, cam.proj[5] * 540, 0.1, 1)
    assert end - start < d.meshlet_count / 4


def test_blend_band_steps_are_complete_cuts(terrain):
    d = terrain
    blended = 0
    for eye in [(0, 40, 260), (150, 6, -40), (-300, 200, 300)]:
        cam = Camera.perspective_look_at(eye, (0, 0, 0), 60, 16, 9, 0.1, 5000)
        ps = cam.proj[5] * 540
        for t, blend in [(1, 2), (0.7, 1.5), (2, 3)]:
            lo, hi = O.select_blend_cut(d, cam.view, ps, 0.1, t, blend)
            for tt in (t, t * blend * 0.999):
                plain = O.select_cut(d, cam.view, ps, 0.1, tt)
                assert np.all(~plain.astype(bool) | (hi > 0)), "plain cuts at the band ends are inside the band"
            for step in range(255):
                sel = ((lo <= step) & (step < hi)).astype(np.uint8)
                assert len(O.verify_cut_coverage(d, sel)) == 0, f"no holes at step {step}"
                assert len(O.verify_cut_overlap(d, sel)) == 0, f"no overlaps at step {step}"
            blended += int(((hi > 0) & ((lo > 0) | (hi < 255))).sum())
    assert blended > 0
    cam = Camera.perspective_look_at((0, 40, 260), (0, 0, 0), 60, 16, 9, 0.1, 5000)
    ps = cam.proj[5] * 540
    plain = O.select_cut(d, cam.view, ps, 0.1, 1)
    lo, hi = O.select_blend_cut(d, cam.view, ps, 0.1, 1, 1)
    assert np.array_equal(plain == 1, hi > 0)
    assert np.all((hi == 0) | ((lo == 0) & (hi == 255))), "blend 1 = plain cut"
