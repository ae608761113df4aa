"""The visibility buffer (vgc_visibility), the headless consumer that closes the loop after the cut and vgc_expand:
the expanded index buffer drawn with the reference's vertex pulling (GeometryPool.ts:1095-1131, draw-distance
shrink included) and LOD blend mask (lodBlend.ts:36-45) must equal the oracle's image bit for bit, for both cuts, a
blended threshold and an animated blend pattern; every covered pixel names a triangle of the cut."""
import numpy as np
import pytest

import oracle as O
from parity_util import Harness, d2h, small_ruins
from vgcut import engine

pytestmark = pytest.mark.gpu

W, H = 480, 270


@pytest.fixture(scope="module")
def scene():
    spec = small_ruins(seed=5, poses=3, quads=0)
    # every mesh casts a shadow; the two smallest fade out at 60 world units
    order = np.argsort([len(d.meshlet_info) for d in spec.meshes])
    flags = [dict(shadow=True, vertex_data=True) for _ in spec.meshes]
    flags[order[-1]]["vertex_data"] = False  # the largest mesh has no vertex data: not drawn
    for k in order[:2]:
        flags[k]["max_draw_distance"] = 60.0
    return Harness(spec, flags)


def run(h, cam, cut, frame=0, threshold=2.0):
    import torch
    h.gpu(cam, engine.ViewParams(error_threshold=threshold, shadow_sweep=(30.0, -60.0, 10.0)), slot=0)
    cap = h.caps[cut]
    idx = torch.zeros(cap, dtype=torch.int32, device="cuda")
    h.vg.expand(0, cut, idx.data_ptr(), cap)
    vis = torch.zeros((H, W), dtype=torch.int64, device="cuda")
    h.vg.visibility(0, cut, cam, idx.data_ptr(), cap, vis.data_ptr(), W, H, frame=frame)
    torch.cuda.synchronize()
    out = h.vg.output(0)
    draw_list = d2h(out.draw_list[0], 2 * out.max_drawn * 4).reshape(-1, 4)
    regions = out.mesh_slots * 2
    args = d2h(out.draw_args + cut * regions * 5 * 4, regions * 5).reshape(-1, 5)
    maxd = [f.get("max_draw_distance", float("inf")) for f in h.flags]
    want = O.visibility(h.spec.meshes, [f["vertex_data"] for f in h.flags], maxd, h.mats, h.inst_slot, idx.cpu().numpy().view(np.uint32), draw_list, args,
                        cam, W, H, frame=frame)
    return vis.cpu().numpy().view(np.uint64), want, draw_list, args


@pytest.mark.parametrize("cut,frame", [(0, 0), (0, 3), (1, 0)])
def test_visibility_matches_the_oracle(scene, cut, frame):
    cam = scene.spec.cameras[1]
    got, want, draw_list, args = run(scene, cam, cut, frame)
    covered = got != engine.VIS_EMPTY
    assert covered.mean() > 0.05, "the cut covers part of the image"
    assert np.array_equal(got, want), f"{int((got != want).sum())} pixels differ"
    # every covered pixel names a drawn entry of this cut and a triangle inside its meshlet
    ids = (got[covered] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    ds, tri = ids >> 7, ids & 127
    max_drawn = len(draw_list) // 2
    assert ((ds >= cut * max_drawn) & (ds < (cut + 1) * max_drawn)).all()
    assert (tri < (draw_list[ds, 3] & 255)).all()
    if cut == 0:
        blended = (draw_list[np.unique(ds), 3] & 0xFFFF00) != (255 << 16)
        assert blended.any(), "blended (part 1) meshlets reach the image through the blend mask"


def test_blend_pattern_moves_with_the_frame(scene):
    cam = scene.spec.cameras[1]
    a, _, _, _ = run(scene, cam, 0, 0)
    b, _, _, _ = run(scene, cam, 0, 1)
    assert (a != b).any(), "lodBlendFrame shifts the blend pattern"


def test_near_plane_clipping_matches_the_oracle(scene):
    """The visibility pass with the near plane 8 m out: triangles crossing it are clipped into one or two triangles
    (the second drawn in the same warp step), carrying the crossing triangle's id, bit for bit as the oracle."""
    from vgcut.camera import Camera
    base = scene.spec.cameras[1]
    fwd = -np.asarray(base.view).reshape(4, 4).T[2, :3]
    eye = base.extra["eye"]
    cam = Camera.perspective_look_at(tuple(eye), tuple(eye + fwd), 60, 960, 540, 8.0, 5000.0)
    got, want, _, _ = run(scene, cam, 0)
    assert np.array_equal(got, want), f"{int((got != want).sum())} pixels differ"
    depth = (got >> np.uint64(32)).astype(np.uint32).view(np.float32)
    assert (depth < 0.02).sum() > 20, "clipped triangles reach the near plane (within ~0.2 m of it)"
