"""The occluder depth pass (vgc_occluder_depth) and the two-pass occlusion loop it closes: the previous frame's
camera cut of the occluder meshes, drawn depth-only with this frame's camera, must equal the oracle's rasterizer bit
for bit; an HZB built from it then culls this frame's cut exactly as the oracle does with the same HZB."""
import numpy as np
import pytest

import oracle as O
from parity_util import Harness, d2h, key_set, small_ruins
from vgcut import engine
from vgcut.camera import Camera

pytestmark = pytest.mark.gpu

W, H = 480, 270


@pytest.fixture(scope="module")
def occluding():
    spec = small_ruins(seed=9, poses=3, quads=0)
    flags = [dict(occlusion=True, occluder=True) for _ in spec.meshes]
    h = Harness(spec, flags)
    return h


def moved(cam, dx, dyaw):
    eye = cam.extra["eye"]
    inv = np.asarray(cam.view).reshape(4, 4).T
    fwd = -inv[2, :3]  # camera -z in world
    c, s = np.cos(dyaw), np.sin(dyaw)
    f = np.array([c * fwd[0] - s * fwd[2], fwd[1], s * fwd[0] + c * fwd[2]])
    e = eye + dx * fwd
    return Camera.perspective_look_at(tuple(e), tuple(e + f), 60, 960, 540, 0.1, 5000.0)


def gpu_depth(h, src_slot, cam):
    import torch
    d = torch.empty((H, W), dtype=torch.float32, device="cuda")
    h.vg.occluder_depth(src_slot, cam, d.data_ptr(), W, H)
    torch.cuda.synchronize()
    return d


def oracle_depth(h, src_slot, cam):
    entries = h.vg.draw_list(src_slot, 0)
    return O.occluder_depth(h.spec.meshes, [True] * len(h.spec.meshes), h.mats, h.inst_slot, entries, cam, W, H)


def test_occluder_depth_matches_the_oracle(occluding):
    h = occluding
    for k, cam in enumerate(h.spec.cameras):
        h.gpu(cam, engine.ViewParams(error_threshold=1.0), slot=0)  # the "previous frame"
        now = moved(cam, 1.5, 0.03 * (k + 1))
        d = gpu_depth(h, 0, now)
        got = d.cpu().numpy()
        want = oracle_depth(h, 0, now)
        assert (got < 1).mean() > 0.05, "the occluders cover part of the image"
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), \
            f"pose {k}: {int((got != want).sum())} pixels differ"


def test_two_pass_occlusion_matches_the_oracle(occluding):
    h = occluding
    culled = 0
    for k, cam in enumerate(h.spec.cameras):
        h.gpu(cam, engine.ViewParams(error_threshold=1.0), slot=0)
        now = moved(cam, 1.0, -0.02 * (k + 1))
        d = gpu_depth(h, 0, now)
        engine.check(engine.lib().vgc_hzb_build(h.vg.handle, 30, d.data_ptr(), W, H, 1, None))
        hzb = O.hzb_build(oracle_depth(h, 0, now))
        p = engine.ViewParams(error_threshold=1.0, hzb=30)
        lists, res = h.compare(now, p, hzb_oracle=hzb, slot=1)
        open_res, _ = h.oracle(now, engine.ViewParams(error_threshold=1.0))
        culled += len(open_res["entries"][0]) - len(lists[0])
    assert culled > 0, "the previous frame's occluders hide part of this frame's cut"


def large_triangles(h, entries, cam, width, height, min_pixels=1024):
    """Front-facing part-0 triangles of `entries` in front of the camera whose pixel bounding box at width x height
    exceeds `min_pixels` (float64 estimate): those the rasterizer hands to its grid-wide tile pass."""
    e = entries[(entries[:, 3] & 0xFFFF00) == (255 << 16)]
    vp = np.asarray(cam.proj, np.float64).reshape(4, 4).T @ np.asarray(cam.view, np.float64).reshape(4, 4).T
    bases = np.cumsum([0] + [len(d.meshlet_info) // 4 for d in h.spec.meshes])
    found = 0
    for inst, mid, _, w in e:
        k = int(np.searchsorted(bases, mid, side="right")) - 1
        d = h.spec.meshes[k]
        info = np.asarray(d.meshlet_info, np.uint32).reshape(-1, 4)[mid - bases[k]]
        packed = np.asarray(d.meshlet_triangles, np.uint32)[info[1] // 3: info[1] // 3 + (w & 255)]
        local = np.stack([packed & 255, (packed >> 8) & 255, (packed >> 16) & 255], 1)
        ids = np.asarray(d.meshlet_vertices, np.uint32)[info[3] + local]
        p = np.asarray(d.positions, np.float64).reshape(-1, 3)[ids]
        m = np.asarray(h.mats[inst], np.float64).reshape(4, 4).T
        clip = np.einsum("ij,tvj->tvi", vp @ m, np.concatenate([p, np.ones(p.shape[:2] + (1,))], 2))
        ok = (clip[..., 3] > 0).all(1) & (clip[..., 2] >= 0).all(1)
        sx = (clip[..., 0] / clip[..., 3] * 0.5 + 0.5) * width
        sy = (0.5 - clip[..., 1] / clip[..., 3] * 0.5) * height
        area = (sx[:, 1] - sx[:, 0]) * (sy[:, 2] - sy[:, 0]) - (sx[:, 2] - sx[:, 0]) * (sy[:, 1] - sy[:, 0])
        bw = np.clip(sx.max(1), 0, width) - np.clip(sx.min(1), 0, width)
        bh = np.clip(sy.max(1), 0, height) - np.clip(sy.min(1), 0, height)
        found += int((ok & (area < 0) & (bw * bh > min_pixels)).sum())
    return found


def test_large_triangles_match_the_oracle(occluding):
    """A coarse cut drawn at 1920x1080: many triangles cover thousands of pixels, and those go through the tile pass;
    the image is still the oracle's bit for bit."""
    import torch
    h = occluding
    w2, h2 = 1920, 1080
    cam = h.spec.cameras[1]
    h.gpu(cam, engine.ViewParams(error_threshold=24.0), slot=0)
    now = moved(cam, 0.5, 0.02)
    entries = h.vg.draw_list(0, 0)
    assert large_triangles(h, entries, now, w2, h2) > 50, "the case reaches the tile pass"
    d = torch.empty((h2, w2), dtype=torch.float32, device="cuda")
    h.vg.occluder_depth(0, now, d.data_ptr(), w2, h2)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    want = O.occluder_depth(h.spec.meshes, [True] * len(h.spec.meshes), h.mats, h.inst_slot, entries, now, w2, h2)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"{int((got != want).sum())} pixels differ"


def test_near_plane_clipping_matches_the_oracle(occluding):
    """With the near plane 8 m out, many occluder triangles cross it: each is clipped in clip space into one or two
    triangles (queued and clipped by their own kernel), and the image equals the oracle's bit for bit; the clipped
    parts reach depth 0 at the near plane."""
    h = occluding
    cam = h.spec.cameras[0]
    h.gpu(cam, engine.ViewParams(error_threshold=1.0), slot=0)
    fwd = -np.asarray(cam.view).reshape(4, 4).T[2, :3]
    eye = cam.extra["eye"]
    near = Camera.perspective_look_at(tuple(eye), tuple(eye + fwd), 60, 960, 540, 8.0, 5000.0)
    got = gpu_depth(h, 0, near).cpu().numpy()
    want = oracle_depth(h, 0, near)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"{int((got != want).sum())} pixels differ"
    assert (got < 1e-3).sum() > 20, "clipped triangles reach the near plane"


def test_batch_call_equals_single_calls(occluding):
    """vgc_occluder_depth_batch draws the same images as one vgc_occluder_depth call per image."""
    import torch
    h = occluding
    cams = [moved(c, 1.2, 0.02 * (k + 1)) for k, c in enumerate(h.spec.cameras)]
    for k, cam in enumerate(h.spec.cameras):
        h.gpu(cam, engine.ViewParams(error_threshold=1.0), slot=k)
    single = [gpu_depth(h, k, cams[k]) for k in range(len(cams))]
    batch = [torch.empty((H, W), dtype=torch.float32, device="cuda") for _ in cams]
    h.vg.occluder_depth_batch(list(range(len(cams))), cams, [d.data_ptr() for d in batch], W, H)
    torch.cuda.synchronize()
    for k, (a, b) in enumerate(zip(single, batch)):
        assert (a < 1).float().mean() > 0.05
        assert torch.equal(a.view(torch.int32), b.view(torch.int32)), f"image {k} differs"
