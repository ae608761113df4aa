"""The raster passes when their tile queue is full: 80 screen-filling quads at 2048x2048 queue about 1.3M tiles of
32x16 pixels, more than the queue's 1,048,576, so the last large triangles take the fallback path (the warp that set
them up draws them itself). The occluder depth image and the visibility buffer must still equal the oracle's bit for
bit."""
from types import SimpleNamespace

import numpy as np
import pytest

import oracle as O
from parity_util import Harness, d2h
from vgcut import build as B
from vgcut import engine
from vgcut.camera import Camera

pytestmark = pytest.mark.gpu

N, S = 2048, 80


@pytest.fixture(scope="module")
def wall():
    pos = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], np.float32)
    quad = B.build_virtual_mesh(pos, np.array([0, 1, 2, 0, 2, 3], np.uint32))
    mats = np.zeros((S, 16), np.float32)
    for k in range(S):  # 400 x 400 quads facing the camera, 5 to 5.79 units in front of it
        mats[k] = [200, 0, 0, 0, 0, 200, 0, 0, 0, 0, 1, 0, 0, 0, -5.0 - 0.01 * k, 1]
    spec = SimpleNamespace(meshes=[quad], instances=[mats])
    h = Harness(spec, [dict(occluder=True, vertex_data=True)], max_meshlets=4096, max_triangles=100_000)
    cam = Camera.perspective_look_at((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), 60, N, N, 0.1, 5000.0)
    h.gpu(cam, engine.ViewParams(), slot=0)
    assert len(h.vg.draw_list(0, 0)) == S
    return h, cam


def test_occluder_depth_with_a_full_tile_queue(wall):
    import torch
    h, cam = wall
    d = torch.empty((N, N), dtype=torch.float32, device="cuda")
    h.vg.occluder_depth(0, cam, d.data_ptr(), N, N)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    want = O.occluder_depth(h.spec.meshes, [True], h.mats, h.inst_slot, h.vg.draw_list(0, 0), cam, N, N)
    assert (got < 1).all(), "the nearest quad covers the image"
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"{int((got != want).sum())} pixels differ"


def test_visibility_with_a_full_tile_queue(wall):
    import torch
    h, cam = wall
    cap = 300_000
    idx = torch.zeros(cap, dtype=torch.int32, device="cuda")
    h.vg.expand(0, 0, idx.data_ptr(), cap)
    vis = torch.zeros((N, N), dtype=torch.int64, device="cuda")
    h.vg.visibility(0, 0, cam, idx.data_ptr(), cap, vis.data_ptr(), N, N)
    torch.cuda.synchronize()
    out = h.vg.output(0)
    draw_list = d2h(out.draw_list[0], 2 * out.max_drawn * 4).reshape(-1, 4)
    args = d2h(out.draw_args, out.mesh_slots * 2 * 5).reshape(-1, 5)
    want = O.visibility(h.spec.meshes, [True], [float("inf")], h.mats, h.inst_slot,
                        idx.cpu().numpy().view(np.uint32), draw_list, args, cam, N, N)
    got = vis.cpu().numpy().view(np.uint64)
    assert (got != np.uint64(engine.VIS_EMPTY)).all()
    assert np.array_equal(got, want), f"{int((got != want).sum())} pixels differ"
