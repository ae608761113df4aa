"""Edge cases of the cut against the oracle: an empty context, a mesh with no instances beside one with a single
instance, a camera that sees nothing, a removed mesh (its cells stay, pointing at a disabled slot,
GeometryPool.ts:358-363), a small mesh with 200,000 instances, and the raster consumers of an empty cut."""
from types import SimpleNamespace

import numpy as np
import pytest

from parity_util import Harness, grid_matrices
from vgcut import engine, scenes
from vgcut.camera import Camera

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def meshes():
    return [scenes.icosphere_mesh(10, seed=1), scenes.icosphere_mesh(24, seed=2), scenes.icosphere_mesh(6, seed=3)]


def camera_at(eye, target):
    return Camera.perspective_look_at(eye, target, 60, 960, 540, 0.1, 5000.0)


def test_empty_context():
    import torch
    vg = engine.VirtualGeometry(max_triangles=100_000, max_shadow_triangles=100_000, max_meshlets=4096)
    cam = camera_at((0.0, 2.0, 10.0), (0.0, 0.0, 0.0))
    vg.cut([engine.make_view(cam, engine.ViewParams(shadow_sweep=(1.0, -2.0, 0.5)))])
    st = vg.read_stats(0)
    assert st["visible_cells"] == 0 and st["selected"] == [0, 0] and st["requested_indices"] == [0, 0]
    assert len(vg.draw_list(0, 0)) == 0 and len(vg.draw_list(0, 1)) == 0
    depth = torch.zeros((54, 96), dtype=torch.float32, device="cuda")
    vg.occluder_depth(0, cam, depth.data_ptr(), 96, 54)
    idx = torch.zeros(300, dtype=torch.int32, device="cuda")
    vg.expand(0, 0, idx.data_ptr(), 300)
    vis = torch.zeros((54, 96), dtype=torch.int64, device="cuda")
    vg.visibility(0, 0, cam, idx.data_ptr(), 300, vis.data_ptr(), 96, 54)
    torch.cuda.synchronize()
    assert (depth == 1.0).all()
    assert (vis.cpu().numpy().view(np.uint64) == np.uint64(engine.VIS_EMPTY)).all()
    vg.dispose()


def test_zero_and_single_instance_meshes(meshes):
    spec = SimpleNamespace(meshes=meshes, instances=[np.zeros((0, 16), np.float32), grid_matrices(1, 4.0, 1),
                                                     grid_matrices(300, 4.0, 2)])
    h = Harness(spec, [dict(shadow=True) for _ in meshes])
    h.check_layout()
    for eye in [(-3.0, 2.0, -3.0), (30.0, 8.0, 30.0), (0.2, 0.5, 1.5)]:
        cam = camera_at(eye, (20.0, 0.0, 20.0))
        for t in (0.5, 1.0, 2.0):
            lists, res = h.compare(cam, engine.ViewParams(error_threshold=t, shadow_sweep=(5.0, -10.0, 2.0)))
    assert len(lists[0]) > 0


def test_camera_that_sees_nothing(meshes):
    spec = SimpleNamespace(meshes=meshes, instances=[grid_matrices(64, 4.0, s) for s in (3, 4, 5)])
    h = Harness(spec)
    cam = camera_at((0.0, 50.0, -500.0), (0.0, 60.0, -1000.0))  # looking away from the grid
    lists, res = h.compare(cam, engine.ViewParams())
    assert len(lists[0]) == 0 and res["counters"][0] == 0


def test_removed_mesh(meshes):
    spec = SimpleNamespace(meshes=meshes, instances=[grid_matrices(200, 4.0, s) for s in (6, 7, 8)])
    flags = [dict(shadow=True) for _ in meshes]
    h = Harness(spec, flags)
    cam = camera_at((-5.0, 6.0, -5.0), (25.0, 0.0, 25.0))
    before, _ = h.compare(cam, engine.ViewParams(shadow_sweep=(5.0, -10.0, 2.0)))
    h.vg.meshes[1].dispose()
    flags[1]["enabled"] = False  # the oracle scene keeps the mesh's cells, with the slot disabled
    from oracle import scene_from_spec
    h.scene, h.mats, h.orders = scene_from_spec(spec.meshes, spec.instances, flags)
    after, _ = h.compare(cam, engine.ViewParams(shadow_sweep=(5.0, -10.0, 2.0)))
    removed = set(np.nonzero(h.inst_slot == 1)[0].tolist())
    assert any(int(i) in removed for i in before[0][:, 0]), "the removed mesh was drawn before"
    assert not any(int(i) in removed for cut in (0, 1) for i in after[cut][:, 0])


def test_many_instances_of_a_small_mesh(meshes):
    n = 200_000
    spec = SimpleNamespace(meshes=[meshes[2]], instances=[grid_matrices(n, 3.0, 9)])
    h = Harness(spec, max_meshlets=1 << 18, max_triangles=8_000_000)
    h.check_layout()
    cam = camera_at((-10.0, 15.0, -10.0), (600.0, 0.0, 600.0))
    lists, res = h.compare(cam, engine.ViewParams(error_threshold=1.0))
    assert res["counters"][0] > 100, "many cells are visible"
