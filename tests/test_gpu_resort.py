"""Instance re-sort (vgc_instances_resort): after every instance has moved, mortonOrder (GeometryPool.ts:1263-1284)
applied to the current positions on the device gives the oracle's stable order of the current GPU order by Morton
code, the device cells equal the host's and the oracle's computeCell bit for bit, the cells are tighter than before,
and the cut equals the oracle's on the re-sorted scene; a scene not yet resident takes the host path to the same
order."""
import numpy as np
import pytest

import oracle as O
from parity_util import Harness
from test_gpu_edges import camera_at, grid_matrices
from vgcut import engine, scenes

pytestmark = pytest.mark.gpu


def scattered(n, seed):
    rng = np.random.default_rng(seed)
    m = grid_matrices(n, 3.0, seed)
    perm = rng.permutation(n)
    m[:, 12], m[:, 14] = m[perm, 12], m[perm, 14]  # every instance moves to another's place
    return m


@pytest.mark.parametrize("resident", [True, False])
def test_resort_matches_the_oracle(resident):
    from types import SimpleNamespace
    mesh_data = scenes.icosphere_mesh(8, seed=4)
    n = 6000
    start = grid_matrices(n, 3.0, 11)
    spec = SimpleNamespace(meshes=[mesh_data], instances=[start])
    h = Harness(spec, [dict(shadow=True)])
    cam = camera_at((-10.0, 12.0, -10.0), (120.0, 0.0, 120.0))
    params = engine.ViewParams(shadow_sweep=(5.0, -10.0, 2.0))
    mesh = h.vg.meshes[0]
    moved = scattered(n, 12)  # input order
    if resident:
        h.compare(cam, params)
        for i in range(n):
            mesh.set_matrix_at(i, moved[i])
        mesh.commit_instances()
    else:  # nothing uploaded yet: the host path
        h.vg.dispose()
        spec_moved = SimpleNamespace(meshes=[mesh_data], instances=[start])
        h = Harness(spec_moved, [dict(shadow=True)])
        mesh = h.vg.meshes[0]
        for i in range(n):
            mesh.set_matrix_at(i, moved[i])
        mesh.commit_instances()
    before_cells = h.vg.debug_scene()[0]  # host mirror: reading it leaves a pending upload pending
    prev_gpu = moved[mesh.gpu_to_input]  # current GPU-order matrices
    new_to_old = mesh.resort()
    want = np.argsort(O.morton_codes(prev_gpu, mesh_data.bounding_sphere), kind="stable").astype(np.uint32)
    assert np.array_equal(new_to_old, want), "device order differs from the oracle's stable Morton order"
    dev = h.vg.debug_cells_device()
    host, gpu_mats = h.vg.debug_scene()
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32)), "device cells differ from the host's"
    h.scene, h.mats, h.orders = O.scene_from_spec(spec.meshes, [moved], h.flags, orders_in=[mesh.gpu_to_input])
    assert np.array_equal(gpu_mats, h.mats)
    ocells = np.asarray(h.scene.keep[-1]).reshape(-1, 8)
    assert np.array_equal(dev.view(np.uint32), ocells.view(np.uint32)), "device cells differ from the oracle's"
    assert dev[:, 3].sum() < 0.5 * before_cells[:, 3].sum(), "re-sorted cells are compact again"
    for t in (0.8, 2.0):
        h.compare(cam, engine.ViewParams(error_threshold=t, shadow_sweep=(5.0, -10.0, 2.0)))
