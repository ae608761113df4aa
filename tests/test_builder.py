"""DAG builder invariants: the checks of the reference's tests/preprocess.test.ts:8-94 on meshes built here,
plus the fast-path bound invariants of tests/fastpath.test.ts:17-47."""
import math

import numpy as np
import pytest

from vgcut import build as B

import oracle as O


def noisy_sphere():
    # IcosahedronGeometry(1, 40) displaced by 1 + 0.1 sin(9x) cos(7y) (preprocess.test.ts:53-63); the geodesic
    # sphere here has 20 * 41^2 triangles
    pos, idx = B.gen_icosphere(41, 1.0, 0.0, 1.0, 1)
    n = 1 + 0.1 * np.sin(pos[:, 0] * 9) * np.cos(pos[:, 1] * 7)
    return (pos * n[:, None]).astype(np.float32), idx


def small_terrain():
    return B.gen_terrain(100.0, 64, 4.0, 0.2, 0.13)


def check_dag(name, pos, idx, **opts):
    d = B.build_virtual_mesh(pos, idx, **opts)
    b = d.meshlet_bounds.reshape(-1, 16)
    info = d.meshlet_info.reshape(-1, 4)
    assert d.meshlet_count > 0, name
    assert d.stats["lodLevels"] > 1, f"{name}: more than one LOD level"
    assert d.stats["leafTriangles"] == len(idx) // 3, f"{name}: leaf level covers every input triangle"
    assert np.all(b[:, 9] >= b[:, 8]), f"{name}: parent error >= own error"
    assert np.all((info[:, 0] > 0) & (info[:, 0] <= 128)), f"{name}: 1..128 triangles per meshlet"
    assert int((b[:, 9] >= 1e30).sum()) == d.stats["rootMeshlets"], f"{name}: root count matches stats"
    # packed meshlet triangles decode to the flat index list
    for i in range(d.meshlet_count):
        tc, fi, _, vo = info[i]
        p = d.meshlet_triangles[fi // 3: fi // 3 + tc]
        for k in range(3):
            local = (p >> (8 * k)) & 255
            assert np.array_equal(d.meshlet_vertices[vo + local], d.indices[fi + np.arange(tc) * 3 + k]), name
    # meshlets sorted by level, levels contiguous
    assert np.all(np.diff(info[:, 2].astype(np.int64)) >= 0)
    lr = d.level_ranges.reshape(-1, 2)
    assert lr[0, 0] == 0 and np.all(lr[1:, 0] == lr[:-1, 0] + lr[:-1, 1]) and lr[-1].sum() == d.meshlet_count
    return d


@pytest.mark.parametrize("name,maker", [("noisy sphere", noisy_sphere), ("terrain", small_terrain),
                                        ("box lattice", lambda: B.gen_box_lattice(8, 6, 1.0, 3))])
def test_dag_invariants(name, maker):
    pos, idx = maker()
    check_dag(name, pos, idx)


def test_complete_cut_at_distances():
    """A complete cut at 5 distances (preprocess.test.ts:83-86)."""
    pos, idx = B.gen_box_lattice(10, 5, 4.0, 9)
    d = check_dag("lattice", pos, idx)
    for distance in [5, 20, 60, 200, 800]:
        view = np.eye(4)
        view[:3, 3] = (0, -8, -distance)
        sel = O.select_cut(d, view.T.reshape(-1), 1000.0, 0.1, 1.0)
        assert len(O.verify_cut_coverage(d, sel)) == 0
        assert len(O.verify_cut_overlap(d, sel)) == 0


def test_group_size_option():
    pos, idx = small_terrain()
    for g in (4, 8, 32):
        d = check_dag(f"terrain g{g}", pos, idx, group_size=g)
        assert d.meshlet_count > d.stats["leafMeshlets"]


def test_fastpath_bound_invariants(terrain):
    """cullBoundsSphere / lodBoundsSphere enclose their members and levelGuardErrors are the per-level extremes
    (fastpath.test.ts:17-47)."""
    d = terrain
    b = d.meshlet_bounds.reshape(-1, 16).astype(np.float64)
    C = d.cull_bounds_sphere.astype(np.float64)
    assert np.all(np.linalg.norm(b[:, 12:15] - C[:3], axis=1) + b[:, 15] <= C[3])
    L = d.lod_bounds_sphere.astype(np.float64)
    assert np.all(np.linalg.norm(b[:, 0:3] - L[:3], axis=1) + b[:, 3] <= L[3])
    nonroot = b[:, 9] < 1e29
    assert np.all(np.linalg.norm(b[nonroot, 4:7] - L[:3], axis=1) + b[nonroot, 7] <= L[3])
    lr = d.level_ranges.reshape(-1, 2)
    for l, (s, n) in enumerate(lr):
        assert d.level_guard_errors[l * 2] == b[s:s + n, 8].max().astype(np.float32)
        assert d.level_guard_errors[l * 2 + 1] == b[s:s + n, 9].min().astype(np.float32)
        assert d.level_errors[l * 2] == b[s:s + n, 8].min().astype(np.float32)
        assert d.level_errors[l * 2 + 1] == b[s:s + n, 9].max().astype(np.float32)


def test_builder_rejects_bad_input():
    with pytest.raises(RuntimeError):
        B.build_virtual_mesh(np.zeros((3, 3), np.float32), np.array([0, 1], np.uint32))
    with pytest.raises(RuntimeError):
        B.build_virtual_mesh(np.zeros((3, 3), np.float32), np.array([0, 1, 7], np.uint32))


def test_generators_are_seeded():
    a = B.gen_icosphere(10, 1.0, 0.02, 3.0, 5)
    b = B.gen_icosphere(10, 1.0, 0.02, 3.0, 5)
    c = B.gen_icosphere(10, 1.0, 0.02, 3.0, 6)
    assert np.array_equal(a[0], b[0]) and not np.array_equal(a[0], c[0])
    assert len(a[1]) // 3 == 20 * 10 * 10
    r1, r2 = B.Mulberry32(42), B.Mulberry32(42)
    assert [r1() for _ in range(5)] == [r2() for _ in range(5)]
